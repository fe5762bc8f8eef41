// Small helpers shared by the kernels and the host code.
#pragma once
#include <stdint.h>

#include "layout.h"

namespace prb {

__host__ __device__ inline int ctz64(unsigned long long x) {
#ifdef __CUDA_ARCH__
    return __ffsll((long long)x) - 1;
#else
    return __builtin_ctzll(x);
#endif
}

// Cards of a hand given its colex index h = c1 + c2 (c2 - 1) / 2, c1 < c2
// (src/cuda/evaluator.cuh:35-41 decodes the same index). Off the hot path.
__host__ __device__ inline void hand_cards(int h, int *c1, int *c2) {
    int b = 1;
    while ((b + 1) * b / 2 <= h) b++;
    *c2 = b;
    *c1 = h - b * (b - 1) / 2;
}

// Colex index of a 2-card set (src/cuda/evaluator.cuh:25-33).
__host__ __device__ inline int pair_index(unsigned long long set) {
    int a = ctz64(set);
    set &= set - 1;
    int b = ctz64(set);
    return a + b * (b - 1) / 2;
}

}  // namespace prb
