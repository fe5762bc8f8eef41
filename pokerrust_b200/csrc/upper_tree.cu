// The preflop, flop and turn tree of the fixed-flop game on the device.
//
// Same arithmetic as the host traversal in game.cu (state.rs:219-376, strategy.rs:37-82,
// permutation_handler.rs:7-34), organised level by level: a top-down sweep computes the
// reach vectors of both players at every node (children's ranges = parent's ranges, the
// actor's scaled by the regret-matched strategy; chance nodes mask the new board cards) and
// gathers the river roots' ranges into the river solver's input rows; a bottom-up sweep
// combines child values (strategy-weighted sum, or max for a best response, at the
// updater's nodes; plain sum at the opponent's), evaluates folds, averages the chance
// nodes and updates regrets and average-strategy sums. One CTA per node, threads over the
// 1326 hands; every kernel of a half-iteration goes on one stream, so the whole iteration
// can be captured into a CUDA graph.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "layout.h"
#include "upper_tree.h"

namespace prb {
namespace {

constexpr int UT = 256;

template <typename T>
__device__ __forceinline__ T neg_inf();
template <>
__device__ __forceinline__ float neg_inf<float>() {
    return -__int_as_float(0x7f800000);
}
template <>
__device__ __forceinline__ double neg_inf<double>() {
    return -__longlong_as_double(0x7ff0000000000000ll);
}

// Products rounded on their own, never fused into a following add: the host traversal
// (game.cu) rounds every product, and the two sweeps then agree bit for bit.
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }

__device__ __forceinline__ unsigned long long hand_mask(int h) {
    int c1, c2;
    // h = c1 + c2 (c2 - 1) / 2; c2 from the inverse of the triangular numbers
    c2 = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)h)) * 0.5f);
    while (c2 * (c2 - 1) / 2 > h) c2--;
    while ((c2 + 1) * c2 / 2 <= h) c2++;
    c1 = h - c2 * (c2 - 1) / 2;
    return (1ull << c1) | (1ull << c2);
}

// Regret matching of one hand at a decision node (strategy.rs:68-81).
// Decision nodes have at most 3 children; the loops over them unroll so that the per-hand
// strategy stays in registers.
constexpr int kMaxKids = 3;

template <typename T>
__device__ __forceinline__ void match(const float *reg, int n, int h, T *p) {
    T r[kMaxKids];
    T sum = T(0);
#pragma unroll
    for (int k = 0; k < kMaxKids; k++) {
        r[k] = k < n ? T(reg[(size_t)k * kHands + h]) : T(0);
        if (k < n) sum += r[k];
    }
#pragma unroll
    for (int k = 0; k < kMaxKids; k++) p[k] = sum <= T(1e-4f) ? T(1) / T(n) : r[k] / sum;
}

template <typename T>
__global__ void __launch_bounds__(UT) down_kernel(UpperView v, const int *__restrict__ level_nodes, int upd,
                                                   T *__restrict__ R, T *__restrict__ river_opp,
                                                   float *__restrict__ river_own) {
    const int n = level_nodes[blockIdx.x];
    const DevNode nd = v.nodes[n];
    const T *rs = R + (size_t)n * 2 * kRangeStride;  // [0] small blind, [1] big blind
    const T *rb = rs + kRangeStride;
    if (nd.kind == kUDecide) {
        const float *reg = v.regrets + nd.regret;
        for (int h = threadIdx.x; h < kHands; h += UT) {
            T p[kMaxKids];
            match(reg, nd.nchild, h, p);
#pragma unroll
            for (int k = 0; k < kMaxKids; k++) {
                if (k >= nd.nchild) break;
                T *c = R + (size_t)v.kids[nd.first + k] * 2 * kRangeStride;
                c[h] = nd.actor == 0 ? mul(rs[h], p[k]) : rs[h];
                c[kRangeStride + h] = nd.actor == 1 ? mul(rb[h], p[k]) : rb[h];
            }
        }
    } else if (nd.kind == kUFlop || nd.kind == kUTurn) {
        for (int k = 0; k < nd.nchild; k++) {
            const int ci = v.kids[nd.first + k];
            const unsigned long long cards = v.nodes[ci].cards;
            T *c = R + (size_t)ci * 2 * kRangeStride;
            for (int h = threadIdx.x; h < kHands; h += UT) {
                const bool blocked = hand_mask(h) & cards;
                c[h] = blocked ? T(0) : rs[h];
                c[kRangeStride + h] = blocked ? T(0) : rb[h];
            }
        }
    } else if (nd.kind == kURiver) {
        // state.rs:379-387: the opponent's range is the river pass's input
        T *dst = river_opp + (size_t)nd.river * kRangeStride;
        for (int h = threadIdx.x; h < kRangeStride; h += UT) dst[h] = h < kHands ? (upd == 0 ? rb[h] : rs[h]) : T(0);
        if (river_own) {
            float *own = river_own + (size_t)nd.river * kRangeStride;
            for (int h = threadIdx.x; h < kRangeStride; h += UT)
                own[h] = h < kHands ? float(upd == 0 ? rs[h] : rb[h]) : 0.0f;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(UT) up_kernel(UpperView v, const int *__restrict__ level_nodes, int upd,
                                                 int best_response, const T *__restrict__ R,
                                                 T *__restrict__ V, const T *__restrict__ river_val,
                                                 float *__restrict__ regrets, float *__restrict__ avg) {
    const int n = level_nodes[blockIdx.x];
    const DevNode nd = v.nodes[n];
    T *out = V + (size_t)n * kRangeStride;
    const T *rs = R + (size_t)n * 2 * kRangeStride;
    const T *rb = rs + kRangeStride;
    switch (nd.kind) {
        case kURiver: {
            const T *src = river_val + (size_t)nd.river * kRangeStride;
            for (int h = threadIdx.x; h < kHands; h += UT) out[h] = src[h];
            return;
        }
        case kUSBWins:
        case kUBBWins: {
            // evaluate_fold (state.rs:456-492): total and per-card sums of the opponent range
            __shared__ T coll[52];
            __shared__ T total;
            const T *opp = upd == 0 ? rb : rs;
            for (int c = threadIdx.x; c < 52; c += UT) coll[c] = T(0);
            if (threadIdx.x == 0) total = T(0);
            __syncthreads();
            // one thread per card keeps the sums deterministic
            if (threadIdx.x < 52) {
                const int c = threadIdx.x;
                T s = T(0);
                for (int o = 0; o < 52; o++) {
                    if (o == c) continue;
                    const int h = c < o ? c + o * (o - 1) / 2 : o + c * (c - 1) / 2;
                    s += opp[h];
                }
                coll[c] = s;
            }
            if (threadIdx.x == 64) {
                T s = T(0);
                for (int h = 0; h < kHands; h++) s += opp[h];
                total = s;
            }
            __syncthreads();
            const int folder = nd.kind == kUSBWins ? 1 : 0;
            const T b = T(folder == 0 ? nd.sb : nd.bb);
            const T m = b * (upd == folder ? T(-1) : T(1));
            for (int h = threadIdx.x; h < kHands; h += UT) {
                int c1, c2;
                hand_cards(h, &c1, &c2);
                T x = total + opp[h];
                x -= coll[c1];
                x -= coll[c2];
                out[h] = mul(x, m);
            }
            return;
        }
        case kUFlop: {
            // state.rs:301-336 with permutation_handler.rs:7-34
            for (int h = threadIdx.x; h < kHands; h += UT) out[h] = T(0);
            __syncthreads();
            int count = 0;
            for (int k = 0; k < nd.nchild; k++) {
                const int ci = v.kids[nd.first + k];
                const DevNode cn = v.nodes[ci];
                const T *cv = V + (size_t)ci * kRangeStride;
                for (int p = 0; p < cn.nperm; p++) {
                    const int *map = v.perm_maps + (size_t)(cn.perm_first + p) * kHands;
                    for (int h = threadIdx.x; h < kHands; h += UT)
                        out[map[h]] += (hand_mask(h) & cn.cards) ? T(0) : cv[h];
                    __syncthreads();
                    count++;
                }
            }
            const T scale = T(1) / T(count);
            for (int h = threadIdx.x; h < kHands; h += UT) out[h] *= scale;
            return;
        }
        case kUTurn: {
            // state.rs:337-376: mean over the turn cards, in child order
            for (int h = threadIdx.x; h < kHands; h += UT) {
                T s = T(0);
                for (int k = 0; k < nd.nchild; k++) {
                    const int ci = v.kids[nd.first + k];
                    s += (hand_mask(h) & v.nodes[ci].cards) ? T(0) : V[(size_t)ci * kRangeStride + h];
                }
                out[h] = s * (T(1) / T(nd.nchild));
            }
            return;
        }
        default: {
            // decision node (state.rs:236-296)
            const bool mine = upd == nd.actor;
            float *reg = regrets + nd.regret;
            for (int h = threadIdx.x; h < kHands; h += UT) {
                T p[kMaxKids], u[kMaxKids];
                match(reg, nd.nchild, h, p);
                T acc = (mine && best_response) ? neg_inf<T>() : T(0);
#pragma unroll
                for (int k = 0; k < kMaxKids; k++) {
                    if (k >= nd.nchild) break;
                    u[k] = V[(size_t)v.kids[nd.first + k] * kRangeStride + h];
                    if (mine) acc = best_response ? (acc > u[k] ? acc : u[k]) : acc + mul(u[k], p[k]);
                    else acc += u[k];
                }
                out[h] = acc;
                if (mine && !best_response) {
                    // RegularStrategy::update_add (strategy.rs:57-66); average sums
                    const T own = nd.actor == 0 ? rs[h] : rb[h];
#pragma unroll
                    for (int k = 0; k < kMaxKids; k++) {
                        if (k >= nd.nchild) break;
                        float &r = reg[(size_t)k * kHands + h];
                        r = fmaxf(r + float(u[k] - acc), 0.0f);
                        if (avg) avg[nd.regret + (size_t)k * kHands + h] += float(mul(own, p[k]));
                    }
                }
            }
            return;
        }
    }
}

}  // namespace

template <typename T>
cudaError_t upper_down(const UpperView &v, const int *level_nodes, int count, int upd, T *R, T *river_opp,
                       float *river_own, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    down_kernel<T><<<count, UT, 0, s>>>(v, level_nodes, upd, R, river_opp, river_own);
    return cudaGetLastError();
}

template <typename T>
cudaError_t upper_up(const UpperView &v, const int *level_nodes, int count, int upd, int best_response,
                     const T *R, T *V, const T *river_val, float *regrets, float *avg, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    up_kernel<T><<<count, UT, 0, s>>>(v, level_nodes, upd, best_response, R, V, river_val, regrets, avg);
    return cudaGetLastError();
}

template cudaError_t upper_down<float>(const UpperView &, const int *, int, int, float *, float *, float *,
                                       cudaStream_t);
template cudaError_t upper_down<double>(const UpperView &, const int *, int, int, double *, double *, float *,
                                        cudaStream_t);
template cudaError_t upper_up<float>(const UpperView &, const int *, int, int, int, const float *, float *,
                                     const float *, float *, float *, cudaStream_t);
template cudaError_t upper_up<double>(const UpperView &, const int *, int, int, int, const double *, double *,
                                      const double *, float *, float *, cudaStream_t);

__global__ void set_root_ranges_kernel(float *Rf, double *Rd) {
    for (int h = threadIdx.x; h < 2 * kRangeStride; h += blockDim.x) {
        const int i = h % kRangeStride;
        if (Rf) Rf[h] = i < kHands ? 1.0f : 0.0f;
        if (Rd) Rd[h] = i < kHands ? 1.0 : 0.0;
    }
}

cudaError_t upper_set_root(float *Rf, double *Rd, cudaStream_t s) {
    set_root_ranges_kernel<<<1, 256, 0, s>>>(Rf, Rd);
    return cudaGetLastError();
}

}  // namespace prb
