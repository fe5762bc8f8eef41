// tcgen05 BF16 GEMM launchers (mlp_gemm.cu).
#pragma once
#include <cuda_runtime.h>

namespace prb {

// D[m][n] (f32, leading dimension ldd) = sum_k A[m][k] B[n][k] for m < rows_live, n < cols_live;
// A: M x K, B: N x K, bf16, stored K-major ([M][K], [N][K]) or, with a_mn / b_mn, MN-major
// ([K][M], [K][N]); M % 128 == 0, N % bn == 0, K % 64 == 0, bn in {128, 256}. err: device
// int, error bits of timed-out waits.
cudaError_t gemm_bf16_f32(const void *A, const void *B, float *D, int M, int N, int K, int ldd, int rows_live,
                          int cols_live, int bn, int *err, cudaStream_t stream, bool a_mn = false,
                          bool b_mn = false);

}  // namespace prb
