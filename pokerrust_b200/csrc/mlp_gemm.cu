// Host launchers of the tcgen05 BF16 GEMM (mlp_gemm.cuh) and its epilogues.
#include <cuda_runtime.h>
#include <stdio.h>

#include "mlp_gemm.cuh"
#include "mlp_gemm.h"

namespace prb {
namespace gemm {

// D (f32, leading dimension ldd) = accumulator, rows < rows_live and columns < cols_live.
// A thread's 32 values that are 32 consecutive columns of one live row inside the live
// columns, on a 16-byte boundary, go out as eight 16-byte stores; others one by one.
struct EpiF32 {
    float *D;
    int ldd, rows_live, cols_live;
    template <class R, class P>
    __device__ void operator()(R const &reg, P const &pos, int m0, int n0, int) const {
        if (size(reg) == 32) {
            const int mr = get<0>(pos(0)), nr = get<1>(pos(0));
            bool run = true;
#pragma unroll
            for (int i = 1; i < 32; i++) run &= get<0>(pos(i)) == mr && get<1>(pos(i)) == nr + i;
            const int m = m0 + mr, n = n0 + nr;
            float *d = D + (size_t)m * ldd + n;
            if (run && m < rows_live && n + 32 <= cols_live && (reinterpret_cast<uintptr_t>(d) & 15) == 0) {
                float4 *o = reinterpret_cast<float4 *>(d);
#pragma unroll
                for (int q = 0; q < 8; q++) o[q] = make_float4(reg(4 * q), reg(4 * q + 1), reg(4 * q + 2), reg(4 * q + 3));
                return;
            }
        }
#pragma unroll
        for (int i = 0; i < size(reg); i++) {
            const int m = m0 + get<0>(pos(i)), n = n0 + get<1>(pos(i));
            if (m < rows_live && n < cols_live) D[(size_t)m * ldd + n] = reg(i);
        }
    }
};

// Split-K part z of D (f32, leading dimension ldd) goes to D + z * zstride.
struct EpiParts {
    float *D;
    int ldd;
    size_t zstride;
    template <class R, class P>
    __device__ void operator()(R const &reg, P const &pos, int m0, int n0, int z) const {
        float *d = D + (size_t)z * zstride;
        if (size(reg) == 32) {
            const int mr = get<0>(pos(0)), nr = get<1>(pos(0));
            bool run = true;
#pragma unroll
            for (int i = 1; i < 32; i++) run &= get<0>(pos(i)) == mr && get<1>(pos(i)) == nr + i;
            float *row = d + (size_t)(m0 + mr) * ldd + n0 + nr;
            if (run && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
                float4 *o = reinterpret_cast<float4 *>(row);
#pragma unroll
                for (int q = 0; q < 8; q++) o[q] = make_float4(reg(4 * q), reg(4 * q + 1), reg(4 * q + 2), reg(4 * q + 3));
                return;
            }
        }
#pragma unroll
        for (int i = 0; i < size(reg); i++) d[(size_t)(m0 + get<0>(pos(i))) * ldd + n0 + get<1>(pos(i))] = reg(i);
    }
};

}  // namespace gemm

namespace {
template <int BN>
cudaError_t run_majors(const gemm::bf16 *a, const gemm::bf16 *b, int M, int N, int K, gemm::EpiF32 epi, bool a_mn,
                       bool b_mn, int *err, cudaStream_t stream) {
    using gemm::kKMajor;
    using gemm::kMNMajor;
    if (!a_mn && !b_mn) return gemm::run<BN, kKMajor, kKMajor>(a, b, M, N, K, epi, err, stream);
    if (!a_mn && b_mn) return gemm::run<BN, kKMajor, kMNMajor>(a, b, M, N, K, epi, err, stream);
    if (a_mn && !b_mn) return gemm::run<BN, kMNMajor, kKMajor>(a, b, M, N, K, epi, err, stream);
    return gemm::run<BN, kMNMajor, kMNMajor>(a, b, M, N, K, epi, err, stream);
}
}  // namespace

cudaError_t gemm_bf16_f32(const void *A, const void *B, float *D, int M, int N, int K, int ldd, int rows_live,
                          int cols_live, int bn, int *err, cudaStream_t stream, bool a_mn, bool b_mn) {
    gemm::EpiF32 epi{D, ldd, rows_live, cols_live};
    const gemm::bf16 *a = reinterpret_cast<const gemm::bf16 *>(A);
    const gemm::bf16 *b = reinterpret_cast<const gemm::bf16 *>(B);
    if (bn == 256) return run_majors<256>(a, b, M, N, K, epi, a_mn, b_mn, err, stream);
    if (bn == 128) return run_majors<128>(a, b, M, N, K, epi, a_mn, b_mn, err, stream);
    return cudaErrorInvalidValue;
}

}  // namespace prb

extern "C" {

namespace {
int gemm_sync(const void *A, const void *B, float *D, int M, int N, int K, int bn, void *stream, bool a_mn,
              bool b_mn) {
    int *d_err = nullptr;
    cudaError_t e = cudaMalloc(&d_err, sizeof(int));
    if (e != cudaSuccess) return 1;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(d_err, 0, sizeof(int), s);
    e = prb::gemm_bf16_f32(A, B, D, M, N, K, N, M, N, bn, d_err, s, a_mn, b_mn);
    if (e == cudaErrorInvalidValue) {
        cudaFree(d_err);
        return 2;
    }
    int err = 0;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    if (e != cudaSuccess) {
        fprintf(stderr, "pokerrust_b200: gemm: %s\n", cudaGetErrorString(e));
        return 1;
    }
    if (err) {
        fprintf(stderr, "pokerrust_b200: gemm: a wait timed out (error bits %d)\n", err);
        return 1;
    }
    return 0;
}

}  // namespace

// D[M][N] (f32) = A[M][K] . B[N][K]^T on the tensor cores, device pointers, synchronous.
// Returns 0, 2 for bad shapes, or 1 with the kernel's error bits printed on a timed-out wait.
int pr_gemm_bf16(const void *A, const void *B, float *D, int M, int N, int K, int bn, void *stream) {
    return gemm_sync(A, B, D, M, N, K, bn, stream, false, false);
}

// The same product with either operand MN-major: a_mn = 1 reads A from [K][M] storage
// (D = A^T-stored . B^T), b_mn = 1 reads B from [K][N] storage.
int pr_gemm_bf16_major(const void *A, const void *B, float *D, int M, int N, int K, int bn, int a_mn, int b_mn,
                       void *stream) {
    return gemm_sync(A, B, D, M, N, K, bn, stream, a_mn != 0, b_mn != 0);
}

// The K-major product launched asynchronously on `stream`; err: a device int that collects
// the kernel's error bits (timed-out waits). 0 or 2 (bad shapes) or 1 (launch error).
int pr_gemm_bf16_async(const void *A, const void *B, float *D, int M, int N, int K, int bn, int *err,
                       void *stream) {
    const cudaError_t e =
        prb::gemm_bf16_f32(A, B, D, M, N, K, N, M, N, bn, err, (cudaStream_t)stream, false, false);
    return e == cudaSuccess ? 0 : (e == cudaErrorInvalidValue ? 2 : 1);
}

// The persistent form (one CTA per SM walking the tiles, double-buffered accumulator):
// D[z][M][N] (f32) = split-K part z of A . B^T, z < splits, either operand MN-major.
// Synchronous; 0, 2 for bad shapes, 1 on a CUDA error or a timed-out wait.
int pr_gemm_bf16_persistent(const void *A, const void *B, float *D, int M, int N, int K, int bn, int a_mn, int b_mn,
                            int splits, void *stream) {
    using namespace prb::gemm;
    int *d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) return 1;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(d_err, 0, sizeof(int), s);
    EpiParts epi{D, N, (size_t)M * N};
    const bf16 *a = reinterpret_cast<const bf16 *>(A);
    const bf16 *b = reinterpret_cast<const bf16 *>(B);
    cudaError_t e = cudaErrorInvalidValue;
    auto go = [&](auto bn_tag) {
        constexpr int BN = decltype(bn_tag)::value;
        if (!a_mn && !b_mn) return run_persistent<BN, kKMajor, kKMajor>(a, b, M, N, K, epi, d_err, s, splits);
        if (!a_mn && b_mn) return run_persistent<BN, kKMajor, kMNMajor>(a, b, M, N, K, epi, d_err, s, splits);
        if (a_mn && !b_mn) return run_persistent<BN, kMNMajor, kKMajor>(a, b, M, N, K, epi, d_err, s, splits);
        return run_persistent<BN, kMNMajor, kMNMajor>(a, b, M, N, K, epi, d_err, s, splits);
    };
    if (bn == 256) e = go(std::integral_constant<int, 256>{});
    else if (bn == 128) e = go(std::integral_constant<int, 128>{});
    if (e == cudaErrorInvalidValue) {
        cudaFree(d_err);
        return 2;
    }
    int err = 0;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    if (e != cudaSuccess || err) {
        fprintf(stderr, "pokerrust_b200: gemm (persistent): %s (error bits %d)\n", cudaGetErrorString(e), err);
        return 1;
    }
    return 0;
}

// The K-major persistent product launched asynchronously on `stream` (D = A . B^T, f32);
// err: a device int that collects the kernel's error bits. 0, 2 (bad shapes) or 1.
int pr_gemm_bf16_persistent_async(const void *A, const void *B, float *D, int M, int N, int K, int bn, int *err,
                                  void *stream) {
    using namespace prb::gemm;
    EpiF32 epi{D, N, M, N};
    const bf16 *a = reinterpret_cast<const bf16 *>(A);
    const bf16 *b = reinterpret_cast<const bf16 *>(B);
    cudaError_t e = cudaErrorInvalidValue;
    if (bn == 256) e = run_persistent<256>(a, b, M, N, K, epi, err, (cudaStream_t)stream);
    else if (bn == 128) e = run_persistent<128>(a, b, M, N, K, epi, err, (cudaStream_t)stream);
    return e == cudaSuccess ? 0 : (e == cudaErrorInvalidValue ? 2 : 1);
}

// Test of the bounded waits: the K-major product with wait limit `wait_ns` and, when
// withhold_k >= 0, CTA (0, 0)'s load of k tile withhold_k armed but never issued, so that its
// MMA warp's wait runs out. Synchronous; returns the kernel's error bits (0 when every wait
// was met), or -2 for bad shapes (K must span more than 4 k tiles of 64 when a load is
// withheld, so that the producer's own wait runs out too and the teardown waits for the loads
// it issued), or -1 on a CUDA error.
int pr_gemm_bf16_wait_test(const void *A, const void *B, float *D, int M, int N, int K, int bn,
                           unsigned long long wait_ns, int withhold_k, void *stream) {
    if (bn != 128 && bn != 256) return -2;
    if (withhold_k >= 0 && (K / prb::gemm::kBK <= 4 || withhold_k >= K / prb::gemm::kBK)) return -2;
    int *d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) return -1;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(d_err, 0, sizeof(int), s);
    prb::gemm::EpiF32 epi{D, N, M, N};
    prb::gemm::Hooks hooks;
    hooks.wait_ns = wait_ns;
    hooks.withhold_k = withhold_k;
    const prb::gemm::bf16 *a = reinterpret_cast<const prb::gemm::bf16 *>(A);
    const prb::gemm::bf16 *b = reinterpret_cast<const prb::gemm::bf16 *>(B);
    using prb::gemm::kKMajor;
    cudaError_t e = bn == 256 ? prb::gemm::run<256, kKMajor, kKMajor>(a, b, M, N, K, epi, d_err, s, 1, hooks)
                              : prb::gemm::run<128, kKMajor, kKMajor>(a, b, M, N, K, epi, d_err, s, 1, hooks);
    int err = 0;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    if (e == cudaErrorInvalidValue) return -2;
    return e == cudaSuccess ? err : -1;
}

}  // extern "C"
