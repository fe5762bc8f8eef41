// Turn-leaf value network: a 5-layer MLP (2706 -> 4 x 1024 GELU -> 2652) trained and run on
// the device with the tcgen05 GEMM of mlp_gemm.cuh (BF16 operands, FP32 accumulation),
// fused epilogues (bias + GELU, bias, GELU derivative), an MSE loss kernel, bias-gradient
// reductions and Adam on FP32 master weights. The backward GEMMs read transposed operands
// (activations for the weight gradients, weights for the input gradients) MN-major, straight
// from their row-major arrays.
//
// Input per sample: both players' ranges over the 1326 hands, the 4 turn-board cards as a
// 52-wide 0/1 vector, pot and stack scaled to [0, 1] (pot / 200, stack / (10 pot)).
// Output: both players' counterfactual values per hand divided by the pot.
// Shapes are padded for the GEMM tiles: input 2706 -> 2816 columns, output 2652 -> 2816 (11
// tiles of 256 columns; the padded weights and biases stay zero, as their gradients are zero).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "../../include/pokerrust_b200.h"
#include "mlp_gemm.cuh"
#include "trace.h"

namespace prb {
namespace mlp {

using gemm::bf16;

constexpr int kIn = 2706, kInPad = 2816, kHid = 1024, kOut = 2652, kOutPad = 2816;
constexpr int kLayers = 5;
constexpr int kK[kLayers] = {kInPad, kHid, kHid, kHid, kHid};       // padded fan-in
constexpr int kN[kLayers] = {kHid, kHid, kHid, kHid, kOutPad};      // padded fan-out
constexpr int kKLive[kLayers] = {kIn, kHid, kHid, kHid, kHid};
constexpr int kNLive[kLayers] = {kHid, kHid, kHid, kHid, kOut};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// ---- GEMM epilogues (called with 32 accumulator values of one row per thread) ----
// When a thread's 32 values are 32 consecutive columns of one row (the tcgen05.ld
// 32dp32b32x layout), the epilogues move them with 16-byte loads and stores.
template <class P>
__device__ __forceinline__ bool row_run(P const &pos, int *m, int *n) {
    *m = cute::get<0>(pos(0));
    *n = cute::get<1>(pos(0));
    bool ok = true;
#pragma unroll
    for (int i = 1; i < 32; i++) ok &= cute::get<0>(pos(i)) == *m && cute::get<1>(pos(i)) == *n + i;
    return ok;
}

__device__ __forceinline__ uint4 pack8(const float *v) {
    uint4 u;
    uint32_t w[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const bf16 lo(v[2 * k]), hi(v[2 * k + 1]);
        w[k] = (uint32_t)lo.raw() | ((uint32_t)hi.raw() << 16);
    }
    u.x = w[0];
    u.y = w[1];
    u.z = w[2];
    u.w = w[3];
    return u;
}

__device__ __forceinline__ void unpack8(uint4 u, float *v) {
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[2 * k] = float(bf16::bitcast((uint16_t)(w[k] & 0xFFFF)));
        v[2 * k + 1] = float(bf16::bitcast((uint16_t)(w[k] >> 16)));
    }
}
struct EpiBiasGelu {  // Z = acc + b, H = gelu(Z), both bf16
    const float *bias;
    bf16 *Z, *H;
    int ld;
    template <class R, class P>
    __device__ void operator()(R const &reg, P const &pos, int m0, int n0, int) const {
        int mr, nr;
        if (cute::size(reg) == 32 && row_run(pos, &mr, &nr)) {
            const int m = m0 + mr, n = n0 + nr;
            float z[32], h[32];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const float4 bq = *reinterpret_cast<const float4 *>(bias + n + 4 * q);
                z[4 * q] = reg(4 * q) + bq.x;
                z[4 * q + 1] = reg(4 * q + 1) + bq.y;
                z[4 * q + 2] = reg(4 * q + 2) + bq.z;
                z[4 * q + 3] = reg(4 * q + 3) + bq.w;
            }
#pragma unroll
            for (int i = 0; i < 32; i++) h[i] = gelu(z[i]);
            uint4 *zo = reinterpret_cast<uint4 *>(Z + (size_t)m * ld + n);
            uint4 *ho = reinterpret_cast<uint4 *>(H + (size_t)m * ld + n);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                zo[q] = pack8(z + 8 * q);
                ho[q] = pack8(h + 8 * q);
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < cute::size(reg); i++) {
            const int m = m0 + cute::get<0>(pos(i)), n = n0 + cute::get<1>(pos(i));
            const float z = reg(i) + bias[n];
            Z[(size_t)m * ld + n] = bf16(z);
            H[(size_t)m * ld + n] = bf16(gelu(z));
        }
    }
};
struct EpiBiasF32 {  // Y = acc + b (f32)
    const float *bias;
    float *Y;
    int ld;
    template <class R, class P>
    __device__ void operator()(R const &reg, P const &pos, int m0, int n0, int) const {
        int mr, nr;
        if (cute::size(reg) == 32 && row_run(pos, &mr, &nr)) {
            const int m = m0 + mr, n = n0 + nr;
            float4 *yo = reinterpret_cast<float4 *>(Y + (size_t)m * ld + n);
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const float4 bq = *reinterpret_cast<const float4 *>(bias + n + 4 * q);
                yo[q] = make_float4(reg(4 * q) + bq.x, reg(4 * q + 1) + bq.y, reg(4 * q + 2) + bq.z,
                                    reg(4 * q + 3) + bq.w);
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < cute::size(reg); i++) {
            const int m = m0 + cute::get<0>(pos(i)), n = n0 + cute::get<1>(pos(i));
            Y[(size_t)m * ld + n] = reg(i) + bias[n];
        }
    }
};
struct EpiGeluGrad {  // dZ = acc * gelu'(Z), bf16
    const bf16 *Z;
    bf16 *dZ;
    int ld;
    template <class R, class P>
    __device__ void operator()(R const &reg, P const &pos, int m0, int n0, int) const {
        int mr, nr;
        if (cute::size(reg) == 32 && row_run(pos, &mr, &nr)) {
            const size_t at = (size_t)(m0 + mr) * ld + (n0 + nr);
            const uint4 *zi = reinterpret_cast<const uint4 *>(Z + at);
            uint4 *dzo = reinterpret_cast<uint4 *>(dZ + at);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float z[8], g[8];
                unpack8(zi[q], z);
#pragma unroll
                for (int i = 0; i < 8; i++) g[i] = reg(8 * q + i) * gelu_grad(z[i]);
                dzo[q] = pack8(g);
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < cute::size(reg); i++) {
            const int m = m0 + cute::get<0>(pos(i)), n = n0 + cute::get<1>(pos(i));
            const size_t at = (size_t)m * ld + n;
            dZ[at] = bf16(reg(i) * gelu_grad(float(Z[at])));
        }
    }
};
struct EpiStore {  // D = acc (f32); split-K part z goes to D + z * zstride
    float *D;
    int ld;
    size_t zstride;
    template <class R, class P>
    __device__ void operator()(R const &reg, P const &pos, int m0, int n0, int z) const {
        float *D = this->D + (size_t)z * zstride;
        int mr, nr;
        if (cute::size(reg) == 32 && row_run(pos, &mr, &nr)) {
            float4 *o = reinterpret_cast<float4 *>(D + (size_t)(m0 + mr) * ld + (n0 + nr));
#pragma unroll
            for (int q = 0; q < 8; q++) o[q] = make_float4(reg(4 * q), reg(4 * q + 1), reg(4 * q + 2), reg(4 * q + 3));
            return;
        }
#pragma unroll
        for (int i = 0; i < cute::size(reg); i++) {
            const int m = m0 + cute::get<0>(pos(i)), n = n0 + cute::get<1>(pos(i));
            D[(size_t)m * ld + n] = reg(i);
        }
    }
};

// ---- element-wise kernels ----
// inputs: ranges [n][2][1326], boards (4 cards) [n], scalars [n][2] -> X [rows][kInPad] bf16
__global__ void assemble_kernel(const float *__restrict__ ranges, const unsigned long long *__restrict__ boards,
                                const float *__restrict__ scalars, bf16 *__restrict__ X, int n) {
    const int s = blockIdx.x;
    bf16 *x = X + (size_t)s * kInPad;
    for (int i = threadIdx.x; i < kInPad; i += blockDim.x) {
        float v = 0.0f;
        if (s < n) {
            if (i < 2 * 1326) v = ranges[(size_t)s * 2 * 1326 + i];
            else if (i < 2 * 1326 + 52) v = (boards[s] >> (i - 2 * 1326)) & 1ull ? 1.0f : 0.0f;
            else if (i < kIn) v = scalars[(size_t)s * 2 + (i - 2 * 1326 - 52)];
        }
        x[i] = bf16(v);
    }
}

// dY = 2 (Y - T) / (n * kOut) on live outputs of live rows (bf16), and per-block squared errors
__global__ void loss_kernel(const float *__restrict__ Y, const float *__restrict__ T, bf16 *__restrict__ dY,
                            double *__restrict__ partial, int n, int rows) {
    const int m = blockIdx.x;
    __shared__ double red[256];
    double acc = 0.0;
    const float scale = 2.0f / ((float)n * (float)kOut);
    for (int j = threadIdx.x; j < kOutPad; j += blockDim.x) {
        float g = 0.0f;
        if (m < n && j < kOut) {
            const float d = Y[(size_t)m * kOutPad + j] - T[(size_t)m * kOut + j];
            acc += (double)d * d;
            g = d * scale;
        }
        dY[(size_t)m * kOutPad + j] = bf16(g);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[m] = red[0];
    (void)rows;
}

// Bias gradients db[c] = sum over rows of G[r][c] (G: [rows][cols] bf16), in two fixed-order
// steps: kBiasChunks row chunks per column (a CTA of 64 columns, two per thread, x 8 row
// phases per chunk), then the chunks in order.
constexpr int kBiasChunks = 16;

__global__ void bias_part_kernel(const bf16 *__restrict__ G, float *__restrict__ part, int cols, int rows) {
    __shared__ float red[8][2][33];
    const int c = blockIdx.x * 64 + 2 * threadIdx.x;
    const int per = rows / kBiasChunks;
    const int r0 = blockIdx.y * per;
    float a0 = 0.0f, a1 = 0.0f;
    for (int r = r0 + threadIdx.y; r < r0 + per; r += 8) {
        const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(G + (size_t)r * cols + c);
        a0 += __low2float(v);
        a1 += __high2float(v);
    }
    red[threadIdx.y][0][threadIdx.x] = a0;
    red[threadIdx.y][1][threadIdx.x] = a1;
    __syncthreads();
    if (threadIdx.y == 0) {
        float t0 = 0.0f, t1 = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            t0 += red[i][0][threadIdx.x];
            t1 += red[i][1][threadIdx.x];
        }
        part[(size_t)blockIdx.y * cols + c] = t0;
        part[(size_t)blockIdx.y * cols + c + 1] = t1;
    }
}

__global__ void bias_sum_kernel(const float *__restrict__ part, float *__restrict__ db, int cols) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float t = 0.0f;
    for (int k = 0; k < kBiasChunks; k++) t += part[(size_t)k * cols + c];
    db[c] = t;
}

// Adam over every layer's weights and biases in one launch. Each entry is one parameter
// array; its gradient is the sum of `splits` split-K parts in part order (the weights) or
// one array (the biases). Padding (rows >= n_live or columns >= k_live) stays zero.
struct AdamEntry {
    float *w, *m1, *m2;
    const float *grad;  // [splits][rows][cols]
    bf16 *wb;           // bf16 copy, or null
    int rows, cols, n_live, k_live, splits;
};
struct AdamArgs {
    AdamEntry e[2 * kLayers];
    int count;
    float lr, b1, b2, c1, c2, eps;
};

// blockIdx.y picks the entry; CTAs stride over its rows, threads over 4-column groups
// (every padded width is a multiple of 4), so no index needs a division.
__global__ void adam_all_kernel(const __grid_constant__ AdamArgs a) {
    const AdamEntry &E = a.e[blockIdx.y];
    const size_t n = (size_t)E.rows * E.cols;
    const int cols4 = E.cols / 4;
    for (int r = blockIdx.x; r < E.rows; r += gridDim.x) {
        for (int q = threadIdx.x; q < cols4; q += blockDim.x) {
            const size_t li = (size_t)r * E.cols + 4 * q;
            float4 w = *reinterpret_cast<const float4 *>(E.w + li);
            float4 m1 = *reinterpret_cast<const float4 *>(E.m1 + li);
            float4 m2 = *reinterpret_cast<const float4 *>(E.m2 + li);
            float4 g = *reinterpret_cast<const float4 *>(E.grad + li);
            for (int z = 1; z < E.splits; z++) {
                const float4 v = *reinterpret_cast<const float4 *>(E.grad + (size_t)z * n + li);
                g.x += v.x;
                g.y += v.y;
                g.z += v.z;
                g.w += v.w;
            }
            float *wv = &w.x, *av = &m1.x, *bv = &m2.x;
            const float *gv = &g.x;
#pragma unroll
            for (int t = 0; t < 4; t++) {
                if (r >= E.n_live || 4 * q + t >= E.k_live) {
                    wv[t] = 0.0f;
                    continue;
                }
                const float m = a.b1 * av[t] + (1.0f - a.b1) * gv[t];
                const float v = a.b2 * bv[t] + (1.0f - a.b2) * gv[t] * gv[t];
                av[t] = m;
                bv[t] = v;
                wv[t] -= a.lr * ((m / a.c1) / (sqrtf(v / a.c2) + a.eps));
            }
            *reinterpret_cast<float4 *>(E.w + li) = w;
            *reinterpret_cast<float4 *>(E.m1 + li) = m1;
            *reinterpret_cast<float4 *>(E.m2 + li) = m2;
            if (E.wb) {
                const bf16 h[4] = {bf16(w.x), bf16(w.y), bf16(w.z), bf16(w.w)};
                uint2 u;
                u.x = (uint32_t)h[0].raw() | ((uint32_t)h[1].raw() << 16);
                u.y = (uint32_t)h[2].raw() | ((uint32_t)h[3].raw() << 16);
                *reinterpret_cast<uint2 *>(E.wb + li) = u;
            }
        }
    }
}

// dW = sum of the split-K parts, in part order
__global__ void split_sum_kernel(const float *__restrict__ parts, float *__restrict__ out, size_t n, int splits) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n / 4; i += (size_t)gridDim.x * blockDim.x) {
        float4 acc = reinterpret_cast<const float4 *>(parts)[i];
        for (int z = 1; z < splits; z++) {
            const float4 v = reinterpret_cast<const float4 *>(parts + (size_t)z * n)[i];
            acc.x += v.x;
            acc.y += v.y;
            acc.z += v.z;
            acc.w += v.w;
        }
        reinterpret_cast<float4 *>(out)[i] = acc;
    }
}

__global__ void to_bf16_kernel(const float *__restrict__ w, bf16 *__restrict__ wb, size_t total) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        wb[i] = bf16(w[i]);
}

__global__ void copy_out_kernel(const float *__restrict__ Y, float *__restrict__ out, int n) {
    const int m = blockIdx.x;
    if (m >= n) return;
    for (int j = threadIdx.x; j < kOut; j += blockDim.x) out[(size_t)m * kOut + j] = Y[(size_t)m * kOutPad + j];
}

struct Net {
    int rows = 0;  // batch rows (multiple of 256)
    cudaStream_t stream = nullptr;
    int *d_err = nullptr;
    // parameters (f32 master, bf16 copy), gradients, Adam moments
    float *W[kLayers] = {}, *b[kLayers] = {}, *dW[kLayers] = {}, *db[kLayers] = {};
    float *mW[kLayers] = {}, *vW[kLayers] = {}, *mb[kLayers] = {}, *vb[kLayers] = {};
    bf16 *Wb[kLayers] = {};
    // activations
    bf16 *X = nullptr;
    bf16 *Z[4] = {}, *H[4] = {}, *dZ[4] = {};
    float *Y = nullptr;
    bf16 *dY = nullptr;
    double *partial = nullptr;
    float *parts[kLayers] = {};  // per layer: split-K partial products of the weight gradients
    float *bias_parts = nullptr;  // [kBiasChunks][cols] partial bias gradients
    int step = 0;
    static constexpr int kSplits = 4;
    // GEMM form: one CTA per 128 x 256 tile (0), or the persistent form over 128 x 128 tiles
    // (1), whose epilogues overlap the next tile's main loop; both give the same bits
    int persistent = 0;

    template <int BN, gemm::UMMA::Major MA = gemm::kKMajor, gemm::UMMA::Major MB = gemm::kKMajor, class Epi>
    cudaError_t mm(const bf16 *A, const bf16 *B, int M, int N, int K, Epi epi, int splits = 1) {
        if (persistent) return gemm::run_persistent<128, MA, MB>(A, B, M, N, K, epi, d_err, stream, splits);
        return gemm::run<BN, MA, MB>(A, B, M, N, K, epi, d_err, stream, splits);
    }
    std::vector<void *> owned;

    template <class T>
    bool alloc(T **p, size_t n) {
        if (cudaMalloc((void **)p, n * sizeof(T)) != cudaSuccess) return false;
        owned.push_back(*p);
        return cudaMemsetAsync(*p, 0, n * sizeof(T), stream) == cudaSuccess;
    }
    ~Net() {
        if (stream) cudaStreamSynchronize(stream);
        for (void *p : owned) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }

    int check(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return 0;
        fprintf(stderr, "pokerrust_b200: value network: %s: %s\n", what, cudaGetErrorString(e));
        return e == cudaErrorInvalidValue ? 2 : 1;
    }

    // forward pass over X (rows), Y = output pre-loss (f32)
    int forward() {
        cudaError_t e = cudaSuccess;
        const bf16 *in = X;
        for (int l = 0; l < 4 && e == cudaSuccess; l++) {
            EpiBiasGelu epi{b[l], Z[l], H[l], kN[l]};
            e = mm<256>(in, Wb[l], rows, kN[l], kK[l], epi);
            in = H[l];
        }
        if (e == cudaSuccess) {
            EpiBiasF32 epi{b[4], Y, kOutPad};
            e = mm<256>(in, Wb[4], rows, kOutPad, kHid, epi);
        }
        return check(e, "forward");
    }

    // dW[M][N] of layer l = G^T . In over the batch (G: [rows][M], In: [rows][N], both read
    // MN-major), as kSplits split-K GEMMs (the weight-gradient GEMMs have few output tiles)
    // whose parts stay apart: Adam sums them in part order
    cudaError_t weight_grad(const bf16 *G, const bf16 *In, int M, int N, int l) {
        EpiStore epi{parts[l], N, (size_t)M * N};
        return mm<256, gemm::kMNMajor, gemm::kMNMajor>(G, In, M, N, rows, epi, kSplits);
    }

    // the gradient of layer l's weights as one array (dW[l]), from its split-K parts
    int materialize_grad(int l) {
        split_sum_kernel<<<592, 256, 0, stream>>>(parts[l], dW[l], (size_t)kN[l] * kK[l], kSplits);
        return check(cudaGetLastError(), "gradient sum");
    }

    void bias_grad(const bf16 *G, float *dbout, int cols) {
        bias_part_kernel<<<dim3(cols / 64, kBiasChunks), dim3(32, 8), 0, stream>>>(G, bias_parts, cols, rows);
        bias_sum_kernel<<<(cols + 255) / 256, 256, 0, stream>>>(bias_parts, dbout, cols);
    }

    // backward from dY (bf16), gradients into dW / db; the input gradients dZ . W read the
    // weights [out][in] MN-major
    int backward() {
        cudaError_t e = weight_grad(dY, H[3], kOutPad, kHid, 4);
        bias_grad(dY, db[4], kOutPad);
        if (e == cudaSuccess) {
            EpiGeluGrad epi{Z[3], dZ[3], kHid};
            e = mm<256, gemm::kKMajor, gemm::kMNMajor>(dY, Wb[4], rows, kHid, kOutPad, epi);
        }
        for (int l = 3; l >= 0 && e == cudaSuccess; l--) {
            e = weight_grad(dZ[l], l > 0 ? H[l - 1] : X, kHid, kK[l], l);
            bias_grad(dZ[l], db[l], kHid);
            if (e == cudaSuccess && l > 0) {
                EpiGeluGrad epi2{Z[l - 1], dZ[l - 1], kHid};
                e = mm<256, gemm::kKMajor, gemm::kMNMajor>(dZ[l], Wb[l], rows, kHid, kHid, epi2);
            }
        }
        if (e == cudaSuccess) e = cudaGetLastError();
        return check(e, "backward");
    }

    int adam(float lr) {
        step++;
        AdamArgs a{};
        a.lr = lr;
        a.b1 = 0.9f;
        a.b2 = 0.999f;
        a.eps = 1e-8f;
        a.c1 = 1.0f - powf(a.b1, (float)step);
        a.c2 = 1.0f - powf(a.b2, (float)step);
        for (int l = 0; l < kLayers; l++) {
            a.e[a.count++] = AdamEntry{W[l], mW[l], vW[l], parts[l], Wb[l], kN[l], kK[l], kNLive[l], kKLive[l], kSplits};
            a.e[a.count++] = AdamEntry{b[l], mb[l], vb[l], db[l], nullptr, 1, kN[l], 1, kNLive[l], 1};
        }
        adam_all_kernel<<<dim3(296, a.count), 256, 0, stream>>>(a);
        return check(cudaGetLastError(), "adam");
    }

    int refresh_copies() {
        for (int l = 0; l < kLayers; l++) to_bf16_kernel<<<592, 256, 0, stream>>>(W[l], Wb[l], (size_t)kN[l] * kK[l]);
        return check(cudaGetLastError(), "weights");
    }
};

uint64_t splitmix(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace mlp
}  // namespace prb

using namespace prb::mlp;

extern "C" {

void *pr_mlp_new(int rows, uint64_t seed) {
    if (rows <= 0 || rows % 256) {
        fprintf(stderr, "pokerrust_b200: value network: batch rows must be a positive multiple of 256\n");
        return nullptr;
    }
    Net *n = new Net();
    n->rows = rows;
    bool ok = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) == cudaSuccess && n->alloc(&n->d_err, 1);
    for (int l = 0; l < kLayers && ok; l++) {
        const size_t sz = (size_t)kN[l] * kK[l];
        ok = n->alloc(&n->W[l], sz) && n->alloc(&n->dW[l], sz) && n->alloc(&n->mW[l], sz) && n->alloc(&n->vW[l], sz) &&
             n->alloc(&n->Wb[l], sz) && n->alloc(&n->b[l], kN[l]) &&
             n->alloc(&n->db[l], kN[l]) && n->alloc(&n->mb[l], kN[l]) && n->alloc(&n->vb[l], kN[l]);
    }
    ok = ok && n->alloc(&n->X, (size_t)rows * kInPad) && n->alloc(&n->Y, (size_t)rows * kOutPad) &&
         n->alloc(&n->dY, (size_t)rows * kOutPad) && n->alloc(&n->partial, rows) &&
         n->alloc(&n->bias_parts, (size_t)kBiasChunks * kOutPad);
    for (int l = 0; l < kLayers && ok; l++) ok = n->alloc(&n->parts[l], (size_t)Net::kSplits * kN[l] * kK[l]);
    for (int l = 0; l < 4 && ok; l++)
        ok = n->alloc(&n->Z[l], (size_t)rows * kHid) && n->alloc(&n->H[l], (size_t)rows * kHid) &&
             n->alloc(&n->dZ[l], (size_t)rows * kHid);
    if (!ok) {
        fprintf(stderr, "pokerrust_b200: value network: allocation failed\n");
        delete n;
        return nullptr;
    }
    // He-uniform weights on the live block, zero biases
    uint64_t st = seed * 0x2545F4914F6CDD1Dull + 1;
    for (int l = 0; l < kLayers; l++) {
        std::vector<float> w((size_t)kN[l] * kK[l], 0.0f);
        const float bound = sqrtf(6.0f / (float)kKLive[l]) * (l == kLayers - 1 ? 0.5f : 1.0f);
        for (int r = 0; r < kNLive[l]; r++)
            for (int c = 0; c < kKLive[l]; c++) {
                const double u = (double)(splitmix(st) >> 11) / 9007199254740992.0;
                w[(size_t)r * kK[l] + c] = (float)((2.0 * u - 1.0) * bound);
            }
        if (cudaMemcpyAsync(n->W[l], w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, n->stream) !=
            cudaSuccess) {
            delete n;
            return nullptr;
        }
        cudaStreamSynchronize(n->stream);
    }
    if (n->refresh_copies() || cudaStreamSynchronize(n->stream) != cudaSuccess) {
        delete n;
        return nullptr;
    }
    return n;
}

void pr_mlp_free(void *net) { delete (Net *)net; }

int pr_mlp_rows(void *net) { return net ? ((Net *)net)->rows : 0; }

// GEMM form of the network's passes: 1 the persistent form, 0 one CTA per tile. Returns the
// previous setting, or -1 for a null network.
int pr_mlp_set_persistent(void *net, int on) {
    Net *n = (Net *)net;
    if (!n) return -1;
    const int was = n->persistent;
    n->persistent = on ? 1 : 0;
    return was;
}

namespace {
int load_inputs(Net *n, const float *ranges, const unsigned long long *boards, const float *scalars, int count) {
    if (count < 1 || count > n->rows) return 2;
    assemble_kernel<<<n->rows, 256, 0, n->stream>>>(ranges, boards, scalars, n->X, count);
    return n->check(cudaGetLastError(), "inputs");
}
int finish(Net *n) {
    int err = 0;
    cudaError_t e = cudaStreamSynchronize(n->stream);
    if (e == cudaSuccess) e = cudaMemcpy(&err, n->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return n->check(e, "pass");
    if (err) {
        fprintf(stderr, "pokerrust_b200: value network: a GEMM wait timed out (bits %d)\n", err);
        return 1;
    }
    return 0;
}
}  // namespace

// Inference: inputs on the device (ranges [count][2][1326], boards [count] (4-card masks),
// scalars [count][2]); out [count][2652] on the device. count <= rows.
int pr_mlp_forward(void *net, const float *ranges, const uint64_t *boards, const float *scalars, float *out,
                   int count) {
    prb::TraceRange trace("value network forward");
    Net *n = (Net *)net;
    if (!n || !ranges || !boards || !scalars || !out) return 2;
    if (int st = load_inputs(n, ranges, (const unsigned long long *)boards, scalars, count)) return st;
    if (int st = n->forward()) return st;
    copy_out_kernel<<<count, 256, 0, n->stream>>>(n->Y, out, count);
    return finish(n);
}

// One training step on `count` samples (targets [count][2652] on the device): forward, MSE
// loss, backward, Adam (lr). loss: mean squared error before the update.
int pr_mlp_train_step(void *net, const float *ranges, const uint64_t *boards, const float *scalars,
                      const float *targets, int count, float lr, double *loss) {
    prb::TraceRange trace("value network training step");
    Net *n = (Net *)net;
    if (!n || !ranges || !boards || !scalars || !targets) return 2;
    if (int st = load_inputs(n, ranges, (const unsigned long long *)boards, scalars, count)) return st;
    if (int st = n->forward()) return st;
    loss_kernel<<<n->rows, 256, 0, n->stream>>>(n->Y, targets, n->dY, n->partial, count, n->rows);
    if (int st = n->backward()) return st;
    if (lr > 0.0f)
        if (int st = n->adam(lr)) return st;
    if (int st = finish(n)) return st;
    if (loss) {
        std::vector<double> p(n->rows);
        cudaMemcpy(p.data(), n->partial, sizeof(double) * n->rows, cudaMemcpyDeviceToHost);
        double s = 0;
        for (int i = 0; i < count; i++) s += p[i];
        *loss = s / ((double)count * kOut);
    }
    return 0;
}

// Layer l's live parameters (host f32): W [n_live][k_live] (fan-out x fan-in), b [n_live];
// the gradients of the last training step in the same layout.
int pr_mlp_layer_shape(int l, int *fan_out, int *fan_in) {
    if (l < 0 || l >= kLayers) return 2;
    *fan_out = kNLive[l];
    *fan_in = kKLive[l];
    return 0;
}

namespace {
int layer_io(Net *n, int l, float *dev_w, float *dev_b, float *W, float *bias, bool to_host) {
    if (!n || l < 0 || l >= kLayers) return 2;
    cudaStreamSynchronize(n->stream);
    const int rows = kNLive[l], cols = kKLive[l];
    cudaError_t e = cudaSuccess;
    if (W) {
        if (to_host)
            e = cudaMemcpy2D(W, cols * sizeof(float), dev_w, kK[l] * sizeof(float), cols * sizeof(float), rows,
                             cudaMemcpyDeviceToHost);
        else
            e = cudaMemcpy2D(dev_w, kK[l] * sizeof(float), W, cols * sizeof(float), cols * sizeof(float), rows,
                             cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && bias)
        e = to_host ? cudaMemcpy(bias, dev_b, rows * sizeof(float), cudaMemcpyDeviceToHost)
                    : cudaMemcpy(dev_b, bias, rows * sizeof(float), cudaMemcpyHostToDevice);
    return n->check(e, "parameter copy");
}
}  // namespace

int pr_mlp_get_layer(void *net, int l, float *W, float *bias) {
    Net *n = (Net *)net;
    return n ? layer_io(n, l, n->W[l], n->b[l], W, bias, true) : 2;
}

int pr_mlp_set_layer(void *net, int l, const float *W, const float *bias) {
    Net *n = (Net *)net;
    if (!n) return 2;
    if (int st = layer_io(n, l, n->W[l], n->b[l], const_cast<float *>(W), const_cast<float *>(bias), false))
        return st;
    if (int st = n->refresh_copies()) return st;
    return finish(n);
}

int pr_mlp_get_grad(void *net, int l, float *dW, float *dbias) {
    Net *n = (Net *)net;
    if (!n || l < 0 || l >= kLayers) return 2;
    if (int st = n->materialize_grad(l)) return st;
    return layer_io(n, l, n->dW[l], n->db[l], dW, dbias, true);
}

}  // extern "C"
