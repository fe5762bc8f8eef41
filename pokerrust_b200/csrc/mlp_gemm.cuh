// BF16 GEMM on the 5th-generation tensor cores (tcgen05) for the turn-leaf value network:
// D[M][N] = A[M][K] . B[N][K]^T with FP32 accumulation in tensor memory and fused
// element-wise epilogues. Each operand is K-major (stored [M][K] / [N][K], K contiguous) or
// MN-major (stored [K][M] / [K][N], M or N contiguous): the tensor cores read either
// shared-memory layout, so transposed operands need no transpose in memory.
//
// One CTA computes one 128 x BN tile. Warp 0 (one thread) streams 128 x 64 / BN x 64 tiles
// of A and B into shared memory with TMA (128-byte swizzle, 4-deep ring, no multicast); warp 1 (one thread) issues tcgen05.mma (M = 128, N = BN, K = 16 per
// instruction) into a TMEM accumulator and frees each stage with tcgen05.commit; then the
// four warps read the accumulator rows back with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31) and run the epilogue. Every mbarrier wait is bounded: on time-out the kernel
// records an error, waits (bounded) for its copies and MMAs in flight, frees TMEM and
// returns.
//
// The layouts, descriptors and TMA boxes come from CuTe's sm100 atoms
// (SM100_MMA_F16BF16_SS, UMMA::Layout_K_SW128_Atom / Layout_MN_SW128_Atom,
// make_tma_atom_A/B_sm100 with the non-multicast SM90_TMA_LOAD, SM100_TMEM_LOAD_32dp32b*).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>

#include <cutlass/cutlass.h>
#include <cute/tensor.hpp>
#include <cute/arch/tmem_allocator_sm100.hpp>
#include <cute/atom/copy_atom.hpp>
#include <cute/atom/mma_atom.hpp>
#include <cutlass/arch/barrier.h>
#include <cutlass/numeric_types.h>

namespace prb {
namespace gemm {

using namespace cute;
using bf16 = cutlass::bfloat16_t;

constexpr int kBM = 128;
constexpr int kBK = 64;
// 16 warps: warp 0 streams tiles, warp 1 issues the MMAs, and all 16 run the epilogue, the
// four warpgroups taking every fourth 32-column chunk (warp w reads TMEM lanes
// 32 (w % 4) .. 32 (w % 4) + 31), so that transcendental epilogues have warps to overlap
constexpr int kThreads = 512;
constexpr unsigned long long kWaitNs = 2000000000ull;  // give up on an mbarrier after 2 s

// Wait limit and a load to leave out, for the test of the bounded waits: with withhold_k =
// k >= 0, CTA (0, 0, 0) arms stage k % kStages for k tile k but issues no copy into it, so
// the MMA warp's wait for that stage runs out after wait_ns. Launches outside that test use
// {kWaitNs, -1}.
struct Hooks {
    unsigned long long wait_ns = kWaitNs;
    int withhold_k = -1;
};

constexpr UMMA::Major kKMajor = UMMA::Major::K;
constexpr UMMA::Major kMNMajor = UMMA::Major::MN;

// 128-byte-swizzled shared-memory atom of an operand with the given major mode, and the order
// its copies tile a (rows, K, stage) buffer: K-major atoms along the rows first; MN-major
// atoms (64 rows x 8 K) along K first, so that each 64-row block holds all 64 K values of a
// stage contiguously and one TMA box of 64 x 64 fills it
template <UMMA::Major MJ>
using SwAtom = std::conditional_t<MJ == UMMA::Major::K, UMMA::Layout_K_SW128_Atom<bf16>,
                                  UMMA::Layout_MN_SW128_Atom<bf16>>;
template <UMMA::Major MJ>
using TileOrder = std::conditional_t<MJ == UMMA::Major::K, GenColMajor, Step<_2, _1, _3>>;

template <int BN, UMMA::Major MA = kKMajor, UMMA::Major MB = kKMajor>
struct Cfg {
    // stages of the TMA ring (a 3-stage ring with two 128 x 128 CTAs per SM measured slower)
    static constexpr int kStages = 4;
    using TiledMma = decltype(make_tiled_mma(SM100_MMA_F16BF16_SS<bf16, bf16, float, kBM, BN, MA, MB>{}));
    using Tiler = Shape<Int<kBM>, Int<BN>, Int<kBK>>;
    using ShapeA = decltype(partition_shape_A(TiledMma{}, make_shape(Int<kBM>{}, Int<kBK>{})));
    using ShapeB = decltype(partition_shape_B(TiledMma{}, make_shape(Int<BN>{}, Int<kBK>{})));
    using SmemA =
        decltype(UMMA::tile_to_mma_shape(SwAtom<MA>{}, append(ShapeA{}, Int<kStages>{}), TileOrder<MA>{}));
    using SmemB =
        decltype(UMMA::tile_to_mma_shape(SwAtom<MB>{}, append(ShapeB{}, Int<kStages>{}), TileOrder<MB>{}));
    static constexpr int kBytesA = kBM * kBK * 2;
    static constexpr int kBytesB = BN * kBK * 2;

    struct Shared {
        alignas(1024) cute::ArrayEngine<bf16, cute::cosize_v<SmemA>> A;
        alignas(1024) cute::ArrayEngine<bf16, cute::cosize_v<SmemB>> B;
        alignas(8) uint64_t full[kStages];
        alignas(8) uint64_t empty[kStages];
        alignas(8) uint64_t acc;
        uint32_t tmem_base;
        int failed;
    };
    static constexpr size_t kSmem = sizeof(Shared) + 1024;  // room to align the base to 1024
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase with parity `phase` of an mbarrier; false after limit_ns of wall time.
// Each try_wait suspends for at most about a microsecond (its time hint), so the bound holds.
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t phase, unsigned long long limit_ns) {
    const uint32_t a = cute::cast_smem_ptr_to_uint(bar);
    unsigned long long start = 0;
    for (unsigned i = 0;; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(phase), "r"(1000u)
            : "memory");
        if (ok) return true;
        const unsigned long long now = global_ns();
        if (i == 0) start = now;
        else if (now - start > limit_ns) return false;
    }
}

__device__ __forceinline__ void tmem_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// Error bits written to `err` (device int) on a timed-out wait.
enum : int { kErrProducer = 1, kErrMma = 2, kErrEpilogue = 4 };

template <int BN, UMMA::Major MA, UMMA::Major MB, class TmaA, class TmaB, class Epi>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_kernel(CUTE_GRID_CONSTANT TmaA const tma_a, CUTE_GRID_CONSTANT TmaB const tma_b, int M, int N, int K,
                Epi epi, int *err, Hooks hooks) {
    using C = Cfg<BN, MA, MB>;
    extern __shared__ char smem_raw[];
    typename C::Shared &ss = *reinterpret_cast<typename C::Shared *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    // split-K: CTA z of gridDim.z covers k tiles [k_begin, k_begin + k_tiles)
    const int k_all = K / kBK;
    const int k_begin = (int)(((long long)k_all * blockIdx.z) / gridDim.z);
    const int k_tiles = (int)(((long long)k_all * (blockIdx.z + 1)) / gridDim.z) - k_begin;

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::kStages; s++) {
            cutlass::arch::ClusterTransactionBarrier::init(&ss.full[s], 1);
            cutlass::arch::ClusterBarrier::init(&ss.empty[s], 1);
        }
        cutlass::arch::ClusterBarrier::init(&ss.acc, 1);
        ss.failed = 0;
        cutlass::arch::fence_barrier_init();
    }
    if (warp == 1) {
        cute::TMEM::Allocator1Sm alloc;
        alloc.allocate(BN, &ss.tmem_base);
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();

    typename C::TiledMma tiled_mma;
    ThrMMA cta_mma = tiled_mma.get_slice(0);
    Tensor mA = tma_a.get_tma_tensor(make_shape(M, K));
    Tensor mB = tma_b.get_tma_tensor(make_shape(N, K));
    auto coord = make_coord(blockIdx.x, blockIdx.y, _);
    Tensor gA = local_tile(mA, typename C::Tiler{}, coord, Step<_1, X, _1>{});  // (BM, BK, k)
    Tensor gB = local_tile(mB, typename C::Tiler{}, coord, Step<X, _1, _1>{});  // (BN, BK, k)
    Tensor tCgA = cta_mma.partition_A(gA);
    Tensor tCgB = cta_mma.partition_B(gB);
    Tensor sA = make_tensor(make_smem_ptr(ss.A.begin()), typename C::SmemA{});
    Tensor sB = make_tensor(make_smem_ptr(ss.B.begin()), typename C::SmemB{});
    auto [tAgA, tAsA] = tma_partition(tma_a, Int<0>{}, Layout<_1>{}, group_modes<0, 3>(sA), group_modes<0, 3>(tCgA));
    auto [tBgB, tBsB] = tma_partition(tma_b, Int<0>{}, Layout<_1>{}, group_modes<0, 3>(sB), group_modes<0, 3>(tCgB));
    Tensor tCrA = cta_mma.make_fragment_A(sA);
    Tensor tCrB = cta_mma.make_fragment_B(sB);
    Tensor cC = make_identity_tensor(make_shape(Int<kBM>{}, Int<BN>{}));
    Tensor tCcC = cta_mma.partition_C(cC);
    Tensor tCtAcc = cta_mma.make_fragment_C(tCcC);
    tCtAcc.data() = ss.tmem_base;

    int issued = 0;
    if (warp == 0 && lane == 0) {
        // producer: TMA loads of A and B tiles into the stage ring
        for (int k = 0; k < k_tiles; k++) {
            const int s = k % C::kStages;
            if (k >= C::kStages && !bar_wait(&ss.empty[s], ((k / C::kStages) - 1) & 1, hooks.wait_ns)) {
                atomicOr(err, kErrProducer);
                ss.failed = 1;
                break;
            }
            cutlass::arch::ClusterTransactionBarrier::arrive_and_expect_tx(&ss.full[s], C::kBytesA + C::kBytesB);
            if (k == hooks.withhold_k && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0) {
                issued++;  // armed, never filled: the teardown's bounded wait gives it up
                continue;
            }
            copy(tma_a.with(ss.full[s]), tAgA(_, k_begin + k), tAsA(_, s));
            copy(tma_b.with(ss.full[s]), tBgB(_, k_begin + k), tBsB(_, s));
            issued++;
        }
    } else if (warp == 1) {
        // MMA issuer: one elected thread (inside the atom) per instruction
        tiled_mma.accumulate_ = UMMA::ScaleOut::Zero;
        bool ok = true;
        for (int k = 0; k < k_tiles && ok; k++) {
            const int s = k % C::kStages;
            // warp-uniform decision: the MMA and commit below are warp-collective
            if (!__all_sync(0xffffffffu, bar_wait(&ss.full[s], (k / C::kStages) & 1, hooks.wait_ns))) {
                if (lane == 0) atomicOr(err, kErrMma);
                ok = false;
                break;
            }
            tmem_fence_after_sync();
#pragma unroll
            for (int kb = 0; kb < size<2>(tCrA); kb++) {
                cute::gemm(tiled_mma, tCrA(_, _, kb, s), tCrB(_, _, kb, s), tCtAcc);
                tiled_mma.accumulate_ = UMMA::ScaleOut::One;
            }
            // tcgen05.commit from the lane that issued the MMAs (umma_arrive elects it; the
            // whole warp calls it)
            cutlass::arch::umma_arrive(&ss.empty[s]);
            __syncwarp();
        }
        cutlass::arch::umma_arrive(&ss.acc);
        __syncwarp();
    }

    __syncwarp();

    // epilogue: all warps, TMEM rows -> registers -> global, 32 columns at a time; warpgroup g
    // takes chunks g, g + 4, ...
    const bool acc_ok = __all_sync(0xffffffffu, bar_wait(&ss.acc, 0, hooks.wait_ns));  // tcgen05.ld is warp-collective
    if (!acc_ok && lane == 0) atomicOr(err, kErrEpilogue);
    tmem_fence_after_sync();
    if (acc_ok) {
        Tensor acc = tCtAcc(make_coord(_, _), 0, 0);  // (BM, BN) in TMEM
        Tensor crd = tCcC(make_coord(_, _), 0, 0);    // (BM, BN) tile coordinates
        const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
#pragma unroll 1
        for (int j = warp / 4; j < BN / 32; j += kThreads / 128) {
            Tensor acc_j = local_tile(acc, Shape<Int<kBM>, _32>{}, make_coord(0, j));
            Tensor crd_j = local_tile(crd, Shape<Int<kBM>, _32>{}, make_coord(0, j));
            auto t2r = make_tmem_copy(SM100_TMEM_LOAD_32dp32b32x{}, acc_j);
            ThrCopy thr = t2r.get_slice(threadIdx.x % 128);
            Tensor src = thr.partition_S(acc_j);
            Tensor pos = thr.partition_D(crd_j);
            Tensor reg = make_tensor<float>(shape(pos));
            copy(t2r, src, reg);
            cutlass::arch::fence_view_async_tmem_load();
            epi(reg, pos, m0, n0, (int)blockIdx.z);
        }
    }

    // teardown: copies and MMAs in flight finish before shared memory and TMEM go away
    if (warp == 0 && lane == 0 && ss.failed) {
        // only the last ring of loads can still be in flight (earlier stages were consumed)
        for (int k = issued > C::kStages ? issued - C::kStages : 0; k < issued; k++)
            bar_wait(&ss.full[k % C::kStages], (k / C::kStages) & 1, hooks.wait_ns);
    }
    if (!acc_ok) bar_wait(&ss.acc, 0, hooks.wait_ns);
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        tmem_fence_after_sync();
        cute::TMEM::Allocator1Sm alloc;
        alloc.release_allocation_lock();
        alloc.free(ss.tmem_base, BN);
    }
}

// ---- persistent form ----
// One CTA per SM walks the output tiles (tile t, t + grid, ...; a tile is (m, n, split)) with
// a double-buffered accumulator in tensor memory (2 x BN columns), so that the epilogue of
// one tile runs while the main loop of the next fills the other accumulator. Roles, 256
// threads: warp 0 streams tiles with TMA through the stage ring (stage and phase counters
// continue across tiles), warp 1 issues tcgen05.mma and commits each finished accumulator,
// warps 4-19 (four warpgroups; warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31, and
// warpgroup g takes every fourth 32-column chunk from chunk g) drain accumulators with
// tcgen05.ld through the same epilogues as gemm_kernel; warps 2-3 only take part in set-up and
// teardown. Every wait is bounded: a role whose wait runs out records its error bit and raises
// `abort`, the others stop at their next tile, and the teardown waits (bounded) for copies
// and MMAs in flight before tensor memory is freed.
constexpr int kPThreads = 640;
constexpr int kPEpiWarps = 16;

template <int BN, UMMA::Major MA, UMMA::Major MB>
struct PCfg {
    using C = Cfg<BN, MA, MB>;
    struct Shared {
        typename C::Shared core;     // stage ring, full / empty barriers, tmem_base
        alignas(8) uint64_t accf[2];  // accumulator b holds a finished tile (MMA commit)
        alignas(8) uint64_t acce[2];  // accumulator b is drained (one arrival per epilogue warp)
        alignas(8) uint64_t fin;      // every MMA issued has completed (teardown)
        int abort;
    };
    static constexpr size_t kSmem = sizeof(Shared) + 1024;
};

template <int BN, UMMA::Major MA, UMMA::Major MB, class TmaA, class TmaB, class Epi>
__global__ void __launch_bounds__(kPThreads, 1)
    gemm_persistent_kernel(CUTE_GRID_CONSTANT TmaA const tma_a, CUTE_GRID_CONSTANT TmaB const tma_b, int M, int N,
                           int K, int splits, Epi epi, int *err, unsigned long long wait_ns) {
    using C = Cfg<BN, MA, MB>;
    using PC = PCfg<BN, MA, MB>;
    extern __shared__ char smem_raw[];
    typename PC::Shared &ps = *reinterpret_cast<typename PC::Shared *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    typename C::Shared &ss = ps.core;
    volatile int *abort_flag = &ps.abort;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const int tiles_m = M / kBM, tiles_n = N / BN;
    const int tiles = tiles_m * tiles_n * splits;
    const int k_all = K / kBK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::kStages; s++) {
            cutlass::arch::ClusterTransactionBarrier::init(&ss.full[s], 1);
            cutlass::arch::ClusterBarrier::init(&ss.empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            cutlass::arch::ClusterBarrier::init(&ps.accf[b], 1);
            cutlass::arch::ClusterBarrier::init(&ps.acce[b], kPEpiWarps);
        }
        cutlass::arch::ClusterBarrier::init(&ps.fin, 1);
        ps.abort = 0;
        cutlass::arch::fence_barrier_init();
    }
    if (warp == 1) {
        cute::TMEM::Allocator1Sm alloc;
        alloc.allocate(2 * BN, &ss.tmem_base);
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();

    typename C::TiledMma tiled_mma;
    ThrMMA cta_mma = tiled_mma.get_slice(0);
    Tensor mA = tma_a.get_tma_tensor(make_shape(M, K));
    Tensor mB = tma_b.get_tma_tensor(make_shape(N, K));
    Tensor gA = local_tile(mA, typename C::Tiler{}, make_coord(_, _, _), Step<_1, X, _1>{});  // (BM, BK, m, k)
    Tensor gB = local_tile(mB, typename C::Tiler{}, make_coord(_, _, _), Step<X, _1, _1>{});  // (BN, BK, n, k)
    Tensor tCgA = cta_mma.partition_A(gA);
    Tensor tCgB = cta_mma.partition_B(gB);
    Tensor sA = make_tensor(make_smem_ptr(ss.A.begin()), typename C::SmemA{});
    Tensor sB = make_tensor(make_smem_ptr(ss.B.begin()), typename C::SmemB{});
    auto [tAgA, tAsA] = tma_partition(tma_a, Int<0>{}, Layout<_1>{}, group_modes<0, 3>(sA), group_modes<0, 3>(tCgA));
    auto [tBgB, tBsB] = tma_partition(tma_b, Int<0>{}, Layout<_1>{}, group_modes<0, 3>(sB), group_modes<0, 3>(tCgB));
    Tensor tCrA = cta_mma.make_fragment_A(sA);
    Tensor tCrB = cta_mma.make_fragment_B(sB);
    Tensor cC = make_identity_tensor(make_shape(Int<kBM>{}, Int<BN>{}));
    Tensor tCcC = cta_mma.partition_C(cC);
    Tensor tCtAcc = cta_mma.make_fragment_C(tCcC);

    // tile t -> (m tile, n tile, split); the m tile varies fastest, so CTAs that run at the
    // same time share B tiles in L2
    auto decode = [&](int t, int &mt, int &nt, int &z, int &kb, int &kn) {
        mt = t % tiles_m;
        nt = (t / tiles_m) % tiles_n;
        z = t / (tiles_m * tiles_n);
        kb = (int)(((long long)k_all * z) / splits);
        kn = (int)(((long long)k_all * (z + 1)) / splits) - kb;
    };

    int issued = 0;
    if (warp == 0 && lane == 0) {
        int it = 0;
        for (int t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x) {
            int mt, nt, z, kb, kn;
            decode(t, mt, nt, z, kb, kn);
            for (int k = 0; k < kn; k++, it++) {
                const int s = it % C::kStages;
                if (it >= C::kStages && !bar_wait(&ss.empty[s], ((it / C::kStages) - 1) & 1, wait_ns)) {
                    atomicOr(err, kErrProducer);
                    *abort_flag = 1;
                    break;
                }
                cutlass::arch::ClusterTransactionBarrier::arrive_and_expect_tx(&ss.full[s], C::kBytesA + C::kBytesB);
                copy(tma_a.with(ss.full[s]), tAgA(_, mt, kb + k), tAsA(_, s));
                copy(tma_b.with(ss.full[s]), tBgB(_, nt, kb + k), tBsB(_, s));
                issued = it + 1;
            }
        }
    } else if (warp == 1) {
        int it = 0, local = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, local++) {
            if (__any_sync(0xffffffffu, *abort_flag)) break;  // warp-uniform: the loop holds warp-collective calls
            int mt, nt, z, kb, kn;
            decode(t, mt, nt, z, kb, kn);
            const int b = local & 1;
            // the accumulator's previous tile (two tiles back) must be drained
            if (local >= 2 && !__all_sync(0xffffffffu, bar_wait(&ps.acce[b], ((local >> 1) - 1) & 1, wait_ns))) {
                if (lane == 0) atomicOr(err, kErrMma);
                *abort_flag = 1;
                break;
            }
            tmem_fence_after_sync();
            tCtAcc.data() = ss.tmem_base + (uint32_t)(b * BN);
            tiled_mma.accumulate_ = UMMA::ScaleOut::Zero;
            for (int k = 0; k < kn; k++, it++) {
                const int s = it % C::kStages;
                if (!__all_sync(0xffffffffu, bar_wait(&ss.full[s], (it / C::kStages) & 1, wait_ns))) {
                    if (lane == 0) atomicOr(err, kErrMma);
                    *abort_flag = 1;
                    ok = false;
                    break;
                }
                tmem_fence_after_sync();
#pragma unroll
                for (int q = 0; q < size<2>(tCrA); q++) {
                    cute::gemm(tiled_mma, tCrA(_, _, q, s), tCrB(_, _, q, s), tCtAcc);
                    tiled_mma.accumulate_ = UMMA::ScaleOut::One;
                }
                cutlass::arch::umma_arrive(&ss.empty[s]);
                __syncwarp();
            }
            if (!ok) break;
            cutlass::arch::umma_arrive(&ps.accf[b]);
            __syncwarp();
        }
        // every MMA issued so far completes before the teardown frees tensor memory
        cutlass::arch::umma_arrive(&ps.fin);
        __syncwarp();
    } else if (warp >= 4) {
        const int et = threadIdx.x % 128;  // thread within its epilogue warpgroup
        const int eg = (warp - 4) / 4;       // the epilogue warpgroup
        int local = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, local++) {
            if (__any_sync(0xffffffffu, *abort_flag)) break;
            int mt, nt, z, kb, kn;
            decode(t, mt, nt, z, kb, kn);
            const int b = local & 1;
            if (!__all_sync(0xffffffffu, bar_wait(&ps.accf[b], (local >> 1) & 1, wait_ns))) {
                if (lane == 0) atomicOr(err, kErrEpilogue);
                *abort_flag = 1;
                break;
            }
            tmem_fence_after_sync();
            tCtAcc.data() = ss.tmem_base + (uint32_t)(b * BN);
            Tensor acc = tCtAcc(make_coord(_, _), 0, 0);
            Tensor crd = tCcC(make_coord(_, _), 0, 0);
            const int m0 = mt * kBM, n0 = nt * BN;
#pragma unroll 1
            for (int j = eg; j < BN / 32; j += kPEpiWarps / 4) {
                Tensor acc_j = local_tile(acc, Shape<Int<kBM>, _32>{}, make_coord(0, j));
                Tensor crd_j = local_tile(crd, Shape<Int<kBM>, _32>{}, make_coord(0, j));
                auto t2r = make_tmem_copy(SM100_TMEM_LOAD_32dp32b32x{}, acc_j);
                ThrCopy thr = t2r.get_slice(et);
                Tensor src = thr.partition_S(acc_j);
                Tensor pos = thr.partition_D(crd_j);
                Tensor reg = make_tensor<float>(shape(pos));
                copy(t2r, src, reg);
                cutlass::arch::fence_view_async_tmem_load();
                epi(reg, pos, m0, n0, z);
            }
            tmem_fence_before_sync();
            __syncwarp();
            if (lane == 0) cutlass::arch::ClusterBarrier::arrive(&ps.acce[b]);
        }
    }

    __syncwarp();
    // teardown: loads and MMAs in flight finish before shared memory and TMEM go away
    if (warp == 0 && lane == 0 && *abort_flag) {
        for (int it = issued > C::kStages ? issued - C::kStages : 0; it < issued; it++)
            bar_wait(&ss.full[it % C::kStages], (it / C::kStages) & 1, wait_ns);
    }
    if (warp == 1) bar_wait(&ps.fin, 0, wait_ns);
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        tmem_fence_after_sync();
        cute::TMEM::Allocator1Sm alloc;
        alloc.release_allocation_lock();
        alloc.free(ss.tmem_base, 2 * BN);
    }
}

// The (rows x K) view of an operand: K-major [rows][K] or MN-major [K][rows] in memory.
template <UMMA::Major MJ>
inline auto operand_view(const bf16 *p, int rows, int K) {
    if constexpr (MJ == UMMA::Major::K)
        return make_tensor(make_gmem_ptr(p), make_shape(rows, K), make_stride(K, Int<1>{}));
    else
        return make_tensor(make_gmem_ptr(p), make_shape(rows, K), make_stride(Int<1>{}, rows));
}

// Launches D = A . B^T with epilogue `epi` on `stream` (host side; see gemm_kernel). MA / MB:
// the major mode of A ([M][K] or [K][M] in memory) and B ([N][K] or [K][N]).
template <int BN, UMMA::Major MA = kKMajor, UMMA::Major MB = kKMajor, class Epi>
inline cudaError_t run(const bf16 *A, const bf16 *B, int M, int N, int K, Epi epi, int *err, cudaStream_t stream,
                       int splits = 1, Hooks hooks = Hooks()) {
    using C = Cfg<BN, MA, MB>;
    if (M % kBM || N % BN || K % kBK || K <= 0 || splits < 1 || splits > K / kBK) return cudaErrorInvalidValue;
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) return cudaErrorInvalidValue;
    Tensor gA = operand_view<MA>(A, M, K);
    Tensor gB = operand_view<MB>(B, N, K);
    typename C::TiledMma mma;
    auto cluster_vmnk = tiled_divide(make_layout(Shape<_1, _1, _1>{}), make_tile(typename C::TiledMma::AtomThrID{}));
    auto tma_a = make_tma_atom_A_sm100<bf16>(SM90_TMA_LOAD{}, gA, typename C::SmemA{}(_, _, _, 0),
                                             typename C::Tiler{}, mma, cluster_vmnk);
    auto tma_b = make_tma_atom_B_sm100<bf16>(SM90_TMA_LOAD{}, gB, typename C::SmemB{}(_, _, _, 0),
                                             typename C::Tiler{}, mma, cluster_vmnk);
    auto kernel = gemm_kernel<BN, MA, MB, decltype(tma_a), decltype(tma_b), Epi>;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::kSmem);
    if (e != cudaSuccess) return e;
    dim3 grid(M / kBM, N / BN, splits);
    kernel<<<grid, kThreads, C::kSmem, stream>>>(tma_a, tma_b, M, N, K, epi, err, hooks);
    return cudaGetLastError();
}

// The persistent form of run(): one CTA per SM (at most one per tile) walks the tiles with a
// double-buffered accumulator, so epilogues overlap the next tile's main loop.
template <int BN, UMMA::Major MA = kKMajor, UMMA::Major MB = kKMajor, class Epi>
inline cudaError_t run_persistent(const bf16 *A, const bf16 *B, int M, int N, int K, Epi epi, int *err,
                                  cudaStream_t stream, int splits = 1, unsigned long long wait_ns = kWaitNs) {
    using C = Cfg<BN, MA, MB>;
    using PC = PCfg<BN, MA, MB>;
    if (M % kBM || N % BN || K % kBK || K <= 0 || splits < 1 || splits > K / kBK) return cudaErrorInvalidValue;
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) return cudaErrorInvalidValue;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    Tensor gA = operand_view<MA>(A, M, K);
    Tensor gB = operand_view<MB>(B, N, K);
    typename C::TiledMma mma;
    auto cluster_vmnk = tiled_divide(make_layout(Shape<_1, _1, _1>{}), make_tile(typename C::TiledMma::AtomThrID{}));
    auto tma_a = make_tma_atom_A_sm100<bf16>(SM90_TMA_LOAD{}, gA, typename C::SmemA{}(_, _, _, 0),
                                             typename C::Tiler{}, mma, cluster_vmnk);
    auto tma_b = make_tma_atom_B_sm100<bf16>(SM90_TMA_LOAD{}, gB, typename C::SmemB{}(_, _, _, 0),
                                             typename C::Tiler{}, mma, cluster_vmnk);
    auto kernel = gemm_persistent_kernel<BN, MA, MB, decltype(tma_a), decltype(tma_b), Epi>;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PC::kSmem);
    if (e != cudaSuccess) return e;
    const int tiles = (M / kBM) * (N / BN) * splits;
    kernel<<<std::min(tiles, sms), kPThreads, PC::kSmem, stream>>>(tma_a, tma_b, M, N, K, splits, epi, err, wait_ns);
    return cudaGetLastError();
}

}  // namespace gemm
}  // namespace prb
