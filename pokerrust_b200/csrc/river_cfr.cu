// River-subtree CFR kernel: one CTA solves one river subgame over all 48 river cards.
//
// Replaces evaluate_all / evaluate_river / evaluate_showdown / evaluate_fold /
// apply_updates of the reference (src/cuda/poker.cu:163-605) with a different
// organisation of the same arithmetic:
//
//  * Strategies are per bucket and fixed during a half-iteration (the reference defers
//    regret updates to apply_updates, poker.cu:600-602 / state.rs:429), so the reach of
//    both players at every leaf is a per-bucket table that does not depend on the river
//    card. It is built once per subgame (thread = bucket) instead of once per river.
//  * The 17 leaves (9 showdowns, 8 folds) are "channels" processed together: for every
//    live hand the opponent weight x_L(o) = range(o) * reach_L(bucket(o)) is formed for all
//    leaves from one bucket-row load.
//  * Showdown value of hand h at leaf L is
//        sum_{o worse, o shares no card with h} x_L(o) - sum_{o better, ...} x_L(o)
//    = [W(g) - B(g)] - [W_c1 - B_c1] - [W_c2 - B_c2]
//    with W/B prefix sums over the rank-sorted live hands ("rank list") and over the 46
//    live hands holding each card ("card lists"), evaluated at tie-group bounds
//    (inclusion-exclusion of blockers; state.rs:494-569, poker.cu:163-302). The scans
//    leave one value per tie group, so a hand needs five group lookups per channel.
//  * Fold value is T - C[c1] - C[c2] + x(h) (state.rs:456-492, poker.cu:305-371).
//  * Regret updates are linear in the leaf values, so the per-bucket leaf sums are
//    accumulated over all 48 rivers and the tree is walked once per subgame at the end
//    (poker.cu:450-487 accumulate per river and per node instead).
//  * Hands blocked by the board carry zero reach but the reference still adds their
//    (non-zero) counterfactual values into bucket 0 when it sums a leaf by bucket
//    (poker.cu:281-288, strategy.rs:118-126 run over all 1326 hands and blocked hands have
//    bucket 0). Over the 245 blocked hands that sum is -235 T at a showdown and +235 T at a
//    fold, T the leaf's total opponent weight; it is added in closed form.
//
// Best response (MODE kModeBR) takes the per-hand maximum over the updater's actions
// (state.rs:273-284, poker.cu:437-471) and can run in double precision (V = double), the
// only double-precision step of the solver.
//
// Shared memory is laid out at launch: the group arrays are sized by the largest tie-group
// counts of the flop's boards (BoardPack::num_groups / num_card_groups).
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "layout.h"
#include "river_cfr.h"
#include "river_tree.h"

namespace prb {

namespace {

constexpr int NT = 512;                // threads per CTA
constexpr int kGPer = 9;               // warps 0-3: rank list slots per lane (128 * 9 >= 1082)
constexpr int kCPer = 6;               // card list slots per lane (8 lanes * 6 = 48)
// Opponent-weight channels. A fold by the updater leaves the opponent's reach where the
// sibling call (a showdown) leaves it, so that fold shares the showdown's channel: per
// updater there are 9 showdown channels and 4 channels of folds by the opponent.
constexpr int kNumCh = kNumSD + kNumFold / 2;
// Opponent reach row: showdowns 0-8, pad, opponent folds 12-15 (16 values, four 16-byte
// chunks). In double precision rows are 20 wide (an odd number of 16-byte chunks, so that rows
// of different buckets start in all eight bank groups) and the first 16 values are loaded.
// In single precision the rows are kept in kPioCopies interleaved copies: chunk k of bucket b
// of copy q at chunk index (b * 4 + k) * 4 + q, which lies in bank group 4 (k & 1) + q whatever
// the bucket. Lane position p of a quarter warp reads copy p & 3 and, for p >= 4, the chunks in
// the order 1, 0, 3, 2, so the eight lanes of a quarter warp read eight bank groups at every
// load (the gathers by data-dependent bucket otherwise conflict; see pio_row).
constexpr int kPioW = 20;
constexpr int kPioLoad = 16;
constexpr int kPioCopies = 4;
constexpr int kUFCol = 12;
constexpr int kWownW = 20;             // updater reach row (CFR): showdowns 0-8, pad, the 8 folds 12-19
constexpr int kFoldCol = 12;
// Channel of fold f (0..7) for updater `upd`: fold f is at state kLeaf(kNumSD + f) and its
// folder is the player to act at its parent. A fold by the updater takes the channel of its
// sibling call, showdown f + 1; the opponent's folds get channels 9-12 in fold order.
// (Plain arithmetic, so that it folds to a constant inside unrolled loops; the static_assert
// below checks it against the tree tables.)
__host__ __device__ constexpr int folder(int f) { return (f & 1) ^ (f >> 2); }
__host__ __device__ constexpr int fold_channel(int f, int upd) {
    return folder(f) == upd ? f + 1 : kNumSD + (f >> 1);
}
__host__ __device__ constexpr int leaf_channel(int leaf, int upd) {
    return leaf < kNumSD ? leaf : fold_channel(leaf - kNumSD, upd);
}
__host__ __device__ constexpr int pio_col(int ch) { return ch < kNumSD ? ch : kUFCol + (ch - kNumSD); }
__host__ __device__ constexpr bool fold_channels_hold() {
    for (int f = 0; f < kNumFold; f++) {
        const int st = kLeaf(kNumSD + f), par = kParent(st);
        if (kActor(par) != folder(f)) return false;                      // who folds
        if (kChild(par, 0) != st || kChild(par, 1) != kLeaf(f + 1)) return false;  // fold, then call
        if (kTerm(kLeaf(f + 1)) != kShowdown) return false;
    }
    for (int k = 0; k < kNumFold / 2; k++)  // each pair of folds has one fold by each player
        if (folder(2 * k) == folder(2 * k + 1)) return false;
    return true;
}
static_assert(fold_channels_hold(), "a fold by the updater shares its sibling showdown's opponent reach");
constexpr int kOutPer = 3;             // output phase: hands per lane, in bucket order
constexpr int kOutWarps = 12;          // 12 * 32 * 3 >= 1081
constexpr int kRowW = 12;              // group rows: 9 showdown channels padded to 16-byte loads
// Card sums of the fold channels are kept in 8 copies, 16-byte chunk c of card k of copy p at
// chunk index (k * chunks + c) * 8 + p: lane position p of a quarter warp reads copy p, which
// lies in bank group p, so the per-hand card lookups never conflict.
constexpr int kCfCopies = 8;

// Byte offsets of the shared-memory arrays; computed the same way on host and device.
struct Layout {
    unsigned pio, wown, Pg, VG, VC, abar, r, own, out, Cf, Tf, Tsd, gwarp, scale, stage, stage_key, total;
};

__host__ __device__ inline unsigned take(unsigned *o, unsigned bytes) {
    const unsigned at = *o;
    *o += (bytes + 15u) & ~15u;
    return at;
}

// acc: per-bucket sums carried over the rivers (the 17 leaves, plus the updater's own range
// mass when average strategies are accumulated).
__host__ __device__ inline Layout make_layout(bool cfr, unsigned vb, unsigned groups, unsigned card_groups,
                                              unsigned acc = kNumLeaves) {
    Layout L;
    unsigned o = 0;
    L.pio = take(&o, vb == 4 ? kBuckets * kPioLoad * 4 * kPioCopies : kBuckets * kPioW * vb);
    L.wown = cfr ? take(&o, kBuckets * kWownW * 4) : 0;
    L.Pg = take(&o, (groups + 1) * kNumSD * vb);
    L.VG = take(&o, groups * kRowW * vb);
    L.VC = take(&o, card_groups * kRowW * vb);
    L.abar = cfr ? take(&o, kBuckets * acc * 4) : 0;
    L.r = take(&o, kRangeStride * vb);
    L.own = acc > kNumLeaves ? take(&o, kRangeStride * 4) : 0;
    L.out = take(&o, kRangeStride * vb);
    L.Cf = take(&o, 52 * kNumFold * vb * kCfCopies);
    L.Tf = take(&o, kNumFold * vb);
    L.Tsd = take(&o, kNumSD * vb);
    L.gwarp = take(&o, 4 * kNumCh * vb);
    L.scale = take(&o, kNumLeaves * 4);
    L.stage = cfr ? take(&o, kOutWarps * 2 * acc * 4) : 0;
    L.stage_key = cfr ? take(&o, kOutWarps * 2 * 4) : 0;
    L.total = o;
    return L;
}

template <typename V, int ACC = kNumLeaves>
struct Smem {
    V *pio;                      // opponent reach per bucket and channel (layout: kPioW)
    float (*wown)[kWownW];       // updater reach * leaf scale per bucket and leaf (CFR)
    V (*Pg)[kNumSD];             // rank-list prefix sum at each tie group's start; [G] = total
    V (*VG)[kRowW];              // W - B of each rank-list tie group
    V (*VC)[kRowW];              // W - B of each group of each card list
    float (*abar)[ACC];          // per-bucket leaf sums (and own-range mass) over rivers (CFR)
    V *r;                        // opponent range of the subgame
    float *own;                  // updater's own range (average strategies only)
    V *out;                      // updater's value, summed over rivers
    V *Cf;                       // card sums, fold channels (kCfCopies interleaved copies)
    V *Tf;                       // totals, fold channels
    V *Tsd;                      // totals, showdown channels
    V (*gwarp)[kNumCh];          // rank-list warp totals
    float *scale;                // leaf scales
    float (*stage)[2][ACC];      // bucket runs touching an output warp's ends (CFR)
    int (*stage_key)[2];

    __device__ Smem(unsigned char *base, const Layout &L)
        : pio(reinterpret_cast<V *>(base + L.pio)),
          wown(reinterpret_cast<float(*)[kWownW]>(base + L.wown)),
          Pg(reinterpret_cast<V(*)[kNumSD]>(base + L.Pg)),
          VG(reinterpret_cast<V(*)[kRowW]>(base + L.VG)),
          VC(reinterpret_cast<V(*)[kRowW]>(base + L.VC)),
          abar(reinterpret_cast<float(*)[ACC]>(base + L.abar)),
          r(reinterpret_cast<V *>(base + L.r)),
          own(reinterpret_cast<float *>(base + L.own)),
          out(reinterpret_cast<V *>(base + L.out)),
          Cf(reinterpret_cast<V *>(base + L.Cf)),
          Tf(reinterpret_cast<V *>(base + L.Tf)),
          Tsd(reinterpret_cast<V *>(base + L.Tsd)),
          gwarp(reinterpret_cast<V(*)[kNumCh]>(base + L.gwarp)),
          scale(reinterpret_cast<float *>(base + L.scale)),
          stage(reinterpret_cast<float(*)[2][ACC]>(base + L.stage)),
          stage_key(reinterpret_cast<int(*)[2]>(base + L.stage_key)) {}
};

__device__ __forceinline__ void bar_rank_list() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Loads n consecutive values (n a multiple of 4 floats / 2 doubles) with 16-byte loads.
__device__ __forceinline__ void load_row(const float *p, float *o, int n) {
    const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
    for (int i = 0; i < n / 4; i++) {
        const float4 t = q[i];
        o[4 * i] = t.x;
        o[4 * i + 1] = t.y;
        o[4 * i + 2] = t.z;
        o[4 * i + 3] = t.w;
    }
}
__device__ __forceinline__ void load_row(const double *p, double *o, int n) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
    for (int i = 0; i < n / 2; i++) {
        const double2 t = q[i];
        o[2 * i] = t.x;
        o[2 * i + 1] = t.y;
    }
}

// Bucket b's opponent reach row (kPioLoad values). Single precision: this lane's copy, with
// the chunk order of its half of the quarter warp, then the two halves' chunk pairs put back
// in place (row value i of a swapped lane arrived at position i ^ 4).
template <typename V, int ACC>
__device__ __forceinline__ void pio_row(const Smem<V, ACC> &S, int b, V row[kPioLoad]) {
    if constexpr (sizeof(V) == 4) {
        const int q = threadIdx.x & 3;
        const bool swap = (threadIdx.x >> 2) & 1;
        const float4 *base = reinterpret_cast<const float4 *>(S.pio) + (size_t)b * (4 * kPioCopies) + q;
        float raw[kPioLoad];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float4 t = base[(k ^ (swap ? 1 : 0)) * kPioCopies];
            raw[4 * k] = t.x;
            raw[4 * k + 1] = t.y;
            raw[4 * k + 2] = t.z;
            raw[4 * k + 3] = t.w;
        }
#pragma unroll
        for (int i = 0; i < kPioLoad; i++) row[i] = swap ? raw[i ^ 4] : raw[i];
    } else {
        load_row(S.pio + (size_t)b * kPioW, row, kPioLoad);
    }
}

// Writes bucket b's opponent reach row (kPioLoad values; every copy in single precision).
template <typename V, int ACC>
__device__ __forceinline__ void pio_store(Smem<V, ACC> &S, int b, const V row[kPioLoad]) {
    if constexpr (sizeof(V) == 4) {
        float4 *base = reinterpret_cast<float4 *>(S.pio) + (size_t)b * (4 * kPioCopies);
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int q = 0; q < kPioCopies; q++)
                base[k * kPioCopies + q] = make_float4(row[4 * k], row[4 * k + 1], row[4 * k + 2], row[4 * k + 3]);
    } else {
#pragma unroll
        for (int i = 0; i < kPioW; i++) S.pio[(size_t)b * kPioW + i] = i < kPioLoad ? row[i] : V(0);
    }
}

// x for all 13 channels of one list element (one bucket-row load).
template <typename V, int ACC>
__device__ __forceinline__ void elem_x(const Smem<V, ACC> &S, uint32_t e, V x[kNumCh]) {
    const int h = e & 2047;
    const int b = (e >> 11) & 255;
    const V rh = h != (int)kNoHand ? S.r[h] : V(0);
    V row[kPioLoad];
    pio_row(S, b, row);
#pragma unroll
    for (int c = 0; c < kNumCh; c++) x[c] = rh * row[pio_col(c)];
}

// The fold-channel card sums of `card` from this lane's copy (see kCfCopies).
template <typename V>
__device__ __forceinline__ void cf_row(const V *cf, int card, V out[kNumFold]) {
    constexpr int kPer = 16 / sizeof(V), kChunks = kNumFold / kPer;
    const int p = threadIdx.x & 7;
#pragma unroll
    for (int c = 0; c < kChunks; c++)
        load_row(cf + ((size_t)(card * kChunks + c) * kCfCopies + p) * kPer, out + c * kPer, kPer);
}

// Leaf values (before the leaf's bet/sign scale) of live hand l for all 17 channels:
// showdowns from the group values of the scans, folds from totals and card sums.
template <int UPD, typename V, int ACC>
__device__ __forceinline__ int hand_values(const Smem<V, ACC> &S, const BoardPack *__restrict__ pk, int l,
                                           V v[kNumLeaves]) {
    const uint4 m = __ldg(&pk->meta[l]);
    const int h = m.x & 2047;
    const int b = (m.x >> 11) & 255;
    const int c1 = (m.x >> 19) & 63;
    const int c2 = (m.x >> 25) & 63;
    const int gid = m.y, cg1 = m.z, cg2 = m.w;
    V g[kRowW], a1[kRowW], a2[kRowW];
    load_row(S.VG[gid], g, kRowW);
    load_row(S.VC[cg1], a1, kRowW);
    load_row(S.VC[cg2], a2, kRowW);
#pragma unroll
    for (int c = 0; c < kNumSD; c++) v[c] = g[c] - a1[c] - a2[c];  // (W - B): rank list minus card lists
    const V rh = S.r[h];
    V prow[kPioLoad], xf[kNumFold], ca[kNumFold], cb[kNumFold];
    pio_row(S, b, prow);
#pragma unroll
    for (int f = 0; f < kNumFold; f++) xf[f] = prow[pio_col(fold_channel(f, UPD))];
    cf_row(S.Cf, c1, ca);
    cf_row(S.Cf, c2, cb);
    V tf[kNumFold];
    load_row(S.Tf, tf, kNumFold);
#pragma unroll
    for (int f = 0; f < kNumFold; f++) v[kNumSD + f] = tf[f] - ca[f] - cb[f] + rh * xf[f];
    return h;
}

// Adds the staged warp-boundary bucket runs of the last output phase into abar, in a fixed
// order (one thread per leaf channel), so that bucket sums do not depend on scheduling.
template <int ACC>
__device__ __forceinline__ void resolve_stage(Smem<float, ACC> &S, int c) {
#pragma unroll 1
    for (int w = 0; w < kOutWarps; w++) {
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const int key = S.stage_key[w][side];
            if (key >= 0) S.abar[key][c] += S.stage[w][side][c];
        }
    }
}

template <typename V>
__device__ __forceinline__ V vmax(V a, V b) {
    return a > b ? a : b;
}

template <int MODE, typename V, bool AVG, int UPD>
__global__ void __launch_bounds__(NT, 1)
    river_kernel(const SubgameDesc *__restrict__ desc, const V *__restrict__ ranges, V *__restrict__ results,
                 float *__restrict__ regrets, const BoardPack *__restrict__ packs, unsigned long long flop,
                 int updater, int max_groups, int max_card_groups, const float *__restrict__ own_ranges,
                 float *__restrict__ avg_sums) {
    static_assert(MODE == kModeBR || sizeof(V) == 4, "CFR runs in single precision");
    static_assert(!AVG || MODE == kModeCFR, "average strategies accumulate in CFR passes");
    constexpr int ACC = kNumLeaves + (AVG ? 1 : 0);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Layout L = make_layout(MODE == kModeCFR, sizeof(V), max_groups, max_card_groups, ACC);
    Smem<V, ACC> S(smem_raw, L);
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int sg = blockIdx.x;
    const SubgameDesc d = desc[sg];
    const float bet = d.bet;
    float *greg = regrets + (size_t)sg * kEdges * kBuckets;

    // ---- subgame setup: range, per-bucket reach tables ----
    for (int i = tid; i < kRangeStride; i += NT) {
        S.r[i] = ranges[(size_t)sg * kRangeStride + i];
        S.out[i] = V(0);
        if constexpr (AVG) S.own[i] = own_ranges[(size_t)sg * kRangeStride + i];
    }
    if (tid < kNumLeaves) S.scale[tid] = leaf_scale(kLeaf(tid), updater, bet);
    if (tid < kBuckets) {
        const int b = tid;
        float reg[kEdges];
#pragma unroll
        for (int e = 0; e < kEdges; e++) reg[e] = greg[e * kBuckets + b];
        V psb[kStates], pbb[kStates];
        psb[1] = V(1);
        pbb[1] = V(1);
#pragma unroll
        for (int di = 0; di < kNumDecision; di++) {
            const int s = kDecision(di);
            const int nk = kNChild(s);
            V sum = V(0);
#pragma unroll
            for (int k = 0; k < 3; k++)
                if (k < nk) sum += V(reg[kEdge(s, k)]);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                if (k < nk) {
                    // regret matching with the reference's cutoff (strategy.rs:138-146,
                    // poker.cu:492-510)
                    const V sig = sum <= V(1e-4f) ? V(1) / V(nk) : V(reg[kEdge(s, k)]) / sum;
                    const int c = kChild(s, k);
                    if (kActor(s) == 0) {
                        psb[c] = psb[s] * sig;
                        pbb[c] = pbb[s];
                    } else {
                        pbb[c] = pbb[s] * sig;
                        psb[c] = psb[s];
                    }
                }
            }
        }
        V prow[kPioLoad];
#pragma unroll
        for (int i = 0; i < kPioLoad; i++) prow[i] = V(0);
#pragma unroll
        for (int Lf = 0; Lf < kNumLeaves; Lf++) {
            const int s = kLeaf(Lf);
            const int col = Lf < kNumSD ? Lf : kFoldCol + (Lf - kNumSD);
            // showdowns and the opponent's folds; an updater's fold has its showdown's value
            if (Lf < kNumSD || leaf_channel(Lf, UPD) >= kNumSD)
                prow[pio_col(leaf_channel(Lf, UPD))] = UPD == 0 ? pbb[s] : psb[s];
            if constexpr (MODE == kModeCFR) {
                S.wown[b][col] = float(updater == 0 ? psb[s] : pbb[s]) * leaf_scale(s, updater, bet);
                S.abar[b][Lf] = 0.0f;
            }
        }
        pio_store(S, b, prow);
        if constexpr (AVG) S.abar[b][kNumLeaves] = 0.0f;
        if constexpr (MODE == kModeCFR) {
#pragma unroll
            for (int i = kNumSD; i < kFoldCol; i++) S.wown[b][i] = 0.0f;
        }
    }
    __syncthreads();

    // ---- the 48 river cards ----
    int rc_done = 0;
    for (int rc = 0; rc < 52; rc++) {
        const unsigned long long rb = 1ull << rc;
        if (rb & d.board4) continue;
        const int slot = pair_index((d.board4 | rb) ^ flop);
        const BoardPack *__restrict__ pk = packs + slot;
        __syncthreads();  // previous river's readers are done with Pg, VC, Cf, Tf
        if constexpr (MODE == kModeCFR) {
            if (warp == NT / 32 - 1 && lane < ACC && rc_done > 0) resolve_stage(S, lane);
        }
        rc_done++;

        if (warp < 4) {
            // rank list: lane g holds slots [9g, 9g + 9); writes the prefix sum at every
            // tie-group start (and the total at [G])
            const int g = tid;
            uint32_t ge[kGPer];
            V tot[kNumCh];
#pragma unroll
            for (int c = 0; c < kNumCh; c++) tot[c] = V(0);
#pragma unroll
            for (int i = 0; i < kGPer; i++) {
                const int s = g * kGPer + i;
                const uint32_t e = s < kLive ? __ldg(&pk->gelem[s]) : kNoHand;
                ge[i] = e;
                V x[kNumCh];
                elem_x(S, e, x);
                if ((e & 2047) != kNoHand && (e & kGroupStart)) {
                    V *dst = S.Pg[e >> 20];
#pragma unroll
                    for (int c = 0; c < kNumSD; c++) dst[c] = tot[c];  // lane-local part
                }
#pragma unroll
                for (int c = 0; c < kNumCh; c++) tot[c] += x[c];
            }
            V inc[kNumCh];
#pragma unroll
            for (int c = 0; c < kNumCh; c++) inc[c] = tot[c];
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                for (int c = 0; c < kNumCh; c++) {
                    const V t = __shfl_up_sync(0xffffffffu, inc[c], off);
                    if (lane >= off) inc[c] += t;
                }
            }
            if (lane == 31) {
#pragma unroll
                for (int c = 0; c < kNumCh; c++) S.gwarp[warp][c] = inc[c];
            }
            bar_rank_list();
            V offs[kNumSD];
            V total[kNumCh];
#pragma unroll
            for (int c = 0; c < kNumCh; c++) {
                V before = V(0), all = V(0);
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    const V v = S.gwarp[w][c];
                    if (w < warp) before += v;
                    all += v;
                }
                total[c] = all;
                if (c < kNumSD) offs[c] = before + inc[c] - tot[c];
            }
#pragma unroll
            for (int i = 0; i < kGPer; i++) {
                const uint32_t e = ge[i];
                if ((e & 2047) != kNoHand && (e & kGroupStart)) {
                    V *dst = S.Pg[e >> 20];
#pragma unroll
                    for (int c = 0; c < kNumSD; c++) dst[c] += offs[c];
                }
            }
            const int G = pk->num_groups;
            if (tid == 0) {
#pragma unroll
                for (int c = 0; c < kNumSD; c++) {
                    S.Pg[G][c] = total[c];
                    S.Tsd[c] = total[c];
                }
#pragma unroll
                for (int f = 0; f < kNumFold; f++) S.Tf[f] = total[fold_channel(f, UPD)];
                if constexpr (MODE == kModeCFR) {
                    // blocked hands' contribution to bucket 0 (see the file comment)
#pragma unroll
                    for (int c = 0; c < kNumLeaves; c++)
                        S.abar[0][c] += (c < kNumSD ? -235.0f : 235.0f) * total[leaf_channel(c, UPD)];
                }
            }
            // W - B of every tie group: prefix at its start + prefix at its end - total
            bar_rank_list();
            for (int gg = g; gg < G; gg += 128) {
#pragma unroll
                for (int c = 0; c < kNumSD; c++) S.VG[gg][c] = S.Pg[gg][c] + S.Pg[gg + 1][c] - total[c];
            }
        } else {
            // card lists: 8 lanes per list, 6 slots per lane, 4 lists per warp. Each group of
            // a list gets VC = W - B = prefix(start) + prefix(end) - list total.
            const unsigned FULL = 0xffffffffu;
            const int cw = warp - 4;
            const int sub = lane >> 3;       // list within the warp
            const int sl = lane & 7;         // lane within the list
            const int li = cw * 4 + sub;     // card list index (48 >= 47)
            const bool active = li < kNumLists;
            uint32_t ce[kCPer];
            V xs[kCPer][kNumSD];
            V tot[kNumCh];
#pragma unroll
            for (int c = 0; c < kNumCh; c++) tot[c] = V(0);
#pragma unroll
            for (int i = 0; i < kCPer; i++) {
                const int j = sl * kCPer + i;
                const uint32_t e = (active && j < kListLen) ? __ldg(&pk->celem[li * kLSlots + j]) : kNoHand;
                ce[i] = e;
                V x[kNumCh];
                elem_x(S, e, x);
#pragma unroll
                for (int c = 0; c < kNumCh; c++) tot[c] += x[c];
#pragma unroll
                for (int c = 0; c < kNumSD; c++) xs[i][c] = x[c];
            }
            V inc[kNumCh];
#pragma unroll
            for (int c = 0; c < kNumCh; c++) inc[c] = tot[c];
#pragma unroll
            for (int off = 1; off < 8; off <<= 1) {
#pragma unroll
                for (int c = 0; c < kNumCh; c++) {
                    const V t = __shfl_up_sync(FULL, inc[c], off);
                    if (sl >= off) inc[c] += t;
                }
            }
            {
                // the list total of each fold channel, written by the list's 8 lanes, lane sl
                // into copy sl
                V cf[kNumFold];
#pragma unroll
                for (int f = 0; f < kNumFold; f++) cf[f] = __shfl_sync(FULL, inc[fold_channel(f, UPD)], lane | 7);
                if (active) {
                    constexpr int kPer = 16 / sizeof(V), kChunks = kNumFold / kPer;
                    const int card = pk->list_card[li];
#pragma unroll
                    for (int c = 0; c < kChunks; c++) {
                        V *dst = S.Cf + ((size_t)(card * kChunks + c) * kCfCopies + sl) * kPer;
#pragma unroll
                        for (int q = 0; q < kPer; q++) dst[q] = cf[c * kPer + q];
                    }
                }
            }
            V run[kNumSD], Tc[kNumSD];
#pragma unroll
            for (int c = 0; c < kNumSD; c++) {
                run[c] = inc[c] - tot[c];
                Tc[c] = __shfl_sync(FULL, inc[c], lane | 7);
            }
            bool open = false, any = false;
            int cgo = 0;
            V Wo[kNumSD], Ff[kNumSD];
#pragma unroll
            for (int c = 0; c < kNumSD; c++) Wo[c] = Ff[c] = V(0);
#pragma unroll
            for (int i = 0; i < kCPer; i++) {
                const uint32_t e = ce[i];
                if ((e & 2047) != kNoHand && (e & kGroupStart)) {
                    if (open) {
                        V *dst = S.VC[cgo];
#pragma unroll
                        for (int c = 0; c < kNumSD; c++) dst[c] = Wo[c] + run[c] - Tc[c];
                    }
                    if (!any) {
#pragma unroll
                        for (int c = 0; c < kNumSD; c++) Ff[c] = run[c];
                        any = true;
                    }
                    open = true;
                    cgo = e >> 20;
#pragma unroll
                    for (int c = 0; c < kNumSD; c++) Wo[c] = run[c];
                }
#pragma unroll
                for (int c = 0; c < kNumSD; c++) run[c] += xs[i][c];
            }
            // the group still open at this lane's end closes at the next lane of the list that
            // starts a group, or at the end of the list
            const unsigned m = __ballot_sync(FULL, any);
            const unsigned later = (m >> (lane & ~7)) & 0xffu & ~((2u << sl) - 1u);
            const int nxt = later ? (lane & ~7) + __ffs(later) - 1 : lane;
#pragma unroll
            for (int c = 0; c < kNumSD; c++) {
                const V f = __shfl_sync(FULL, Ff[c], nxt);
                if (open) S.VC[cgo][c] = Wo[c] + (later ? f : Tc[c]) - Tc[c];
            }
        }
        __syncthreads();

        // ---- per live hand, in bucket order: root value and per-bucket leaf sums ----
        if (warp < kOutWarps) {
            const unsigned FULL = 0xffffffffu;
            float F[ACC], Lr[ACC];  // first run / last run of this lane's hands
            int nr = 0, kf = -1, kl = -1;
            if constexpr (MODE == kModeCFR) {
#pragma unroll
                for (int c = 0; c < ACC; c++) F[c] = Lr[c] = 0.0f;
            }
#pragma unroll
            for (int i = 0; i < kOutPer; i++) {
                const int j = tid * kOutPer + i;
                const uint32_t be = j < kLive ? __ldg(&pk->border[j]) : (kNoBucket << 16);
                const int key = be >> 16;
                if (key == (int)kNoBucket) continue;
                V v[ACC];
                const int h = hand_values<UPD>(S, pk, be & 0xffff, v);
                if constexpr (AVG) v[kNumLeaves] = S.own[h];
                if constexpr (MODE == kModeCFR) {
                    float w[kWownW];
                    load_row(S.wown[key], w, kWownW);
                    float acc = 0.0f;
#pragma unroll
                    for (int c = 0; c < kNumSD; c++) acc += v[c] * w[c];
#pragma unroll
                    for (int f = 0; f < kNumFold; f++) acc += v[kNumSD + f] * w[kFoldCol + f];
                    S.out[h] += acc;
                    // runs of equal buckets; a run strictly inside the lane is a whole bucket
                    if (nr == 0) {
                        kf = kl = key;
                        nr = 1;
#pragma unroll
                        for (int c = 0; c < ACC; c++) F[c] = v[c];
                    } else if (key == kl) {
                        if (nr == 1) {
#pragma unroll
                            for (int c = 0; c < ACC; c++) F[c] += v[c];
                        } else {
#pragma unroll
                            for (int c = 0; c < ACC; c++) Lr[c] += v[c];
                        }
                    } else {
                        if (nr >= 2) {
#pragma unroll
                            for (int c = 0; c < ACC; c++) S.abar[kl][c] += Lr[c];
                        }
#pragma unroll
                        for (int c = 0; c < ACC; c++) Lr[c] = v[c];
                        kl = key;
                        nr = nr + 1;
                    }
                } else {
                    V A[kStates];
#pragma unroll
                    for (int Lf = 0; Lf < kNumLeaves; Lf++) A[kLeaf(Lf)] = v[Lf] * V(S.scale[Lf]);
#pragma unroll
                    for (int di = kNumDecision - 1; di >= 0; di--) {
                        const int s = kDecision(di);
                        const int nk = kNChild(s);
                        V acc = A[kChild(s, 0)];
                        if (kActor(s) == updater) {
#pragma unroll
                            for (int k = 1; k < 3; k++)
                                if (k < nk) acc = vmax(acc, A[kChild(s, k)]);
                        } else {
#pragma unroll
                            for (int k = 1; k < 3; k++)
                                if (k < nk) acc += A[kChild(s, k)];
                        }
                        A[s] = acc;
                    }
                    S.out[h] += A[1];
                }
            }
            if constexpr (MODE == kModeCFR) {
                // segmented reduction of bucket runs across the lanes of the warp; runs that
                // touch the warp's first or last hand are staged for resolve_stage
                const bool single = nr <= 1;
                const int kfirst = nr > 0 ? kf : -1 - lane;  // unique keys for empty lanes
                const int klast = nr > 0 ? kl : -1 - lane;
                const int prev_kl = __shfl_up_sync(FULL, klast, 1);
                const bool join = lane > 0 && kfirst == prev_kl;
                const bool link = single && join;
                const unsigned starts = __ballot_sync(FULL, !link);
                const int seg_start = 31 - __clz(starts & (FULL >> (31 - lane)));
                float R[ACC];
#pragma unroll
                for (int c = 0; c < ACC; c++) R[c] = single ? F[c] : Lr[c];
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                    for (int c = 0; c < ACC; c++) {
                        const float t = __shfl_up_sync(FULL, R[c], off);
                        if (lane - off >= seg_start) R[c] += t;
                    }
                }
                float Cin[ACC];
#pragma unroll
                for (int c = 0; c < ACC; c++) {
                    const float t = __shfl_up_sync(FULL, R[c], 1);
                    Cin[c] = join ? t : 0.0f;
                }
                const bool next_join = __shfl_down_sync(FULL, (int)join, 1) && lane < 31;
                const unsigned ends = __ballot_sync(FULL, !single || !next_join);
                const int hend = __ffs(ends) - 1;
                if (lane == 31) S.stage_key[warp][1] = -1;
                if (lane == hend) S.stage_key[warp][0] = -1;
                __syncwarp();
                if (nr > 0) {
                    if (!single) {
                        // first run ends in this lane
                        if (lane == hend) {
                            S.stage_key[warp][0] = kfirst;
#pragma unroll
                            for (int c = 0; c < ACC; c++) S.stage[warp][0][c] = Cin[c] + F[c];
                        } else {
#pragma unroll
                            for (int c = 0; c < ACC; c++) S.abar[kfirst][c] += Cin[c] + F[c];
                        }
                        // last run (R == Lr here) ends here unless the next lane joins it
                        if (lane == 31) {
                            S.stage_key[warp][1] = klast;
#pragma unroll
                            for (int c = 0; c < ACC; c++) S.stage[warp][1][c] = R[c];
                        } else if (!next_join) {
#pragma unroll
                            for (int c = 0; c < ACC; c++) S.abar[klast][c] += R[c];
                        }
                    } else if (!next_join) {
                        // the lane's only run ends here, total R
                        if (lane == hend) {
                            S.stage_key[warp][0] = klast;
#pragma unroll
                            for (int c = 0; c < ACC; c++) S.stage[warp][0][c] = R[c];
                        } else if (lane == 31) {
                            S.stage_key[warp][1] = klast;
#pragma unroll
                            for (int c = 0; c < ACC; c++) S.stage[warp][1][c] = R[c];
                        } else {
#pragma unroll
                            for (int c = 0; c < ACC; c++) S.abar[klast][c] += R[c];
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    if constexpr (MODE == kModeCFR) {
        if (warp == NT / 32 - 1 && lane < ACC) resolve_stage(S, lane);
        __syncthreads();
    }

    // ---- results (state.rs:431 / poker.cu:603: mean over the 48 rivers) ----
    {
        V *dst = results + (size_t)sg * kRangeStride;
        const V inv = V(1) / V(48);
        for (int i = tid; i < kRangeStride; i += NT) dst[i] = i < kHands ? S.out[i] * inv : V(0);
    }

    // ---- regret update, once per subgame (poker.cu:450-487,524-574) ----
    if constexpr (MODE == kModeCFR) {
        if (tid < kBuckets) {
            const int b = tid;
            float reg[kEdges];
#pragma unroll
            for (int e = 0; e < kEdges; e++) reg[e] = greg[e * kBuckets + b];
            if constexpr (AVG) {
                // average-strategy sums: own range mass of the bucket over the rivers, times the
                // updater's reach into the state, times the action probability (current regrets)
                float reach[kStates];
                reach[1] = S.abar[b][kNumLeaves];
                float *gavg = avg_sums + (size_t)sg * kEdges * kBuckets;
#pragma unroll
                for (int di = 0; di < kNumDecision; di++) {
                    const int s = kDecision(di);
                    const int nk = kNChild(s);
                    float sum = 0.0f;
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        if (k < nk) sum += reg[kEdge(s, k)];
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        if (k < nk) {
                            const float sig = sum <= 1e-4f ? 1.0f / (float)nk : reg[kEdge(s, k)] / sum;
                            const int c = kChild(s, k);
                            reach[c] = kActor(s) == updater ? reach[s] * sig : reach[s];
                            if (kActor(s) == updater) gavg[kEdge(s, k) * kBuckets + b] += reach[s] * sig;
                        }
                    }
                }
            }
            float A[kStates];
#pragma unroll
            for (int Lf = 0; Lf < kNumLeaves; Lf++) A[kLeaf(Lf)] = S.abar[b][Lf] * S.scale[Lf];
#pragma unroll
            for (int di = kNumDecision - 1; di >= 0; di--) {
                const int s = kDecision(di);
                const int nk = kNChild(s);
                if (kActor(s) == updater) {
                    float sum = 0.0f;
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        if (k < nk) sum += reg[kEdge(s, k)];
                    float node = 0.0f;
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        if (k < nk) {
                            const float sig = sum <= 1e-4f ? 1.0f / (float)nk : reg[kEdge(s, k)] / sum;
                            node += sig * A[kChild(s, k)];
                        }
                    }
                    A[s] = node;
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        if (k < nk) {
                            const int e = kEdge(s, k);
                            reg[e] = fmaxf(reg[e] + (A[kChild(s, k)] - node), 0.0f);
                            greg[e * kBuckets + b] = reg[e];
                        }
                    }
                } else {
                    float node = 0.0f;
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        if (k < nk) node += A[kChild(s, k)];
                    A[s] = node;
                }
            }
        }
    }
}

template <int MODE, typename V, bool AVG, int UPD>
cudaError_t launch_upd(const SubgameDesc *desc, int n, const V *ranges, V *results, float *regrets,
                       const BoardPack *packs, unsigned long long flop, int max_groups, int max_card_groups,
                       const float *own, float *avg, size_t smem, cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(river_kernel<MODE, V, AVG, UPD>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    river_kernel<MODE, V, AVG, UPD><<<n, NT, smem, stream>>>(desc, ranges, results, regrets, packs, flop, UPD,
                                                             max_groups, max_card_groups, own, avg);
    return cudaGetLastError();
}

template <int MODE, typename V, bool AVG>
cudaError_t launch_one(const SubgameDesc *desc, int n, const V *ranges, V *results, float *regrets,
                       const BoardPack *packs, unsigned long long flop, int updater, int max_groups,
                       int max_card_groups, const float *own, float *avg, cudaStream_t stream) {
    const Layout L = make_layout(MODE == kModeCFR, sizeof(V), max_groups, max_card_groups,
                                 kNumLeaves + (AVG ? 1 : 0));
    if (L.total > 227u * 1024u) return cudaErrorInvalidConfiguration;
    if (updater == 0)
        return launch_upd<MODE, V, AVG, 0>(desc, n, ranges, results, regrets, packs, flop, max_groups,
                                           max_card_groups, own, avg, L.total, stream);
    return launch_upd<MODE, V, AVG, 1>(desc, n, ranges, results, regrets, packs, flop, max_groups, max_card_groups,
                                       own, avg, L.total, stream);
}

}  // namespace

size_t river_smem_bytes(int mode, int fp64, int max_groups, int max_card_groups) {
    return make_layout(mode == kModeCFR, fp64 ? 8 : 4, max_groups, max_card_groups,
                       mode == kModeCFR ? kNumLeaves + 1 : kNumLeaves)
        .total;
}

cudaError_t launch_river(int mode, const SubgameDesc *desc, int n, const float *ranges, float *results,
                         float *regrets, const BoardPack *packs, unsigned long long flop, int updater,
                         int max_groups, int max_card_groups, const float *own_ranges, float *avg_sums,
                         cudaStream_t stream) {
    if (mode == kModeCFR && own_ranges && avg_sums)
        return launch_one<kModeCFR, float, true>(desc, n, ranges, results, regrets, packs, flop, updater,
                                                 max_groups, max_card_groups, own_ranges, avg_sums, stream);
    if (mode == kModeCFR)
        return launch_one<kModeCFR, float, false>(desc, n, ranges, results, regrets, packs, flop, updater,
                                                  max_groups, max_card_groups, nullptr, nullptr, stream);
    return launch_one<kModeBR, float, false>(desc, n, ranges, results, regrets, packs, flop, updater,
                                             max_groups, max_card_groups, nullptr, nullptr, stream);
}

cudaError_t launch_river_br64(const SubgameDesc *desc, int n, const double *ranges, double *results,
                              float *regrets, const BoardPack *packs, unsigned long long flop, int updater,
                              int max_groups, int max_card_groups, cudaStream_t stream) {
    return launch_one<kModeBR, double, false>(desc, n, ranges, results, regrets, packs, flop, updater,
                                              max_groups, max_card_groups, nullptr, nullptr, stream);
}

}  // namespace prb
