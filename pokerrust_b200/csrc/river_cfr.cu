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
//    with W/B prefix sums over the rank-sorted live hands ("global list") and over the
//    46 live hands holding each card ("card lists"), evaluated at tie-group bounds
//    (inclusion-exclusion of blockers; state.rs:494-569, poker.cu:163-302).
//  * Fold value is T - C[c1] - C[c2] + x(h) (state.rs:456-492, poker.cu:305-371).
//  * Regret updates are linear in the leaf values, so the per-bucket leaf sums are
//    accumulated over all 48 rivers and the tree is walked once per subgame at the end
//    (poker.cu:450-487 accumulate per river and per node instead).
//  * Hands blocked by the board carry zero reach but the reference still adds their
//    (non-zero) counterfactual values into bucket 0 when it sums a leaf by bucket
//    (poker.cu:281-288, strategy.rs:118-126 run over all 1326 hands and blocked hands have
//    bucket 0). Over the 245 blocked hands that sum is -235 T at a showdown and +235 T at a
//    fold, T the leaf's total opponent weight; it is added in closed form.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "layout.h"
#include "river_cfr.h"
#include "river_tree.h"

namespace prb {

namespace {

constexpr int NT = 512;                // threads per CTA
constexpr int kGPer = 9;               // warps 0-3: global list slots per lane (128 * 9 >= 1082)
constexpr int kCPer = 6;               // card list slots per lane (8 lanes * 6 = 48)
constexpr int kPioW = 20;              // bucket row: SD channels 0-8, pad, fold channels 12-19
constexpr int kFoldCol = 12;
constexpr int kOutPer = 3;             // output phase: hands per lane, in bucket order
constexpr int kOutWarps = 12;          // 12 * 32 * 3 >= 1081

struct __align__(16) Smem {
    float pio[kBuckets][kPioW];    // opponent reach per bucket and leaf
    float wown[kBuckets][kPioW];   // updater reach * leaf scale per bucket and leaf
    float Pg[kMaxGroups + 1][kNumSD];      // rank-list prefix sum at each tie group's start; [G] = total
    float VC[kMaxCardGroups][kNumSD];      // W - B of each group of each card list
    float abar[kBuckets][kNumLeaves];       // per-bucket leaf sums over rivers
    float r[kRangeStride];         // opponent range of the subgame
    float out[kRangeStride];       // updater's value, summed over rivers
    float Cf[52][kNumFold];        // card sums, fold channels
    float Tf[kNumFold];            // totals, fold channels
    float Tsd[kNumSD];             // totals, showdown channels
    float gwarp[4][kNumLeaves];    // global list warp totals
    float scale[kNumLeaves];
    float stage[kOutWarps][2][kNumLeaves];  // bucket runs touching an output warp's ends
    int stage_key[kOutWarps][2];
};

__device__ __forceinline__ void bar_global_list() {
    asm volatile("bar.sync 1, 128;" ::: "memory");
}

// x for all 17 channels of one list element (bucket row load).
__device__ __forceinline__ void elem_x(const Smem &S, uint32_t e, float x[kNumLeaves]) {
    const int h = e & 2047;
    const int b = (e >> 11) & 255;
    const float rh = h != (int)kNoHand ? S.r[h] : 0.0f;
    const float4 *row = reinterpret_cast<const float4 *>(S.pio[b]);
    float4 q0 = row[0], q1 = row[1], q2 = row[2], q3 = row[3], q4 = row[4];
    x[0] = rh * q0.x; x[1] = rh * q0.y; x[2] = rh * q0.z; x[3] = rh * q0.w;
    x[4] = rh * q1.x; x[5] = rh * q1.y; x[6] = rh * q1.z; x[7] = rh * q1.w;
    x[8] = rh * q2.x;
    x[9] = rh * q3.x; x[10] = rh * q3.y; x[11] = rh * q3.z; x[12] = rh * q3.w;
    x[13] = rh * q4.x; x[14] = rh * q4.y; x[15] = rh * q4.z; x[16] = rh * q4.w;
}

// Leaf values (before the leaf's bet/sign scale) of live hand l for all 17 channels:
// showdowns from the group values of the scans, folds from totals and card sums.
__device__ __forceinline__ int hand_values(const Smem &S, const BoardPack *__restrict__ pk, int l,
                                           float v[kNumLeaves]) {
    const uint4 m = __ldg(&pk->meta[l]);
    const int h = m.x & 2047;
    const int b = (m.x >> 11) & 255;
    const int c1 = (m.x >> 19) & 63;
    const int c2 = (m.x >> 25) & 63;
    const int gid = m.y, cg1 = m.z, cg2 = m.w;
#pragma unroll
    for (int c = 0; c < kNumSD; c++) {
        // (W - B) over the rank list minus (W - B) over the two card lists
        const float wb = S.Pg[gid][c] + S.Pg[gid + 1][c] - S.Tsd[c];
        v[c] = wb - S.VC[cg1][c] - S.VC[cg2][c];
    }
    const float rh = S.r[h];
    const float4 *prow = reinterpret_cast<const float4 *>(S.pio[b]);
    const float4 f0 = prow[3], f1 = prow[4];
    const float xf[8] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w};
    const float4 *cf1 = reinterpret_cast<const float4 *>(S.Cf[c1]);
    const float4 *cf2 = reinterpret_cast<const float4 *>(S.Cf[c2]);
    const float4 a0 = cf1[0], a1 = cf1[1], b0 = cf2[0], b1 = cf2[1];
    const float ca[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float cb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
    for (int f = 0; f < kNumFold; f++) v[kNumSD + f] = S.Tf[f] - ca[f] - cb[f] + rh * xf[f];
    return h;
}

// Adds the staged warp-boundary bucket runs of the last output phase into abar, in a fixed
// order (one thread per leaf channel), so that bucket sums do not depend on scheduling.
__device__ __forceinline__ void resolve_stage(Smem &S, int c) {
#pragma unroll 1
    for (int w = 0; w < kOutWarps; w++) {
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const int key = S.stage_key[w][side];
            if (key >= 0) S.abar[key][c] += S.stage[w][side][c];
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(NT, 1)
    river_kernel(const SubgameDesc *__restrict__ desc, const float *__restrict__ ranges,
                 float *__restrict__ results, float *__restrict__ regrets,
                 const BoardPack *__restrict__ packs, unsigned long long flop, int updater) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem &S = *reinterpret_cast<Smem *>(smem_raw);
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int sg = blockIdx.x;
    const SubgameDesc d = desc[sg];
    const float bet = d.bet;
    float *greg = regrets + (size_t)sg * kEdges * kBuckets;

    // ---- subgame setup: range, per-bucket reach tables ----
    {
        const float4 *src = reinterpret_cast<const float4 *>(ranges + (size_t)sg * kRangeStride);
        float4 *dst = reinterpret_cast<float4 *>(S.r);
        float4 *o = reinterpret_cast<float4 *>(S.out);
        for (int i = tid; i < kRangeStride / 4; i += NT) {
            dst[i] = src[i];
            o[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    if (tid < kNumLeaves) S.scale[tid] = leaf_scale(kLeaf(tid), updater, bet);
    if (tid < kBuckets) {
        const int b = tid;
        float reg[kEdges];
#pragma unroll
        for (int e = 0; e < kEdges; e++) reg[e] = greg[e * kBuckets + b];
        float psb[kStates], pbb[kStates];
        psb[1] = 1.0f;
        pbb[1] = 1.0f;
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
                    // regret matching with the reference's cutoff (strategy.rs:138-146,
                    // poker.cu:492-510)
                    const float sig = sum <= 1e-4f ? 1.0f / (float)nk : reg[kEdge(s, k)] / sum;
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
        float pio_row[kPioW], wown_row[kPioW];
#pragma unroll
        for (int i = 0; i < kPioW; i++) pio_row[i] = wown_row[i] = 0.0f;
#pragma unroll
        for (int L = 0; L < kNumLeaves; L++) {
            const int s = kLeaf(L);
            const int col = L < kNumSD ? L : kFoldCol + (L - kNumSD);
            const float own = updater == 0 ? psb[s] : pbb[s];
            const float opp = updater == 0 ? pbb[s] : psb[s];
            pio_row[col] = opp;
            wown_row[col] = own * leaf_scale(s, updater, bet);
            S.abar[b][L] = 0.0f;
        }
        float4 *pr = reinterpret_cast<float4 *>(S.pio[b]);
        float4 *wr = reinterpret_cast<float4 *>(S.wown[b]);
#pragma unroll
        for (int i = 0; i < kPioW / 4; i++) {
            pr[i] = make_float4(pio_row[4 * i], pio_row[4 * i + 1], pio_row[4 * i + 2], pio_row[4 * i + 3]);
            wr[i] = make_float4(wown_row[4 * i], wown_row[4 * i + 1], wown_row[4 * i + 2], wown_row[4 * i + 3]);
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
        __syncthreads();  // previous river's readers are done with P, CP, Cf, Tf
        if (MODE == kModeCFR && warp == NT / 32 - 1 && lane < kNumLeaves && rc_done > 0) resolve_stage(S, lane);
        rc_done++;

        if (warp < 4) {
            // rank list: lane g holds slots [9g, 9g + 9); writes the prefix sum at every
            // tie-group start (and the total at [G])
            const int g = tid;
            uint32_t ge[kGPer];
            float tot[kNumLeaves];
#pragma unroll
            for (int c = 0; c < kNumLeaves; c++) tot[c] = 0.0f;
#pragma unroll
            for (int i = 0; i < kGPer; i++) {
                const int s = g * kGPer + i;
                const uint32_t e = s < kLive ? __ldg(&pk->gelem[s]) : kNoHand;
                ge[i] = e;
                float x[kNumLeaves];
                elem_x(S, e, x);
                if ((e & 2047) != kNoHand && (e & kGroupStart)) {
                    float *dst = S.Pg[e >> 20];
#pragma unroll
                    for (int c = 0; c < kNumSD; c++) dst[c] = tot[c];  // lane-local part
                }
#pragma unroll
                for (int c = 0; c < kNumLeaves; c++) tot[c] += x[c];
            }
            float inc[kNumLeaves];
#pragma unroll
            for (int c = 0; c < kNumLeaves; c++) inc[c] = tot[c];
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                for (int c = 0; c < kNumLeaves; c++) {
                    const float t = __shfl_up_sync(0xffffffffu, inc[c], off);
                    if (lane >= off) inc[c] += t;
                }
            }
            if (lane == 31) {
#pragma unroll
                for (int c = 0; c < kNumLeaves; c++) S.gwarp[warp][c] = inc[c];
            }
            bar_global_list();
            float offs[kNumSD];
            float total[kNumLeaves];
#pragma unroll
            for (int c = 0; c < kNumLeaves; c++) {
                float before = 0.0f, all = 0.0f;
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    const float v = S.gwarp[w][c];
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
                    float *dst = S.Pg[e >> 20];
#pragma unroll
                    for (int c = 0; c < kNumSD; c++) dst[c] += offs[c];
                }
            }
            if (tid == 0) {
                const int G = pk->num_groups;
#pragma unroll
                for (int c = 0; c < kNumSD; c++) {
                    S.Pg[G][c] = total[c];
                    S.Tsd[c] = total[c];
                }
#pragma unroll
                for (int f = 0; f < kNumFold; f++) S.Tf[f] = total[kNumSD + f];
                if (MODE == kModeCFR) {
                    // blocked hands' contribution to bucket 0 (see the file comment)
#pragma unroll
                    for (int c = 0; c < kNumLeaves; c++)
                        S.abar[0][c] += (c < kNumSD ? -235.0f : 235.0f) * total[c];
                }
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
            float xs[kCPer][kNumSD];
            float tot[kNumLeaves];
#pragma unroll
            for (int c = 0; c < kNumLeaves; c++) tot[c] = 0.0f;
#pragma unroll
            for (int i = 0; i < kCPer; i++) {
                const int j = sl * kCPer + i;
                const uint32_t e = (active && j < kListLen) ? __ldg(&pk->celem[li * kLSlots + j]) : kNoHand;
                ce[i] = e;
                float x[kNumLeaves];
                elem_x(S, e, x);
#pragma unroll
                for (int c = 0; c < kNumLeaves; c++) tot[c] += x[c];
#pragma unroll
                for (int c = 0; c < kNumSD; c++) xs[i][c] = x[c];
            }
            float inc[kNumLeaves];
#pragma unroll
            for (int c = 0; c < kNumLeaves; c++) inc[c] = tot[c];
#pragma unroll
            for (int off = 1; off < 8; off <<= 1) {
#pragma unroll
                for (int c = 0; c < kNumLeaves; c++) {
                    const float t = __shfl_up_sync(FULL, inc[c], off);
                    if (sl >= off) inc[c] += t;
                }
            }
            if (active && sl == 7) {
                const int card = pk->list_card[li];
#pragma unroll
                for (int f = 0; f < kNumFold; f++) S.Cf[card][f] = inc[kNumSD + f];
            }
            float run[kNumSD], Tc[kNumSD];
#pragma unroll
            for (int c = 0; c < kNumSD; c++) {
                run[c] = inc[c] - tot[c];
                Tc[c] = __shfl_sync(FULL, inc[c], lane | 7);
            }
            bool open = false, any = false;
            int cgo = 0;
            float Wo[kNumSD], Ff[kNumSD];
#pragma unroll
            for (int c = 0; c < kNumSD; c++) Wo[c] = Ff[c] = 0.0f;
#pragma unroll
            for (int i = 0; i < kCPer; i++) {
                const uint32_t e = ce[i];
                if ((e & 2047) != kNoHand && (e & kGroupStart)) {
                    if (open) {
                        float *dst = S.VC[cgo];
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
                const float f = __shfl_sync(FULL, Ff[c], nxt);
                if (open) S.VC[cgo][c] = Wo[c] + (later ? f : Tc[c]) - Tc[c];
            }
        }
        __syncthreads();

        // ---- per live hand, in bucket order: root value and per-bucket leaf sums ----
        if (warp < kOutWarps) {
            const unsigned FULL = 0xffffffffu;
            float F[kNumLeaves], L[kNumLeaves];  // first run / last run of this lane's hands
            int nr = 0, kf = -1, kl = -1;
#pragma unroll
            for (int c = 0; c < kNumLeaves; c++) F[c] = L[c] = 0.0f;
#pragma unroll
            for (int i = 0; i < kOutPer; i++) {
                const int j = tid * kOutPer + i;
                const uint32_t be = j < kLive ? __ldg(&pk->border[j]) : (kNoBucket << 16);
                const int key = be >> 16;
                if (key == (int)kNoBucket) continue;
                float v[kNumLeaves];
                const int h = hand_values(S, pk, be & 0xffff, v);
                if (MODE == kModeCFR) {
                    const float4 *wrow = reinterpret_cast<const float4 *>(S.wown[key]);
                    const float4 w0 = wrow[0], w1 = wrow[1], w2 = wrow[2], w3 = wrow[3], w4 = wrow[4];
                    float acc = v[0] * w0.x + v[1] * w0.y + v[2] * w0.z + v[3] * w0.w + v[4] * w1.x +
                                v[5] * w1.y + v[6] * w1.z + v[7] * w1.w + v[8] * w2.x;
                    acc += v[9] * w3.x + v[10] * w3.y + v[11] * w3.z + v[12] * w3.w + v[13] * w4.x +
                           v[14] * w4.y + v[15] * w4.z + v[16] * w4.w;
                    S.out[h] += acc;
                    // runs of equal buckets; a run strictly inside the lane is a whole bucket
                    if (nr == 0) {
                        kf = kl = key;
                        nr = 1;
#pragma unroll
                        for (int c = 0; c < kNumLeaves; c++) F[c] = v[c];
                    } else if (key == kl) {
                        if (nr == 1) {
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) F[c] += v[c];
                        } else {
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) L[c] += v[c];
                        }
                    } else {
                        if (nr >= 2) {
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) S.abar[kl][c] += L[c];
                        }
#pragma unroll
                        for (int c = 0; c < kNumLeaves; c++) L[c] = v[c];
                        kl = key;
                        nr = nr + 1;
                    }
                } else {
                    // best response: max over the updater's actions, sum over the opponent's
                    // (state.rs:273-284, poker.cu:437-471)
                    float A[kStates];
#pragma unroll
                    for (int Lf = 0; Lf < kNumLeaves; Lf++) A[kLeaf(Lf)] = v[Lf] * S.scale[Lf];
#pragma unroll
                    for (int di = kNumDecision - 1; di >= 0; di--) {
                        const int s = kDecision(di);
                        const int nk = kNChild(s);
                        float acc = A[kChild(s, 0)];
                        if (kActor(s) == updater) {
#pragma unroll
                            for (int k = 1; k < 3; k++)
                                if (k < nk) acc = fmaxf(acc, A[kChild(s, k)]);
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
            if (MODE == kModeCFR) {
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
                float R[kNumLeaves];
#pragma unroll
                for (int c = 0; c < kNumLeaves; c++) R[c] = single ? F[c] : L[c];
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                    for (int c = 0; c < kNumLeaves; c++) {
                        const float t = __shfl_up_sync(FULL, R[c], off);
                        if (lane - off >= seg_start) R[c] += t;
                    }
                }
                float Cin[kNumLeaves];
#pragma unroll
                for (int c = 0; c < kNumLeaves; c++) {
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
                            for (int c = 0; c < kNumLeaves; c++) S.stage[warp][0][c] = Cin[c] + F[c];
                        } else {
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) S.abar[kfirst][c] += Cin[c] + F[c];
                        }
                        // last run (R == L here) ends here unless the next lane joins it
                        if (lane == 31) {
                            S.stage_key[warp][1] = klast;
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) S.stage[warp][1][c] = R[c];
                        } else if (!next_join) {
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) S.abar[klast][c] += R[c];
                        }
                    } else if (!next_join) {
                        // the lane's only run ends here, total R
                        if (lane == hend) {
                            S.stage_key[warp][0] = klast;
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) S.stage[warp][0][c] = R[c];
                        } else if (lane == 31) {
                            S.stage_key[warp][1] = klast;
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) S.stage[warp][1][c] = R[c];
                        } else {
#pragma unroll
                            for (int c = 0; c < kNumLeaves; c++) S.abar[klast][c] += R[c];
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    if (MODE == kModeCFR) {
        if (warp == NT / 32 - 1 && lane < kNumLeaves) resolve_stage(S, lane);
        __syncthreads();
    }

    // ---- results (state.rs:431 / poker.cu:603: mean over the 48 rivers) ----
    {
        float *dst = results + (size_t)sg * kRangeStride;
        const float inv = 1.0f / 48.0f;
        for (int i = tid; i < kRangeStride; i += NT) dst[i] = i < kHands ? S.out[i] * inv : 0.0f;
    }

    // ---- regret update, once per subgame (poker.cu:450-487,524-574) ----
    if (MODE == kModeCFR && tid < kBuckets) {
        const int b = tid;
        float reg[kEdges];
#pragma unroll
        for (int e = 0; e < kEdges; e++) reg[e] = greg[e * kBuckets + b];
        float A[kStates];
#pragma unroll
        for (int L = 0; L < kNumLeaves; L++) A[kLeaf(L)] = S.abar[b][L] * S.scale[L];
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

}  // namespace

size_t river_smem_bytes() { return sizeof(Smem); }

cudaError_t launch_river(int mode, const SubgameDesc *desc, int n, const float *ranges,
                         float *results, float *regrets, const BoardPack *packs,
                         unsigned long long flop, int updater, cudaStream_t stream) {
    const size_t smem = sizeof(Smem);
    cudaError_t e;
    if (mode == kModeCFR) {
        e = cudaFuncSetAttribute(river_kernel<kModeCFR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return e;
        river_kernel<kModeCFR><<<n, NT, smem, stream>>>(desc, ranges, results, regrets, packs, flop,
                                                        updater);
    } else {
        e = cudaFuncSetAttribute(river_kernel<kModeBR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return e;
        river_kernel<kModeBR><<<n, NT, smem, stream>>>(desc, ranges, results, regrets, packs, flop,
                                                       updater);
    }
    return cudaGetLastError();
}

}  // namespace prb
