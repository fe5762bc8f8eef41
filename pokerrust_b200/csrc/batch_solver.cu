// Batched solver of general river subgames: per-hand CFR, best response and strategy
// evaluation over many independent subgames in one persistent launch.
//
// A CTA takes subgames from a device work queue (atomicAdd on a head counter) until it is
// empty. For one subgame, the 1081 live hands are held in rank order ("positions"); a
// thread owns K consecutive positions. The bet tree (pre-order nodes) sits in shared
// memory. A pass for player p walks the tree twice per thread, with the per-hand state of
// the open path on depth-indexed stacks (thread-local memory; the innermost open node of the
// bottom-up walk in registers):
//  * top-down: reach of the opponent (times its range) and of p along the path, from
//    regret matching (or the average strategy) of the acting player; at every leaf the
//    opponent weights x(o) go to shared memory;
//  * leaves: for each leaf a CTA-wide pass turns x into p's counterfactual values:
//      showdown  stake * ([W - B] over all live hands - [W - B] over the hands holding each
//                of p's two cards), W / B = weight of strictly worse / better hands, taken
//                at the bounds of the hand's tie group (card removal by inclusion-exclusion);
//      fold      +-stake * (T - C[c1] - C[c2] + x(h)), T the total and C the per-card sums.
//    Prefix sums use a fixed summation tree (warp scans of fixed 64-hand chunks, two hands
//    per lane, and of the card lists), so results do not depend on the CTA size;
//  * bottom-up: values flow to the root; at p's nodes the CFR pass updates regrets
//    r <- max(r + v(child) - v(node), 0) (the child value is added when the child closes and
//    the node value subtracted when the node closes, so no per-child storage is needed), the
//    best response takes the maximum, the evaluation the strategy-weighted sum.
// Leaves are processed in groups sized to shared memory; both walks advance group by group.
// Average-strategy sums (avg += reach of p x action probability) are added in the top-down
// walk of CFR passes.
#include <cuda_runtime.h>
#include <stdint.h>

#include "batch_solver.h"
#include "device_common.cuh"
#include "hand_eval.cuh"

namespace prb {
namespace {

constexpr int kSetupThreads = 256;
constexpr int DS = 6;  // stack depth: trees of depth <= 5 (max_raises <= 3)

// ---------------------------------------------------------------- setup ----

__global__ void __launch_bounds__(kSetupThreads) batch_setup_kernel(const BSub *__restrict__ subs,
                                                                     BPack *__restrict__ packs,
                                                                     const float *__restrict__ ranges_in,
                                                                     float *__restrict__ ranges_pos,
                                                                     int *__restrict__ err) {
    const int s = blockIdx.x;
    const int tid = threadIdx.x;
    const unsigned long long board = subs[s].board;
    BPack *pk = packs + s;
    __shared__ unsigned long long key[2048];
    __shared__ uint16_t hand_at[kBRow];
    __shared__ uint16_t first[kBRow], last[kBRow];
    __shared__ uint8_t lo_li[kBRow], hi_li[kBRow], lo_gs[kBRow], lo_ge[kBRow], hi_gs[kBRow], hi_ge[kBRow];
    __shared__ uint8_t list_card[48];

    if (__popcll(board) != 5 || (board >> 52)) {
        if (tid == 0) atomicOr(err, 1);
        return;
    }
    for (int i = tid; i < 2048; i += kSetupThreads) {
        unsigned long long k = ~0ull;
        if (i < 1326) {
            int c1, c2;
            hand_cards(i, &c1, &c2);
            const unsigned long long hm = (1ull << c1) | (1ull << c2);
            if (!(hm & board)) k = ((unsigned long long)(hand_value(hm | board) + 1u) << 11) | (unsigned)i;
        }
        key[i] = k;
    }
    // bitonic sort, ascending: weakest hand first, ties by hand index
    for (int size = 2; size <= 2048; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (int t = tid; t < 1024; t += kSetupThreads) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool up = (i & size) == 0;
                const unsigned long long a = key[i], b = key[j];
                if ((a > b) == up) {
                    key[i] = b;
                    key[j] = a;
                }
            }
        }
    }
    __syncthreads();
    for (int p = tid; p < kBRow; p += kSetupThreads) hand_at[p] = p < kBLive ? (uint16_t)(key[p] & 2047) : 0xFFFF;
    if (tid == 0) {
        int n = 0;
        for (int c = 0; c < 52; c++)
            if (!((board >> c) & 1)) list_card[n++] = (uint8_t)c;
        list_card[47] = 0;
        // tie groups: equal hand values
        int f = 0;
        for (int p = 0; p < kBLive; p++) {
            if (p > 0 && (key[p] >> 11) != (key[p - 1] >> 11)) f = p;
            first[p] = (uint16_t)f;
        }
        int l = kBLive - 1;
        for (int p = kBLive - 1; p >= 0; p--) {
            if (p < kBLive - 1 && (key[p] >> 11) != (key[p + 1] >> 11)) l = p;
            last[p] = (uint16_t)l;
        }
        for (int p = kBLive; p < kBRow; p++) first[p] = last[p] = (uint16_t)p;
    }
    __syncthreads();
    if (tid < kBLists) {
        // card list: live hands holding the card, in rank order, and each element's tie group
        // bounds inside the list
        const int li = tid;
        const int card = list_card[li];
        uint16_t pos[kBListLen];
        int k = 0;
        for (int p = 0; p < kBLive && k < kBListLen; p++) {
            int c1, c2;
            hand_cards(hand_at[p], &c1, &c2);
            if (c1 == card || c2 == card) pos[k++] = (uint16_t)p;
        }
        if (k != kBListLen) atomicOr(err, 2);
        for (int j = 0; j < 48; j++) pk->clpos[li][j] = j < k ? pos[j] : (uint16_t)(kBRow - 1);
        int j = 0;
        while (j < k) {
            int e = j;
            while (e + 1 < k && first[pos[e + 1]] == first[pos[j]]) e++;
            for (int q = j; q <= e; q++) {
                int c1, c2;
                hand_cards(hand_at[pos[q]], &c1, &c2);
                if (c1 == card) {
                    lo_li[pos[q]] = (uint8_t)li;
                    lo_gs[pos[q]] = (uint8_t)j;
                    lo_ge[pos[q]] = (uint8_t)e;
                } else {
                    hi_li[pos[q]] = (uint8_t)li;
                    hi_gs[pos[q]] = (uint8_t)j;
                    hi_ge[pos[q]] = (uint8_t)e;
                }
            }
            j = e + 1;
        }
    }
    if (tid == kBLists) {
        for (int c = 0; c < 48; c++) pk->list_card[c] = list_card[c];
    }
    __syncthreads();
    for (int p = tid; p < kBRow; p += kSetupThreads) {
        const bool live = p < kBLive;
        pk->grp[p] = (uint32_t)first[p] | ((uint32_t)last[p] << 16);
        pk->lists[p] = live ? ((uint32_t)lo_li[p] | ((uint32_t)hi_li[p] << 8) | ((uint32_t)lo_gs[p] << 16) |
                               ((uint32_t)lo_ge[p] << 24))
                            : 0u;
        pk->lists2[p] = live ? ((uint32_t)hi_gs[p] | ((uint32_t)hi_ge[p] << 8)) : 0u;
        pk->hand[p] = hand_at[p];
    }
    for (int h = tid; h < 1328; h += kSetupThreads) pk->pos_of[h] = 0xFFFF;
    __syncthreads();
    for (int p = tid; p < kBLive; p += kSetupThreads) pk->pos_of[hand_at[p]] = (uint16_t)p;
    for (int i = tid; i < 2 * kBRow; i += kSetupThreads) {
        const int pl = i / kBRow, p = i % kBRow;
        ranges_pos[((size_t)s * 2 + pl) * kBRow + p] =
            p < kBLive ? ranges_in[((size_t)s * 2 + pl) * 1326 + hand_at[p]] : 0.0f;
    }
}

// ---------------------------------------------------------------- solver ----

template <int K>
struct Cfg {
    static constexpr int NT = K == 2 ? 544 : (K == 3 ? 384 : 288);
    static constexpr int MINB = K == 2 ? 1 : 2;  // CTAs per SM the register budget is sized for
};

template <typename V>
__device__ __forceinline__ V neg_inf();
template <>
__device__ __forceinline__ float neg_inf<float>() {
    return -__int_as_float(0x7f800000);
}
template <>
__device__ __forceinline__ double neg_inf<double>() {
    return -__longlong_as_double(0x7ff0000000000000ll);
}

// Asks L2 to fetch [p, p + bytes) (16-byte aligned, size a multiple of 16) ahead of use.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
    const char *c = reinterpret_cast<const char *>(p);
    while (bytes > 0) {
        const unsigned n = bytes > 65536 ? 65536u : (unsigned)bytes;
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c), "r"(n) : "memory");
        c += n;
        bytes -= n;
    }
}

// The regret (and average) rows of subgame s, prefetched into L2.
__device__ __forceinline__ void prefetch_subgame(const BLaunch &a, int s) {
    const BSub sub = a.subs[s];
    const size_t off = (size_t)sub.edge_off * kBRow, bytes = (size_t)sub.num_edges * kBRow * sizeof(float);
    prefetch_l2(a.regrets + off, bytes);
    if (a.avg) prefetch_l2(a.avg + off, bytes);
    prefetch_l2(a.ranges + (size_t)s * 2 * kBRow, 2 * kBRow * sizeof(float));
}

// products rounded on their own (no contraction into a following add)
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }

template <typename V>
struct Smem {
    V *X;     // [group][kBRow] opponent weights, then leaf values
    V *I;     // [2][kBRow] chunk-local inclusive scans
    V *CT;    // [2][kBChunks] chunk totals
    V *SC;    // [2][kBLists][48] inclusive scans of the card lists
    BNode *tn;
    uint16_t *leaf_node;
    uint32_t *clpos;  // [kBLists][24] the card lists' positions, two per word (the pack's clpos)
    V *wsum;  // [32] warp partial sums
};

template <typename V>
__host__ __device__ inline size_t smem_bytes(int group) {
    size_t b = 0;
    b += (size_t)group * kBRow * sizeof(V);
    b += 2 * (size_t)kBRow * sizeof(V);
    b += 2 * (size_t)kBChunks * sizeof(V);
    b += 2 * (size_t)kBLists * 48 * sizeof(V);
    b += (size_t)kBMaxNodes * sizeof(BNode);
    b += (size_t)kBMaxLeaves * sizeof(uint16_t);
    b += (size_t)kBLists * 48 * sizeof(uint16_t);
    b += 32 * sizeof(V);
    return (b + 15) & ~(size_t)15;
}

template <typename V>
__device__ inline Smem<V> carve(unsigned char *base, int group) {
    Smem<V> S;
    V *v = reinterpret_cast<V *>(base);
    S.X = v;
    v += (size_t)group * kBRow;
    S.I = v;
    v += 2 * kBRow;
    S.CT = v;
    v += 2 * kBChunks;
    S.SC = v;
    v += 2 * kBLists * 48;
    S.wsum = v;
    v += 32;
    S.tn = reinterpret_cast<BNode *>(v);
    S.leaf_node = reinterpret_cast<uint16_t *>(S.tn + kBMaxNodes);
    S.clpos = reinterpret_cast<uint32_t *>(S.leaf_node + kBMaxLeaves);
    return S;
}

// A thread's K consecutive positions of a row. With K = 2 or 4 (and kBRow a multiple of 4)
// they are all inside the row or all past it, and move as vector accesses of at most 16 bytes
// (rows start on 16-byte boundaries); with K = 3 they move one by one. Positions past the row
// read as zero and are not written.
static_assert(kBRow % 4 == 0, "vector row accesses");
template <int K, typename T>
struct alignas(K == 3 ? sizeof(T) : (K * sizeof(T) > 16 ? 16 : K * sizeof(T))) Lanes {
    T v[K];
};

template <int K, typename T, typename U>
__device__ __forceinline__ void ld_k(const T *row, int pos0, U (&out)[K]) {
    if constexpr (K == 3) {
#pragma unroll
        for (int k = 0; k < K; k++) out[k] = pos0 + k < kBRow ? U(row[pos0 + k]) : U(0);
    } else {
        if (pos0 < kBRow) {
            const Lanes<K, T> t = *reinterpret_cast<const Lanes<K, T> *>(row + pos0);
#pragma unroll
            for (int k = 0; k < K; k++) out[k] = U(t.v[k]);
        } else {
#pragma unroll
            for (int k = 0; k < K; k++) out[k] = U(0);
        }
    }
}

template <int K, typename T, typename U>
__device__ __forceinline__ void st_k(T *row, int pos0, const U (&in)[K]) {
    if constexpr (K == 3) {
#pragma unroll
        for (int k = 0; k < K; k++)
            if (pos0 + k < kBRow) row[pos0 + k] = T(in[k]);
    } else {
        if (pos0 < kBRow) {
            Lanes<K, T> t;
#pragma unroll
            for (int k = 0; k < K; k++) t.v[k] = T(in[k]);
            *reinterpret_cast<Lanes<K, T> *>(row + pos0) = t;
        }
    }
}

// Rows read by the walks come in edge order (edges are numbered in pre-order): a node's
// strategy sums read rows [edge, edge + nchild), and the next nodes read the rows after them.
// This asks L1 for the 128-byte lines that a warp's positions of rows [first, first + n)
// occupy (rows from `rows` on, past the subgame's last edge, are skipped), one line per lane.
constexpr int kPfRows = 4;  // rows of lookahead
template <int K>
__device__ __forceinline__ void prefetch_rows(const float *base, int first, int n, int rows, int warp, int lane) {
    constexpr int kSpan = 32 * K;                  // floats of a row that one warp covers
    constexpr int kLines = (kSpan + 31) / 32 + 1;  // 128-byte lines the span can touch
    static_assert(kPfRows * kLines <= 32, "one prefetch per lane");
    if (lane < n * kLines) {
        const int row = first + lane / kLines;
        const int f = warp * kSpan + (lane % kLines) * 32;
        if (row < rows && f < kBRow) asm volatile("prefetch.global.L1 [%0];" ::"l"(base + (size_t)row * kBRow + f));
    }
}

// Regret matching with one division per node and hand: a node whose out-edges have
// positive-part sum S keeps scale(S) = 1 / S, or -1 / n when S is at most the cutoff (1e-4
// for regrets, 0 for average sums) and the strategy is uniform; an edge's probability is then
// sigma(val, scale) = max(val, 0) x scale, or 1 / n.
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }  // = 1.0f / x, correctly rounded
__device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }
template <typename V, bool USEAVG>
__device__ __forceinline__ V strategy_scale(V S, int n) {
    const V cut = USEAVG ? V(0) : V(1e-4f);
    return S <= cut ? -(V(1) / V(n)) : recip(S);
}
template <typename V>
__device__ __forceinline__ V sigma(V val, V scale) {
    return scale < V(0) ? -scale : mul(val > V(0) ? val : V(0), scale);
}

// MINB: CTAs per SM the registers are capped for (Cfg<K>::MINB, or 3 for the dense K = 4
// configuration with 10-leaf groups).
template <int K, typename V, int MODE, bool AVG, bool USEAVG, int MINB>
__global__ void __launch_bounds__(Cfg<K>::NT, MINB) batch_kernel(BLaunch a, int group) {
    constexpr int NT = Cfg<K>::NT;
    constexpr int NW = NT / 32;
    static_assert(MODE == kBModeCFR || !AVG, "average sums accumulate in CFR passes");
    static_assert(MODE != kBModeCFR || (sizeof(V) == 4 && !USEAVG), "CFR runs on regrets in single precision");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<V> S = carve<V>(smem_raw, group);
    __shared__ int s_next;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const unsigned FULL = 0xffffffffu;
    const int p = a.player, o = 1 - p;
    const float *src_all = USEAVG ? a.avg : a.regrets;
    // weight of this pass's average-sum terms (1 unless the caller weights iterations)
    const float wavg = AVG && a.avg_weight ? *a.avg_weight : 1.0f;

    // The next queue entry is taken (and its rows prefetched into L2) while the current one
    // is solved.
    if (tid == 0) {
        s_next = atomicAdd(a.head, 1);
        if (s_next < a.count) prefetch_subgame(a, a.order[s_next]);
    }
    for (;;) {
        __syncthreads();
        const int qi = s_next;
        __syncthreads();
        if (qi >= a.count) break;
        if (tid == 0) {
            s_next = atomicAdd(a.head, 1);
            if (s_next < a.count) prefetch_subgame(a, a.order[s_next]);
        }
        const int s = a.order[qi];
        const BSub sub = a.subs[s];
        const BPack *__restrict__ pk = a.packs + s;
        const int N = sub.num_nodes, L = sub.num_leaves;
        for (int i = tid; i < N; i += NT) {
            const BNode nd = a.nodes[sub.node_off + i];
            S.tn[i] = nd;
            if (nd.kind != kBDecision) S.leaf_node[nd.edge] = (uint16_t)i;
        }
        // the card lists' positions, read by every leaf scan, staged once per subgame
        {
            const uint32_t *src = reinterpret_cast<const uint32_t *>(&pk->clpos[0][0]);
            for (int i = tid; i < kBLists * 24; i += NT) S.clpos[i] = __ldg(src + i);
        }
        __syncthreads();
        float *R = a.regrets + (size_t)sub.edge_off * kBRow;
        float *A = a.avg ? a.avg + (size_t)sub.edge_off * kBRow : nullptr;
        const float *Src = src_all + (size_t)sub.edge_off * kBRow;
        const float *rng = a.ranges + (size_t)s * 2 * kBRow;
        const int pos0 = tid * K;
        // this thread's hands' tie-group and card-list bounds, read once per subgame

        // walker state, per owned hand: depth-indexed stacks of the open path (indexed at run
        // time, so they live in local memory, cached in L1). Depth-major with the K hands of a
        // depth adjacent and aligned, so that one depth moves as one vector access.
        alignas(16) V po[DS][K];
        alignas(16) V pp[DS][K];
        alignas(16) V St[DS][K];   // top-down: opponent weight, own reach, strategy scales
        alignas(16) V acc[DS][K];
        alignas(16) V Sb[DS][K];   // bottom-up: node values, strategy scales
        int open_id[DS];
        int open_top = -1;
        int td = 0, bu = 0;
        V root[K];
#pragma unroll
        for (int k = 0; k < K; k++) root[k] = V(0);

        // adds the values v of the child behind edge ie to its parent par, open at depth dp
        // The innermost open node of the bottom-up walk keeps its value and strategy scale in
        // registers (tacc, tsb); the stacks hold the open nodes outside it. Every child's value
        // goes to its parent, which is always that innermost node.
        V tacc[K], tsb[K];
        // between the bottom-up walks of two groups the registers rest in the stack slot of the
        // innermost open node (slot 0 when none is open: then nothing reads them)
        auto park = [&]() {
            const int t = open_top > 0 ? open_top : 0;
#pragma unroll
            for (int k = 0; k < K; k++) {
                acc[t][k] = tacc[k];
                Sb[t][k] = tsb[k];
            }
        };
        auto unpark = [&]() {
            const int t = open_top > 0 ? open_top : 0;
#pragma unroll
            for (int k = 0; k < K; k++) {
                tacc[k] = acc[t][k];
                tsb[k] = Sb[t][k];
            }
        };
#pragma unroll
        for (int k = 0; k < K; k++) tacc[k] = tsb[k] = V(0);
        park();
        auto deliver = [&](int par, int ie, const V(&v)[K]) {
            const BNode pq = S.tn[par];
            if (a.child_out && par == 0) {
                V *co = reinterpret_cast<V *>(a.child_out) + ((size_t)s * 8 + (ie - pq.edge)) * kBRow;
                st_k<K>(co, pos0, v);
            }
            if (pq.actor != p) {
#pragma unroll
                for (int k = 0; k < K; k++) tacc[k] = tacc[k] + v[k];
            } else if (MODE == kBModeBR) {
#pragma unroll
                for (int k = 0; k < K; k++) tacc[k] = tacc[k] > v[k] ? tacc[k] : v[k];
            } else {
                // the edge's strategy from its regret (or average) row; CFR adds the child's
                // value to the regret, which the parent's close turns into the regret update
                const size_t ro = (size_t)ie * kBRow;
                V sv[K];
                if (MODE == kBModeCFR)
                    ld_k<K>(R + ro, pos0, sv);
                else
                    ld_k<K>(Src + ro, pos0, sv);
#pragma unroll
                for (int k = 0; k < K; k++)
                    tacc[k] = tacc[k] + mul(sigma<V>(sv[k], tsb[k]), v[k]);
                if constexpr (MODE == kBModeCFR) {
                    float r[K];
#pragma unroll
                    for (int k = 0; k < K; k++) r[k] = float(sv[k]) + float(v[k]);
                    st_k<K>(R + ro, pos0, r);
                }
            }
        };
        // closes the open nodes at depth >= d, passing each value to its parent
        auto close_to = [&](int d) {
            while (open_top >= d) {
                const int m = open_id[open_top];
                const BNode nm = S.tn[m];
                V v[K];
#pragma unroll
                for (int k = 0; k < K; k++) v[k] = tacc[k];
                if (MODE == kBModeCFR && nm.actor == p) {
                    for (int e = 0; e < nm.nchild; e++) {
                        float *row = R + (size_t)(nm.edge + e) * kBRow;
                        float r[K];
                        ld_k<K>(row, pos0, r);
#pragma unroll
                        for (int k = 0; k < K; k++) r[k] = fmaxf(r[k] - float(v[k]), 0.0f);
                        st_k<K>(row, pos0, r);
                    }
                }
                open_top--;
                if (m == 0) {
#pragma unroll
                    for (int k = 0; k < K; k++) root[k] = v[k];
                } else {
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        tacc[k] = acc[open_top][k];
                        tsb[k] = Sb[open_top][k];
                    }
                    deliver(nm.parent, nm.in_edge, v);
                }
            }
        };
        for (int g0 = 0; g0 < L; g0 += group) {
            const int g1 = min(L, g0 + group);
            const int end = g1 == L ? N : S.leaf_node[g1];
            // ---- top-down walk over nodes [td, end) ----
            // Only decision nodes put their reach and strategy scale on the stacks: their
            // children read them, and nothing reads a leaf's entry.
            for (; td < end; td++) {
                const BNode nd = S.tn[td];
                const int d = nd.depth;
                V npo[K], npp[K];
                if (td == 0) {
                    if (sizeof(V) == 8 && a.ranges64)
                        ld_k<K>(a.ranges64 + ((size_t)s * 2 + o) * kBRow, pos0, npo);
                    else
                        ld_k<K>(rng + o * kBRow, pos0, npo);
                    if (MODE == kBModeCFR && a.own_reach) {
                        ld_k<K>(rng + p * kBRow, pos0, npp);
                    } else {
#pragma unroll
                        for (int k = 0; k < K; k++) npp[k] = V(1);
                    }
                } else {
                    const BNode pm = S.tn[nd.parent];
                    const bool own = pm.actor == p;
                    const bool need = !own || AVG;
                    const size_t ro = (size_t)nd.in_edge * kBRow;
                    V sv[K];
                    if (need) ld_k<K>(Src + ro, pos0, sv);
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        const V po_par = po[d - 1][k];
                        const V pp_par = pp[d - 1][k];
                        const V sg = need ? sigma<V>(sv[k], St[d - 1][k]) : V(1);
                        npo[k] = own ? po_par : mul(po_par, sg);
                        npp[k] = own ? mul(pp_par, sg) : pp_par;
                    }
                    if constexpr (AVG) {
                        if (own) {
                            float av[K];
                            ld_k<K>(A + ro, pos0, av);
#pragma unroll
                            for (int k = 0; k < K; k++) av[k] += wavg * float(npp[k]);
                            st_k<K>(A + ro, pos0, av);
                        }
                    }
                }
                if (nd.kind == kBDecision) {
                    // strategy sums of the node, for its children
                    const bool own = nd.actor == p;
                    V sum[K];
#pragma unroll
                    for (int k = 0; k < K; k++) sum[k] = V(0);
                    if (!own || AVG) {
                        for (int e = 0; e < nd.nchild; e++) {
                            V sv[K];
                            ld_k<K>(Src + (size_t)(nd.edge + e) * kBRow, pos0, sv);
#pragma unroll
                            for (int k = 0; k < K; k++) sum[k] += sv[k] > V(0) ? sv[k] : V(0);
                        }
                        prefetch_rows<K>(Src, nd.edge + nd.nchild, kPfRows, sub.num_edges, warp, lane);
                    }
                    if (AVG && own) prefetch_rows<K>(A, nd.edge, min(nd.nchild, kPfRows), sub.num_edges, warp, lane);
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        po[d][k] = npo[k];
                        pp[d][k] = npp[k];
                        St[d][k] = (!own || AVG) ? strategy_scale<V, USEAVG>(sum[k], nd.nchild) : V(0);
                    }
                } else {
                    V xv[K];
#pragma unroll
                    for (int k = 0; k < K; k++) xv[k] = pos0 + k < kBLive ? npo[k] : V(0);
                    st_k<K>(S.X + (size_t)(nd.edge - g0) * kBRow, pos0, xv);
                }
            }
            __syncthreads();

            // ---- leaves of the group: opponent weights -> p's values ----
            // this thread's hands' tie-group and card-list bounds (read here rather than kept
            // in registers through the walks)
            uint32_t pgrp[K], plist[K], plist2[K];
    #pragma unroll
            for (int k = 0; k < K; k++) {
                const int pq = pos0 + k < kBRow ? pos0 + k : kBRow - 1;
                pgrp[k] = __ldg(&pk->grp[pq]);
                plist[k] = __ldg(&pk->lists[pq]);
                plist2[k] = __ldg(&pk->lists2[pq]);
            }
            // A job is a leaf, or a fold by p followed by its sibling call (a showdown): p's
            // actions leave the opponent weights unchanged, so one scan serves both leaves.
            // Jobs go kJ at a time. With kJ = 2 (buffers 0 and 1) their scans interleave and
            // each hand's tie-group and card-list bounds are unpacked once for both; the dense
            // configuration (MINB = 3) runs one job at a time in alternate buffers instead,
            // which needs no barrier after the values and fits its register cap. Every job's
            // arithmetic is the same either way.
            constexpr int kJ = MINB >= 3 ? 1 : 2;
            int batch_no = 0;
            for (int j = g0; j < g1; batch_no++) {
                // buffer of job q of this step
                auto bufq = [&](int q) { return kJ == 1 ? (batch_no & 1) : q; };
                bool pair[2] = {false, false};
                BNode ln[2], lsd[2];
                V *xs[2], *xfs[2];
                int nj = 0;
                while (nj < kJ && j < g1) {
                    ln[nj] = S.tn[S.leaf_node[j]];
                    lsd[nj] = ln[nj];  // the leaf whose kind and stake give the main value
                    if (ln[nj].kind == kBFold && ln[nj].actor == p && j + 1 < g1) {
                        const BNode nx = S.tn[S.leaf_node[j + 1]];
                        if (nx.kind == kBShowdown && nx.parent == ln[nj].parent) {
                            pair[nj] = true;
                            lsd[nj] = nx;
                        }
                    }
                    xfs[nj] = S.X + (size_t)(j - g0) * kBRow;          // the fold's row when paired
                    xs[nj] = pair[nj] ? xfs[nj] + kBRow : xfs[nj];     // the scanned leaf's row
                    j += pair[nj] ? 2 : 1;
                    nj++;
                }
                // phase A: scans of the rank order in 64-hand chunks (two hands per lane) and
                // scans of the card lists, unit u of both jobs together
                for (int u = warp; u < kBChunks64 + kBLists; u += NW) {
                    if (u < kBChunks64) {
                        V a0[2], v[2];
#pragma unroll
                        for (int q = 0; q < kJ; q++) {
                            a0[q] = v[q] = V(0);
                            if (q < nj) {
                                a0[q] = xs[q][u * 64 + 2 * lane];
                                v[q] = a0[q] + xs[q][u * 64 + 2 * lane + 1];
                            }
                        }
#pragma unroll
                        for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                            for (int q = 0; q < kJ; q++) {
                                const V t = __shfl_up_sync(FULL, v[q], off);
                                if (lane >= off) v[q] += t;
                            }
                        }
#pragma unroll
                        for (int q = 0; q < kJ; q++) {
                            V ex = __shfl_up_sync(FULL, v[q], 1);
                            if (lane == 0) ex = V(0);
                            if (q < nj) {
                                V *I = S.I + bufq(q) * kBRow;
                                I[u * 64 + 2 * lane] = ex + a0[q];
                                I[u * 64 + 2 * lane + 1] = v[q];
                                if (lane == 31) S.CT[bufq(q) * kBChunks + u] = v[q];
                            }
                        }
                    } else {
                        const int li = u - kBChunks64;
                        int c0 = 0, c1 = 0;
                        if (lane < kBListLen / 2) {
                            const uint32_t w = S.clpos[li * 24 + lane];
                            c0 = w & 0xFFFF;
                            c1 = w >> 16;
                        }
                        V a0[2], v[2];
#pragma unroll
                        for (int q = 0; q < kJ; q++) {
                            a0[q] = v[q] = V(0);
                            if (q < nj && lane < kBListLen / 2) {
                                a0[q] = xs[q][c0];
                                v[q] = a0[q] + xs[q][c1];
                            }
                        }
#pragma unroll
                        for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                            for (int q = 0; q < kJ; q++) {
                                const V t = __shfl_up_sync(FULL, v[q], off);
                                if (lane >= off) v[q] += t;
                            }
                        }
#pragma unroll
                        for (int q = 0; q < kJ; q++) {
                            V ex = __shfl_up_sync(FULL, v[q], 1);
                            if (lane == 0) ex = V(0);
                            if (q < nj && lane < kBListLen / 2) {
                                V *SC = S.SC + bufq(q) * kBLists * 48;
                                SC[li * 48 + 2 * lane] = ex + a0[q];
                                SC[li * 48 + 2 * lane + 1] = v[q];
                            }
                        }
                    }
                }
                __syncthreads();
                // phase C: chunk offsets (every warp, same arithmetic; lane c holds chunk c's),
                // then values
                V cofs[2], T[2];
                {
                    V inc[2];
#pragma unroll
                    for (int q = 0; q < kJ; q++) inc[q] = (q < nj && lane < kBChunks64) ? S.CT[bufq(q) * kBChunks + lane] : V(0);
#pragma unroll
                    for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                        for (int q = 0; q < kJ; q++) {
                            const V t = __shfl_up_sync(FULL, inc[q], off);
                            if (lane >= off) inc[q] += t;
                        }
                    }
#pragma unroll
                    for (int q = 0; q < kJ; q++) {
                        cofs[q] = __shfl_up_sync(FULL, inc[q], 1);
                        if (lane == 0) cofs[q] = V(0);
                        T[q] = __shfl_sync(FULL, inc[q], kBChunks64 - 1);
                    }
                }
                V xv[2][K], fv[2][K];
#pragma unroll
                for (int q = 0; q < kJ; q++)
                    if (q < nj) ld_k<K>(xs[q], pos0, xv[q]);
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const int pos = pos0 + k;
                    const uint32_t gr = pgrp[k], l1 = plist[k], l2 = plist2[k];
                    const int gs = gr & 0xFFFF, ge = gr >> 16;
                    const int li1 = l1 & 255, li2 = (l1 >> 8) & 255;
                    const int gs1 = (l1 >> 16) & 255, ge1 = l1 >> 24;
                    const int gs2 = l2 & 255, ge2 = (l2 >> 8) & 255;
                    const int ce = ge >> 6, cs = gs > 0 ? (gs - 1) >> 6 : 0;
#pragma unroll
                    for (int q = 0; q < kJ; q++) {
                        if (q >= nj) continue;
                        // chunk offsets by shuffle (all lanes take part)
                        const V oe = __shfl_sync(FULL, cofs[q], ce);
                        const V os = __shfl_sync(FULL, cofs[q], cs);
                        const V *I = S.I + bufq(q) * kBRow;
                        const V *SC = S.SC + bufq(q) * kBLists * 48;
                        V val = V(0), fval = V(0);
                        if (pos < kBLive) {
                            const V *sc1 = SC + li1 * 48;
                            const V *sc2 = SC + li2 * 48;
                            const V T1 = sc1[kBListLen - 1], T2 = sc2[kBListLen - 1];
                            const V free = ((T[q] - T1) - T2) + xv[q][k];
                            const V stake = V(lsd[q].stake);
                            if (lsd[q].kind == kBShowdown) {
                                const V Pe = oe + I[ge];
                                const V Ps = gs > 0 ? os + I[gs - 1] : V(0);
                                const V vg = (Pe + Ps) - T[q];
                                const V v1 = (sc1[ge1] + (gs1 > 0 ? sc1[gs1 - 1] : V(0))) - T1;
                                const V v2 = (sc2[ge2] + (gs2 > 0 ? sc2[gs2 - 1] : V(0))) - T2;
                                val = mul(stake, (vg - v1) - v2);
                            } else {
                                val = mul(lsd[q].actor == p ? -stake : stake, free);
                            }
                            if (pair[q]) fval = mul(-V(ln[q].stake), free);
                        }
                        xv[q][k] = val;
                        fv[q][k] = fval;
                    }
                }
#pragma unroll
                for (int q = 0; q < kJ; q++) {
                    if (q >= nj) continue;
                    st_k<K>(xs[q], pos0, xv[q]);
                    if (pair[q]) st_k<K>(xfs[q], pos0, fv[q]);
                }
                if constexpr (kJ == 2) __syncthreads();  // the next two jobs rewrite buffers 0 and 1
            }
            if constexpr (kJ == 1) __syncthreads();  // the bottom-up walk reads every leaf's values

            // ---- bottom-up walk over nodes [bu, end) ----
            unpark();
            for (; bu < end; bu++) {
                const BNode nd = S.tn[bu];
                const int d = nd.depth;
                close_to(d);
                if (nd.kind == kBDecision) {
                    // the parent (open at d - 1, or none at the root) moves to the stack
                    if (open_top >= 0) {
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            acc[open_top][k] = tacc[k];
                            Sb[open_top][k] = tsb[k];
                        }
                    }
                    open_top = d;
                    open_id[d] = bu;
                    const bool own = nd.actor == p;
                    V sum[K];
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        tacc[k] = (own && MODE == kBModeBR) ? neg_inf<V>() : V(0);
                        sum[k] = V(0);
                    }
                    if (own && MODE != kBModeBR) {
                        for (int e = 0; e < nd.nchild; e++) {
                            V sv[K];
                            ld_k<K>(Src + (size_t)(nd.edge + e) * kBRow, pos0, sv);
#pragma unroll
                            for (int k = 0; k < K; k++) sum[k] += sv[k] > V(0) ? sv[k] : V(0);
                        }
                        prefetch_rows<K>(Src, nd.edge + nd.nchild, kPfRows, sub.num_edges, warp, lane);
                    }
#pragma unroll
                    for (int k = 0; k < K; k++)
                        tsb[k] = (own && MODE != kBModeBR) ? strategy_scale<V, USEAVG>(sum[k], nd.nchild) : V(0);
                } else {
                    // a leaf: its value goes straight to the parent (the innermost open node)
                    V xv[K];
                    ld_k<K>(S.X + (size_t)(nd.edge - g0) * kBRow, pos0, xv);
                    deliver(nd.parent, nd.in_edge, xv);
                }
            }
            park();
            __syncthreads();  // X is rewritten by the next group
        }
        unpark();
        close_to(0);

        // ---- outputs: root values and their range-weighted sum ----
        if (a.root_out) {
            st_k<K>(reinterpret_cast<V *>(a.root_out) + (size_t)s * kBRow, pos0, root);
        }
        if (a.sum_out) {
            V part = V(0);
            V rv[K];
            ld_k<K>(rng + p * kBRow, pos0, rv);
#pragma unroll
            for (int k = 0; k < K; k++)
                if (pos0 + k < kBRow) part += mul(rv[k], root[k]);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(FULL, part, off);
            if (lane == 0) S.wsum[warp] = part;
            __syncthreads();
            if (tid == 0) {
                V t = V(0);
                for (int w = 0; w < NW; w++) t += S.wsum[w];
                reinterpret_cast<V *>(a.sum_out)[s] = t;
            }
        }
        __syncthreads();
    }
}

__global__ void weight_step_kernel(float *w) { *w += 1.0f; }

template <int K, typename V, int MODE, bool AVG, bool USEAVG, int MINB = Cfg<K>::MINB>
cudaError_t launch_one(const BLaunch &a, int ctas, int group, cudaStream_t stream) {
    const size_t smem = smem_bytes<V>(group);
    cudaError_t e = cudaFuncSetAttribute(batch_kernel<K, V, MODE, AVG, USEAVG, MINB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    batch_kernel<K, V, MODE, AVG, USEAVG, MINB><<<ctas, Cfg<K>::NT, smem, stream>>>(a, group);
    return cudaGetLastError();
}

template <int K>
cudaError_t launch_k(int mode, int fp64, int avg, const BLaunch &a, int ctas, int group, cudaStream_t st,
                     int dense) {
    if (mode == kBModeCFR) {
        if (fp64) return cudaErrorInvalidValue;
        if constexpr (K == 4) {
            if (dense)
                return avg ? launch_one<4, float, kBModeCFR, true, false, 3>(a, ctas, group, st)
                           : launch_one<4, float, kBModeCFR, false, false, 3>(a, ctas, group, st);
        }
        return avg ? launch_one<K, float, kBModeCFR, true, false>(a, ctas, group, st)
                   : launch_one<K, float, kBModeCFR, false, false>(a, ctas, group, st);
    }
    if (mode == kBModeBR) {
        if (fp64)
            return a.use_average ? launch_one<K, double, kBModeBR, false, true>(a, ctas, group, st)
                                 : launch_one<K, double, kBModeBR, false, false>(a, ctas, group, st);
        return a.use_average ? launch_one<K, float, kBModeBR, false, true>(a, ctas, group, st)
                             : launch_one<K, float, kBModeBR, false, false>(a, ctas, group, st);
    }
    if (fp64)
        return a.use_average ? launch_one<K, double, kBModeEval, false, true>(a, ctas, group, st)
                             : launch_one<K, double, kBModeEval, false, false>(a, ctas, group, st);
    return a.use_average ? launch_one<K, float, kBModeEval, false, true>(a, ctas, group, st)
                         : launch_one<K, float, kBModeEval, false, false>(a, ctas, group, st);
}

}  // namespace

cudaError_t launch_batch_setup(const BSub *subs, int count, BPack *packs, const float *ranges_in,
                               float *ranges_pos, int *err, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    batch_setup_kernel<<<count, kSetupThreads, 0, stream>>>(subs, packs, ranges_in, ranges_pos, err);
    return cudaGetLastError();
}

int batch_threads(int K) { return K == 2 ? Cfg<2>::NT : (K == 3 ? Cfg<3>::NT : Cfg<4>::NT); }

int batch_group_leaves(int fp64) { return fp64 ? 8 : 16; }

int batch_dense_group() { return 9; }

size_t batch_smem_bytes(int K, int fp64, int group) {
    (void)K;
    return fp64 ? smem_bytes<double>(group) : smem_bytes<float>(group);
}

cudaError_t launch_weight_step(float *w, cudaStream_t stream) {
    weight_step_kernel<<<1, 1, 0, stream>>>(w);
    return cudaGetLastError();
}

cudaError_t launch_batch_pass(int mode, int K, int fp64, int avg, const BLaunch &a, int ctas, int group,
                              cudaStream_t stream, int dense) {
    if (group < 1 || group > kBMaxLeaves || ctas < 1) return cudaErrorInvalidValue;
    switch (K) {
        case 2: return launch_k<2>(mode, fp64, avg, a, ctas, group, stream, 0);
        case 3: return launch_k<3>(mode, fp64, avg, a, ctas, group, stream, 0);
        case 4: return launch_k<4>(mode, fp64, avg, a, ctas, group, stream, dense);
        default: return cudaErrorInvalidValue;
    }
}

int batch_dense_ctas_per_sm(int avg) {
    int n = 0;
    const size_t smem = smem_bytes<float>(batch_dense_group());
    cudaError_t e;
    if (avg) {
        cudaFuncSetAttribute(batch_kernel<4, float, kBModeCFR, true, false, 3>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<4, float, kBModeCFR, true, false, 3>,
                                                          Cfg<4>::NT, smem);
    } else {
        cudaFuncSetAttribute(batch_kernel<4, float, kBModeCFR, false, false, 3>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<4, float, kBModeCFR, false, false, 3>,
                                                          Cfg<4>::NT, smem);
    }
    return e == cudaSuccess ? n : 0;
}

int batch_ctas_per_sm(int mode, int K, int fp64, int avg) {
    int n = 0;
    const int group = batch_group_leaves(fp64);
    const size_t smem = batch_smem_bytes(K, fp64, group);
    cudaError_t e = cudaSuccess;
#define PRB_OCC(KK, VV, MM, AA, UU)                                                                   \
    do {                                                                                              \
        cudaFuncSetAttribute(batch_kernel<KK, VV, MM, AA, UU, Cfg<KK>::MINB>,                           \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                 \
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<KK, VV, MM, AA, UU, Cfg<KK>::MINB>, \
                                                          Cfg<KK>::NT, smem);                         \
    } while (0)
    if (mode == kBModeCFR) {
        if (K == 2) { if (avg) PRB_OCC(2, float, kBModeCFR, true, false); else PRB_OCC(2, float, kBModeCFR, false, false); }
        else if (K == 3) { if (avg) PRB_OCC(3, float, kBModeCFR, true, false); else PRB_OCC(3, float, kBModeCFR, false, false); }
        else { if (avg) PRB_OCC(4, float, kBModeCFR, true, false); else PRB_OCC(4, float, kBModeCFR, false, false); }
    } else if (fp64) {
        if (K == 2) PRB_OCC(2, double, kBModeBR, false, false);
        else if (K == 3) PRB_OCC(3, double, kBModeBR, false, false);
        else PRB_OCC(4, double, kBModeBR, false, false);
    } else {
        if (K == 2) PRB_OCC(2, float, kBModeBR, false, false);
        else if (K == 3) PRB_OCC(3, float, kBModeBR, false, false);
        else PRB_OCC(4, float, kBModeBR, false, false);
    }
#undef PRB_OCC
    return e == cudaSuccess ? n : 0;
}

}  // namespace prb
