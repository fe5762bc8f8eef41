// Full fixed-flop game with general bets on every street (no reference counterpart: the
// reference's full game is the limit tree of src/game.rs, src/state.rs and
// src/builder.rs). The flop and turn streets (full_tree.h) run on the device level by
// level, one CTA per node and threads over the 1326 hands, in the manner of the reference's
// upper-tree traversal (state.rs:219-376): a top-down sweep carries both players' reach,
// scaled at each decision by the actor's regret-matched (or average) strategy and masked by
// the dealt turn card; a bottom-up sweep evaluates folds with card removal, averages the
// turn deal over its 49 cards, and at the updater's decisions takes the strategy-weighted
// sum (or the maximum, for a best response) and updates regrets r <- max(r + u - v, 0)
// and the average sums avg += reach x strategy.
//
// Every leaf (end of the turn) is a river chance node: its 48 river subgames (one per
// river card, the leaf's pot and stack) are solved by the batched river solver in the same
// pass. Both players' reach at the leaf goes into the subgames' ranges; the subgames' root
// values, averaged over the 48 rivers, come back as the leaf's values. Leaves reached with
// chips behind can instead take their values from the turn-leaf value network
// (net-leaf mode); all-in leaves always use their (betting-free) river subgames.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/pokerrust_b200.h"
#include "batch_internal.h"
#include "batch_solver.h"
#include "device_common.cuh"
#include "full_tree.h"
#include "trace.h"

namespace prb {
namespace {

constexpr int FT = 256;        // threads per CTA
constexpr int kH = 1326;       // hands per vector, colex order
constexpr int kRivers = 48;    // river cards after a 4-card board
constexpr int kNetIn = 2652;   // value network output width (both players' hands)

int ffail(const char *what, cudaError_t e = cudaSuccess) {
    if (e != cudaSuccess) fprintf(stderr, "pokerrust_b200: full game: %s: %s\n", what, cudaGetErrorString(e));
    else fprintf(stderr, "pokerrust_b200: full game: %s\n", what);
    fflush(stderr);
    return e != cudaSuccess ? 1 : 2;
}

__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }

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

__device__ __forceinline__ unsigned long long hand_bits(int h) {
    int c1, c2;
    hand_cards(h, &c1, &c2);
    return (1ull << c1) | (1ull << c2);
}

// Strategy of hand h at a decision node with n actions whose rows start at `first`:
// positive parts of the regrets (or average sums) over their sum, uniform when the sum is
// at most 1e-4 (regrets) or 0 (average sums).
template <typename T>
__device__ __forceinline__ void strategy(const float *src, int first, int n, int h, bool average,
                                         T (&p)[kFMaxKids]) {
    T v[kFMaxKids];
    T sum = T(0);
#pragma unroll
    for (int k = 0; k < kFMaxKids; k++) {
        v[k] = T(0);
        if (k < n) {
            const T x = T(src[(size_t)(first + k) * kH + h]);
            v[k] = x > T(0) ? x : T(0);
            sum += v[k];
        }
    }
    const T cut = average ? T(0) : T(1e-4f);
#pragma unroll
    for (int k = 0; k < kFMaxKids; k++) p[k] = sum <= cut ? T(1) / T(n) : v[k] / sum;
}

// Deterministic CTA sum of per-thread partials (fixed tree over FT threads).
template <typename T>
__device__ T cta_sum(T x, T *red) {
    red[threadIdx.x] = x;
    __syncthreads();
#pragma unroll
    for (int w = FT / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        __syncthreads();
    }
    const T t = red[0];
    __syncthreads();
    return t;
}

struct FView {
    const FNode *nodes;
    const int *kids;
};

// ---- top-down: reach of both players ([node][2][kH]) ----
template <typename T>
__global__ void __launch_bounds__(FT) down_kernel(FView v, const int *__restrict__ level, T *__restrict__ R,
                                                   const float *__restrict__ src, int average) {
    const int n = level[blockIdx.x];
    const FNode nd = v.nodes[n];
    const T *r0 = R + (size_t)n * 2 * kH;
    const T *r1 = r0 + kH;
    if (nd.kind == kFDecision) {
        for (int h = threadIdx.x; h < kH; h += FT) {
            T p[kFMaxKids];
            strategy<T>(src, nd.edge, nd.nchild, h, average != 0, p);
            const T a = r0[h], b = r1[h];
#pragma unroll
            for (int k = 0; k < kFMaxKids; k++) {
                if (k >= nd.nchild) break;
                T *c = R + (size_t)v.kids[nd.kids + k] * 2 * kH;
                c[h] = nd.actor == 0 ? mul(a, p[k]) : a;
                c[kH + h] = nd.actor == 1 ? mul(b, p[k]) : b;
            }
        }
    }
}

// deal nodes, top-down: one CTA per (deal node, card); the card's hands are masked
template <typename T>
__global__ void __launch_bounds__(FT) deal_down_kernel(FView v, const int *__restrict__ deals, T *__restrict__ R) {
    const int n = deals[blockIdx.x];
    const FNode nd = v.nodes[n];
    const int k = blockIdx.y;
    if (k >= nd.nchild) return;
    const int ci = v.kids[nd.kids + k];
    const unsigned long long dealt = v.nodes[ci].board & ~nd.board;
    const T *r = R + (size_t)n * 2 * kH;
    T *c = R + (size_t)ci * 2 * kH;
    for (int h = threadIdx.x; h < kH; h += FT) {
        const bool blocked = (hand_bits(h) & dealt) != 0;
        c[h] = blocked ? T(0) : r[h];
        c[kH + h] = blocked ? T(0) : r[kH + h];
    }
}

// deal nodes, bottom-up: the mean over the cards of the children's values (hands holding the
// card count 0); one CTA per (deal node, FT hands)
template <typename T>
__global__ void __launch_bounds__(FT) deal_up_kernel(FView v, const int *__restrict__ deals, T *__restrict__ V) {
    const int n = deals[blockIdx.x];
    const FNode nd = v.nodes[n];
    const int h = blockIdx.y * FT + threadIdx.x;
    if (h >= kH) return;
    const unsigned long long hb = hand_bits(h);
    T s = T(0);
    for (int k = 0; k < nd.nchild; k++) {
        const int ci = v.kids[nd.kids + k];
        if (hb & (v.nodes[ci].board & ~nd.board)) continue;
        s += V[(size_t)ci * kH + h];
    }
    V[(size_t)n * kH + h] = s / T(nd.nchild);
}

enum { kUpCFR = 0, kUpBR = 1, kUpEval = 2 };

// ---- bottom-up: values of `upd` ([node][kH]) ----
template <typename T, int MODE>
__global__ void __launch_bounds__(FT) up_kernel(FView v, const int *__restrict__ level, int upd,
                                                 const T *__restrict__ R, T *__restrict__ V,
                                                 const T *__restrict__ leafV, float *__restrict__ regrets,
                                                 float *__restrict__ avg, const float *__restrict__ src,
                                                 int average, const float *__restrict__ wt) {
    __shared__ T red[FT];
    __shared__ T csum[52];
    const int n = level[blockIdx.x];
    const FNode nd = v.nodes[n];
    T *out = V + (size_t)n * kH;
    switch (nd.kind) {
        case kFLeaf:
            for (int h = threadIdx.x; h < kH; h += FT) out[h] = leafV[(size_t)nd.edge * kH + h];
            return;
        case kFFold: {
            // opponent weight compatible with each hand: total - both cards' sums + the hand
            const T *opp = R + ((size_t)n * 2 + (1 - upd)) * kH;
            T part = T(0);
            for (int h = threadIdx.x; h < kH; h += FT) part += opp[h];
            const T total = cta_sum(part, red);
            if (threadIdx.x < 52) {
                const int c = threadIdx.x;
                T s = T(0);
                for (int o = 0; o < 52; o++) {
                    if (o == c) continue;
                    s += opp[c < o ? c + o * (o - 1) / 2 : o + c * (c - 1) / 2];
                }
                csum[c] = s;
            }
            __syncthreads();
            const T m = T(nd.stake) * (nd.actor == upd ? T(-1) : T(1));
            for (int h = threadIdx.x; h < kH; h += FT) {
                int c1, c2;
                hand_cards(h, &c1, &c2);
                const T x = ((total - csum[c1]) - csum[c2]) + opp[h];
                out[h] = mul(m, x);
            }
            return;
        }
        default: {
            const bool mine = nd.actor == upd;
            const T *own = R + ((size_t)n * 2 + upd) * kH;
            const float wavg = wt ? *wt : 1.0f;
            for (int h = threadIdx.x; h < kH; h += FT) {
                T p[kFMaxKids], u[kFMaxKids];
                if (mine && MODE != kUpBR) strategy<T>(src, nd.edge, nd.nchild, h, average != 0, p);
                T acc = (mine && MODE == kUpBR) ? neg_inf<T>() : T(0);
#pragma unroll
                for (int k = 0; k < kFMaxKids; k++) {
                    if (k >= nd.nchild) break;
                    u[k] = V[(size_t)v.kids[nd.kids + k] * kH + h];
                    if (!mine) acc += u[k];
                    else if (MODE == kUpBR) acc = acc > u[k] ? acc : u[k];
                    else acc += mul(p[k], u[k]);
                }
                out[h] = acc;
                if (MODE == kUpCFR && mine) {
                    const T w = own[h];
#pragma unroll
                    for (int k = 0; k < kFMaxKids; k++) {
                        if (k >= nd.nchild) break;
                        float &r = regrets[(size_t)(nd.edge + k) * kH + h];
                        r = fmaxf((r + float(u[k])) - float(acc), 0.0f);
                        if (avg) avg[(size_t)(nd.edge + k) * kH + h] += wavg * float(mul(w, p[k]));
                    }
                }
            }
            return;
        }
    }
}

// ---- leaves <-> river subgames ----
// subgame s belongs to slot s / 48 (a leaf node); its ranges are the leaf's reach.
template <typename T>
__global__ void __launch_bounds__(FT) scatter_kernel(const BPack *__restrict__ packs, const T *__restrict__ R,
                                                      const int *__restrict__ slot_node, T *__restrict__ ranges) {
    const int s = blockIdx.x;
    const T *r = R + (size_t)slot_node[s / kRivers] * 2 * kH;
    const uint16_t *hand = packs[s].hand;
    for (int p = threadIdx.x; p < kBRow; p += FT) {
        const int h = hand[p];
        ranges[((size_t)s * 2 + 0) * kBRow + p] = h != 0xFFFF ? r[h] : T(0);
        ranges[((size_t)s * 2 + 1) * kBRow + p] = h != 0xFFFF ? r[kH + h] : T(0);
    }
}

// leaf value = mean over the 48 rivers of the subgames' root values (0 where the river card
// is in the hand)
template <typename T>
__global__ void __launch_bounds__(FT) gather_kernel(const BPack *__restrict__ packs, const T *__restrict__ root,
                                                     const int *__restrict__ slot_node, const FNode *__restrict__ nodes,
                                                     T *__restrict__ leafV) {
    const int j = blockIdx.x;
    T *out = leafV + (size_t)nodes[slot_node[j]].edge * kH;
    for (int h = threadIdx.x; h < kH; h += FT) {
        T s = T(0);
        for (int k = 0; k < kRivers; k++) {
            const int sg = j * kRivers + k;
            const int p = packs[sg].pos_of[h];
            if (p != 0xFFFF) s += root[(size_t)sg * kBRow + p];
        }
        out[h] = s / T(kRivers);
    }
}

// ---- net leaves ----
// inputs of the value network: both ranges normalised to sum 1, the 4-card board, pot / 200
// and stack / (10 pot); the reach masses scale the outputs back.
__global__ void __launch_bounds__(FT) net_in_kernel(const FNode *__restrict__ nodes, const int *__restrict__ slot_node,
                                                     const float *__restrict__ R, float *__restrict__ ranges,
                                                     unsigned long long *__restrict__ boards,
                                                     float *__restrict__ scalars, float *__restrict__ mass) {
    __shared__ float red[FT];
    const int j = blockIdx.x;
    const FNode nd = nodes[slot_node[j]];
    const float *r = R + (size_t)slot_node[j] * 2 * kH;
    for (int pl = 0; pl < 2; pl++) {
        float part = 0.0f;
        for (int h = threadIdx.x; h < kH; h += FT) part += r[pl * kH + h];
        const float m = cta_sum(part, red);
        const float inv = m > 0.0f ? 1.0f / m : 0.0f;
        for (int h = threadIdx.x; h < kH; h += FT) ranges[((size_t)j * 2 + pl) * kH + h] = r[pl * kH + h] * inv;
        if (threadIdx.x == 0) mass[j * 2 + pl] = m;
    }
    if (threadIdx.x == 0) {
        boards[j] = nd.board;
        scalars[j * 2 + 0] = nd.stake / 200.0f;
        scalars[j * 2 + 1] = nd.stack / (10.0f * nd.stake);
    }
}

// leaf value of `upd` = network output x pot x the opponent's reach mass. With zero_sum, the
// outputs are first shifted by -e/2, e = r0 . v0 + r1 . v1 over the normalised input ranges:
// true values of a zero-sum subgame have e = 0 (each player's range-weighted value is minus
// the other's), and the shift restores that, as DeepStack's output layer does.
__global__ void __launch_bounds__(FT) net_out_kernel(const FNode *__restrict__ nodes, const int *__restrict__ slot_node,
                                                      const float *__restrict__ out, const float *__restrict__ mass,
                                                      const float *__restrict__ rin, int zero_sum, int upd,
                                                      float *__restrict__ leafV) {
    __shared__ float red[FT];
    const int j = blockIdx.x;
    const FNode nd = nodes[slot_node[j]];
    const float scale = nd.stake * mass[j * 2 + (1 - upd)];
    const float *o = out + (size_t)j * kNetIn;
    float shift = 0.0f;
    if (zero_sum) {
        float part = 0.0f;
        for (int h = threadIdx.x; h < kH; h += FT)
            part += rin[((size_t)j * 2) * kH + h] * o[h] + rin[((size_t)j * 2 + 1) * kH + h] * o[kH + h];
        shift = 0.5f * cta_sum(part, red);
    }
    float *dst = leafV + (size_t)nd.edge * kH;
    for (int h = threadIdx.x; h < kH; h += FT) dst[h] = (o[upd * kH + h] - shift) * scale;
}

// the next iteration's weight of the average sums (linear averaging: iteration t has weight t)
__global__ void bump_kernel(float *w) { *w += 1.0f; }

__global__ void root_sum_kernel(const double *__restrict__ V, const float *__restrict__ init, int player,
                                double *__restrict__ out) {
    __shared__ double red[FT];
    double part = 0.0;
    for (int h = threadIdx.x; h < kH; h += FT) part += (double)init[player * kH + h] * V[h];
    const double t = cta_sum(part, red);
    if (threadIdx.x == 0) *out = t;
}

struct Game {
    pr_full_spec spec{};
    FullTree tree;
    std::vector<std::vector<int>> levels, deals;  // per level: deal nodes / all other nodes
    std::vector<int> level_off, deal_off;
    std::vector<float> init;  // [2][kH]
    double joint = 0;
    int N = 0, E = 0, L = 0;
    cudaStream_t stream = nullptr;
    FNode *d_nodes = nullptr;
    int *d_kids = nullptr, *d_levels = nullptr;
    float *d_reg = nullptr, *d_avg = nullptr, *d_init = nullptr;
    float *d_R = nullptr, *d_V = nullptr, *d_leafV = nullptr;
    double *d_R64 = nullptr, *d_V64 = nullptr, *d_leafV64 = nullptr, *d_sum = nullptr;
    float *d_wt = nullptr;  // weight of the current iteration's average-sum terms
    bool linear = true;     // average sums weighted by the iteration number (else 1)
    // river subgames: [0] leaves with chips behind, [1] all-in leaves
    void *batch[2] = {nullptr, nullptr};
    std::vector<int> slots[2];
    int *d_slots[2] = {nullptr, nullptr};
    void *d_root[2] = {nullptr, nullptr};  // [subgames][kBRow] doubles (float passes use the front)
    BatchView view[2]{};
    // net-leaf mode
    void *net = nullptr;
    int net_rows = 0;
    bool zero_sum = false;  // shift the network's outputs to zero sum (net_out_kernel)
    float *d_nin = nullptr, *d_nscal = nullptr, *d_nmass = nullptr, *d_nout = nullptr;
    unsigned long long *d_nboard = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool graph_failed = false;

    ~Game() {
        if (graph) cudaGraphExecDestroy(graph);
        if (stream) cudaStreamSynchronize(stream);
        for (int b = 0; b < 2; b++) {
            if (batch[b]) pr_batch_free(batch[b]);
            cudaFree(d_slots[b]);
            cudaFree(d_root[b]);
        }
        for (void *p : {(void *)d_nodes, (void *)d_kids, (void *)d_levels, (void *)d_reg, (void *)d_avg,
                        (void *)d_init, (void *)d_R, (void *)d_V, (void *)d_leafV, (void *)d_R64, (void *)d_V64,
                        (void *)d_leafV64, (void *)d_sum, (void *)d_nin, (void *)d_nscal, (void *)d_nmass,
                        (void *)d_nout, (void *)d_nboard, (void *)d_wt})
            cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }

    FView fview() const { return FView{d_nodes, d_kids}; }
    const int *level_ptr(int l) const { return d_levels + level_off[l]; }
    int level_size(int l) const { return (int)levels[l].size(); }
    const int *deal_ptr(int l) const { return d_levels + deal_off[l]; }
    int deal_size(int l) const { return (int)deals[l].size(); }

    template <typename T>
    int down(T *R, const float *src, int average) {
        for (int l = 0; l + 1 < (int)levels.size(); l++) {
            if (level_size(l)) down_kernel<T><<<level_size(l), FT, 0, stream>>>(fview(), level_ptr(l), R, src, average);
            if (deal_size(l)) deal_down_kernel<T><<<dim3(deal_size(l), 52), FT, 0, stream>>>(fview(), deal_ptr(l), R);
        }
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? 0 : ffail("down sweep", e);
    }

    template <typename T, int MODE>
    int up(int upd, const T *R, T *V, const T *leafV, const float *src, int average) {
        for (int l = (int)levels.size() - 1; l >= 0; l--) {
            if (deal_size(l))
                deal_up_kernel<T><<<dim3(deal_size(l), (kH + FT - 1) / FT), FT, 0, stream>>>(fview(), deal_ptr(l), V);
            if (!level_size(l)) continue;
            up_kernel<T, MODE><<<level_size(l), FT, 0, stream>>>(fview(), level_ptr(l), upd, R, V, leafV,
                                                                 MODE == kUpCFR ? d_reg : nullptr,
                                                                 MODE == kUpCFR ? d_avg : nullptr, src, average,
                                                                 d_wt);
        }
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? 0 : ffail("up sweep", e);
    }

    // river subgames of batch b: ranges from the reach R, one pass, leaf values back
    template <typename T>
    int rivers(int b, int mode, int player, int use_average, const T *R, T *leafV) {
        if (!batch[b]) return 0;
        const BatchView &v = view[b];
        const bool f64 = sizeof(T) == 8;
        scatter_kernel<T><<<v.count, FT, 0, stream>>>(v.packs, R, d_slots[b],
                                                      f64 ? (T *)v.ranges64 : (T *)v.ranges);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return ffail("range scatter", e);
        if (int st = batch_run_pass(batch[b], mode, player, f64 ? 1 : 0, use_average, d_root[b], stream)) return st;
        gather_kernel<T><<<(int)slots[b].size(), FT, 0, stream>>>(v.packs, (const T *)d_root[b], d_slots[b], d_nodes,
                                                                  leafV);
        e = cudaGetLastError();
        return e == cudaSuccess ? 0 : ffail("value gather", e);
    }

    int net_leaves(int player) {
        const int n = (int)slots[0].size();
        if (!n) return 0;
        net_in_kernel<<<n, FT, 0, stream>>>(d_nodes, d_slots[0], d_R, d_nin, d_nboard, d_nscal, d_nmass);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return ffail("net inputs", e);
        for (int j0 = 0; j0 < n; j0 += net_rows) {
            const int c = std::min(net_rows, n - j0);
            if (int st = pr_mlp_forward(net, d_nin + (size_t)j0 * 2 * kH, (const uint64_t *)(d_nboard + j0),
                                        d_nscal + (size_t)j0 * 2, d_nout + (size_t)j0 * kNetIn, c))
                return st;
        }
        net_out_kernel<<<n, FT, 0, stream>>>(d_nodes, d_slots[0], d_nout, d_nmass, d_nin, zero_sum ? 1 : 0, player,
                                             d_leafV);
        e = cudaGetLastError();
        return e == cudaSuccess ? 0 : ffail("net outputs", e);
    }

    // one CFR half-iteration for `player`
    int cfr_pass(int player) {
        if (int st = down<float>(d_R, d_reg, 0)) return st;
        if (net) {
            if (int st = net_leaves(player)) return st;
        } else if (int st = rivers<float>(0, kBModeCFR, player, 0, d_R, d_leafV)) {
            return st;
        }
        if (int st = rivers<float>(1, kBModeCFR, player, 0, d_R, d_leafV)) return st;
        return up<float, kUpCFR>(player, d_R, d_V, d_leafV, d_reg, 0);
    }

    int iteration() {
        for (int p = 0; p < 2; p++)
            if (int st = cfr_pass(p)) return st;
        if (linear) {
            bump_kernel<<<1, 1, 0, stream>>>(d_wt);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return ffail("weight update", e);
        }
        return 0;
    }

    int set_weight(float w) {
        cudaError_t e = cudaMemcpyAsync(d_wt, &w, sizeof(float), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        return e == cudaSuccess ? 0 : ffail("weight reset", e);
    }
};

bool rules_of(const pr_street &s, StreetRules *r) {
    if (s.nfrac < 0 || s.nfrac > kFMaxFracs) return false;
    r->nfrac = s.nfrac;
    for (int k = 0; k < s.nfrac; k++) r->fracs[k] = s.fracs[k];
    r->allin = s.allin != 0;
    r->max_raises = s.max_raises;
    return true;
}

bool build(const pr_full_spec *spec, int max_nodes, FullTree *t) {
    StreetRules fr, tr;
    if (!spec || !rules_of(spec->street[0], &fr) || !rules_of(spec->street[1], &tr)) return false;
    // the river subgames' rules (pr_subgame.sizes and max_raises)
    if ((spec->river_sizes & 7u) == 0 || (spec->river_sizes & ~7u) || spec->river_raises < 1 || spec->river_raises > 3)
        return false;
    return build_full_tree(spec->flop, spec->pot, spec->stack, fr, tr, max_nodes, t);
}

constexpr int kMaxFullNodes = 1 << 20;

}  // namespace
}  // namespace prb

using namespace prb;

namespace {
// pr_full_exploitability's measurement: optional river re-solve, then the FP64 best responses.
int full_exploitability(Game *g, int resolve_iterations, double *br0, double *br1, double *expl) {
    if (resolve_iterations > 0 && g->batch[0]) {
        if (int st = g->down<float>(g->d_R, g->d_avg, 1)) return st;
        const BatchView &v = g->view[0];
        scatter_kernel<float><<<v.count, FT, 0, g->stream>>>(v.packs, g->d_R, g->d_slots[0], v.ranges);
        if (int st = batch_clear(g->batch[0], g->stream)) return st;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) return ffail("re-solve setup", e);
        if (int st = pr_batch_iterate(g->batch[0], resolve_iterations)) return st;
    }
    double br[2];
    for (int p = 0; p < 2; p++) {
        if (int st = g->down<double>(g->d_R64, g->d_avg, 1)) return st;
        for (int b = 0; b < 2; b++)
            if (int st = g->rivers<double>(b, kBModeBR, p, 1, g->d_R64, g->d_leafV64)) return st;
        if (int st = g->up<double, kUpBR>(p, g->d_R64, g->d_V64, g->d_leafV64, g->d_avg, 1)) return st;
        root_sum_kernel<<<1, FT, 0, g->stream>>>(g->d_V64, g->d_init, p, g->d_sum);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&br[p], g->d_sum, sizeof(double), cudaMemcpyDeviceToHost, g->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) return ffail("best response", e);
    }
    if (br0) *br0 = br[0];
    if (br1) *br1 = br[1];
    if (expl) *expl = (br[0] + br[1]) / 2.0 / g->joint;
    return 0;
}
}  // namespace

extern "C" {

int pr_full_tree(const pr_full_spec *spec, void *nodes_out, int max_nodes, int *num_nodes, int *num_edges,
                 int *num_leaves, int *kids_out, int max_kids) {
    FullTree t;
    if (!build(spec, max_nodes > 0 ? max_nodes : kMaxFullNodes, &t)) return 2;
    if (num_nodes) *num_nodes = (int)t.nodes.size();
    if (num_edges) *num_edges = t.num_edges;
    if (num_leaves) *num_leaves = (int)t.leaves.size();
    if (nodes_out) {
        if ((int)t.nodes.size() > max_nodes) return 2;
        memcpy(nodes_out, t.nodes.data(), t.nodes.size() * sizeof(FNode));
    }
    if (kids_out) {
        if ((int)t.kids.size() > max_kids) return 2;
        memcpy(kids_out, t.kids.data(), t.kids.size() * sizeof(int32_t));
    }
    return 0;
}

void *pr_full_new(const pr_full_spec *spec, const float *ranges) {
    if (!spec || !ranges) {
        ffail("pr_full_new: bad arguments");
        return nullptr;
    }
    for (int i = 0; i < 2 * kH; i++)
        if (!std::isfinite(ranges[i]) || ranges[i] < 0.0f) {
            ffail("pr_full_new: a range holds a NaN, an infinity or a negative weight");
            return nullptr;
        }
    Game *g = new Game();
    g->spec = *spec;
    if (!build(spec, kMaxFullNodes, &g->tree)) {
        ffail("pr_full_new: bad spec or tree too large");
        delete g;
        return nullptr;
    }
    const FullTree &t = g->tree;
    g->N = (int)t.nodes.size();
    g->E = t.num_edges;
    g->L = (int)t.leaves.size();
    g->levels.assign(t.levels, {});
    g->deals.assign(t.levels, {});
    for (int i = 0; i < g->N; i++) (t.nodes[i].kind == kFDeal ? g->deals : g->levels)[t.nodes[i].level].push_back(i);
    std::vector<int> flat;
    for (int l = 0; l < t.levels; l++) {
        g->level_off.push_back((int)flat.size());
        flat.insert(flat.end(), g->levels[l].begin(), g->levels[l].end());
        g->deal_off.push_back((int)flat.size());
        flat.insert(flat.end(), g->deals[l].begin(), g->deals[l].end());
    }
    // initial ranges, hands on the flop removed; joint mass of clash-free pairs
    g->init.assign(2 * kH, 0.0f);
    for (int pl = 0; pl < 2; pl++)
        for (int h = 0; h < kH; h++) {
            int c1, c2;
            hand_cards(h, &c1, &c2);
            if (!(((1ull << c1) | (1ull << c2)) & spec->flop)) g->init[pl * kH + h] = ranges[pl * kH + h];
        }
    {
        double tot = 0, card[52] = {0};
        for (int h = 0; h < kH; h++) {
            int c1, c2;
            hand_cards(h, &c1, &c2);
            tot += g->init[kH + h];
            card[c1] += g->init[kH + h];
            card[c2] += g->init[kH + h];
        }
        for (int h = 0; h < kH; h++) {
            int c1, c2;
            hand_cards(h, &c1, &c2);
            g->joint += (double)g->init[h] * (tot - card[c1] - card[c2] + g->init[kH + h]);
        }
    }
    // river subgames of every leaf
    std::vector<pr_subgame> specs[2];
    for (int l = 0; l < g->L; l++) {
        const int node = t.leaves[l];
        const FNode &nd = t.nodes[node];
        const int b = nd.stack > 0.0f ? 0 : 1;
        g->slots[b].push_back(node);
        for (int c = 0; c < 52; c++) {
            if ((nd.board >> c) & 1) continue;
            pr_subgame s{};
            s.board = nd.board | (1ull << c);
            s.pot = nd.stake;
            s.stack = nd.stack;
            s.sizes = spec->river_sizes;
            s.max_raises = spec->river_raises;
            specs[b].push_back(s);
        }
    }
    cudaError_t e;
    const size_t nodes_b = sizeof(FNode) * g->N, rows = (size_t)g->E * kH * sizeof(float);
    if ((e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_nodes, nodes_b)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_kids, sizeof(int) * std::max<size_t>(1, t.kids.size()))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_levels, sizeof(int) * flat.size())) != cudaSuccess ||
        (e = cudaMalloc(&g->d_reg, std::max<size_t>(rows, 4))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_avg, std::max<size_t>(rows, 4))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_init, sizeof(float) * 2 * kH)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_R, sizeof(float) * 2 * kH * g->N)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_V, sizeof(float) * kH * g->N)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_leafV, sizeof(float) * kH * std::max(1, g->L))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_R64, sizeof(double) * 2 * kH * g->N)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_V64, sizeof(double) * kH * g->N)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_leafV64, sizeof(double) * kH * std::max(1, g->L))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_sum, sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_wt, sizeof(float))) != cudaSuccess) {
        ffail("allocation", e);
        delete g;
        return nullptr;
    }
    std::vector<double> init64(g->init.begin(), g->init.end());
    if ((e = cudaMemcpy(g->d_nodes, t.nodes.data(), nodes_b, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (t.kids.size() &&
         (e = cudaMemcpy(g->d_kids, t.kids.data(), sizeof(int) * t.kids.size(), cudaMemcpyHostToDevice)) !=
             cudaSuccess) ||
        (e = cudaMemcpy(g->d_levels, flat.data(), sizeof(int) * flat.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemset(g->d_reg, 0, std::max<size_t>(rows, 4))) != cudaSuccess ||
        (e = cudaMemset(g->d_avg, 0, std::max<size_t>(rows, 4))) != cudaSuccess ||
        (e = cudaMemset(g->d_leafV, 0, sizeof(float) * kH * std::max(1, g->L))) != cudaSuccess ||
        (e = cudaMemcpy(g->d_init, g->init.data(), sizeof(float) * 2 * kH, cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(g->d_R, g->init.data(), sizeof(float) * 2 * kH, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(g->d_R64, init64.data(), sizeof(double) * 2 * kH, cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
        ffail("upload", e);
        delete g;
        return nullptr;
    }
    for (int b = 0; b < 2; b++) {
        if (specs[b].empty()) continue;
        const int count = (int)specs[b].size();
        std::vector<float> zero((size_t)count * 2 * kH, 0.0f);
        g->batch[b] = pr_batch_new(specs[b].data(), count, zero.data());
        if (!g->batch[b] || pr_batch_enable_average(g->batch[b]) || batch_set_own_weight(g->batch[b], true) ||
            batch_set_avg_weight(g->batch[b], g->d_wt) || batch_view(g->batch[b], &g->view[b], true)) {
            ffail("river subgames");
            delete g;
            return nullptr;
        }
        if ((e = cudaMalloc(&g->d_slots[b], sizeof(int) * g->slots[b].size())) != cudaSuccess ||
            (e = cudaMemcpy(g->d_slots[b], g->slots[b].data(), sizeof(int) * g->slots[b].size(),
                            cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMalloc(&g->d_root[b], sizeof(double) * kBRow * count)) != cudaSuccess) {
            ffail("river subgame buffers", e);
            delete g;
            return nullptr;
        }
    }
    if (g->set_weight(1.0f)) {
        delete g;
        return nullptr;
    }
    return g;
}

void pr_full_free(void *game) { delete (Game *)game; }

// Average sums weighted by the iteration number (on, the default: iteration t adds t x
// reach x strategy, the usual weighting with regrets clipped at zero) or by 1 (off). The
// weight restarts at 1.
int pr_full_set_linear_average(void *game, int on) {
    Game *g = (Game *)game;
    if (!g) return 2;
    if (g->graph) {
        cudaGraphExecDestroy(g->graph);
        g->graph = nullptr;
    }
    g->graph_failed = false;
    g->linear = on != 0;
    return g->set_weight(1.0f);
}

int pr_full_shape(void *game, int *num_nodes, int *num_edges, int *num_leaves, int *bet_subgames,
                  int *allin_subgames) {
    Game *g = (Game *)game;
    if (!g) return 2;
    if (num_nodes) *num_nodes = g->N;
    if (num_edges) *num_edges = g->E;
    if (num_leaves) *num_leaves = g->L;
    if (bet_subgames) *bet_subgames = g->batch[0] ? g->view[0].count : 0;
    if (allin_subgames) *allin_subgames = g->batch[1] ? g->view[1].count : 0;
    return 0;
}

// Net-leaf mode: leaves with chips behind take their values from the value network (null:
// back to the river subgames). The network's batch rows bound one forward call; larger leaf
// sets run in several.
int pr_full_set_net(void *game, void *net) {
    Game *g = (Game *)game;
    if (!g) return 2;
    if (g->graph) {
        cudaGraphExecDestroy(g->graph);
        g->graph = nullptr;
    }
    g->graph_failed = false;
    g->net = net;
    if (!net) return 0;
    g->net_rows = pr_mlp_rows(net);
    const size_t n = std::max<size_t>(1, g->slots[0].size());
    if (!g->d_nin) {
        cudaError_t e;
        if ((e = cudaMalloc(&g->d_nin, sizeof(float) * 2 * kH * n)) != cudaSuccess ||
            (e = cudaMalloc(&g->d_nscal, sizeof(float) * 2 * n)) != cudaSuccess ||
            (e = cudaMalloc(&g->d_nmass, sizeof(float) * 2 * n)) != cudaSuccess ||
            (e = cudaMalloc(&g->d_nout, sizeof(float) * kNetIn * n)) != cudaSuccess ||
            (e = cudaMalloc(&g->d_nboard, sizeof(unsigned long long) * n)) != cudaSuccess)
            return ffail("net buffers", e);
    }
    return 0;
}

// Net leaves shifted to zero sum (on = 1; see net_out_kernel) or taken as the network gives
// them (0, the default).
int pr_full_set_zero_sum(void *game, int on) {
    Game *g = (Game *)game;
    if (!g) return 2;
    if (g->graph) {
        cudaGraphExecDestroy(g->graph);
        g->graph = nullptr;
    }
    g->zero_sum = on != 0;
    return 0;
}

// Runs the batched solver's autotuner on both river-subgame batches (launch configuration
// per tree-shape class; their solver state is restored). ms_out[4]: the chosen per-pass
// times of batch 0's and batch 1's two classes, or null.
int pr_full_tune(void *game, double *ms_out) {
    Game *g = (Game *)game;
    if (!g) return 2;
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return ffail("tune", e);
    for (int b = 0; b < 2; b++) {
        double ms[2] = {0.0, 0.0};
        if (g->batch[b])
            if (int st = pr_batch_tune(g->batch[b], ms)) return st;
        if (ms_out) {
            ms_out[2 * b] = ms[0];
            ms_out[2 * b + 1] = ms[1];
        }
    }
    if (g->graph) {
        cudaGraphExecDestroy(g->graph);
        g->graph = nullptr;
    }
    g->graph_failed = false;
    return 0;
}

// One CFR half-iteration for `player` (tests; pr_full_iterate runs whole iterations).
int pr_full_pass(void *game, int player) {
    Game *g = (Game *)game;
    if (!g || (player != 0 && player != 1)) return 2;
    if (int st = g->cfr_pass(player)) return st;
    cudaError_t e = cudaStreamSynchronize(g->stream);
    return e == cudaSuccess ? 0 : ffail("pass", e);
}

// CFR iterations (both players, alternating). Without a network each iteration is one
// CUDA graph, captured on the first call.
int pr_full_iterate(void *game, int iterations) {
    prb::TraceRange trace("full game iterations");
    Game *g = (Game *)game;
    if (!g || iterations < 0) return 2;
    int it = 0;
    if (!g->net && !g->graph && !g->graph_failed && iterations > 0) {
        if (int st = g->iteration()) return st;
        it++;
        cudaError_t e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) return ffail("iteration", e);
        cudaGraph_t gr = nullptr;
        int st = 0;
        e = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            st = g->iteration();
            e = cudaStreamEndCapture(g->stream, &gr);
        }
        if (e == cudaSuccess && !st && gr) e = cudaGraphInstantiate(&g->graph, gr, 0);
        if (gr) cudaGraphDestroy(gr);
        if (e != cudaSuccess || st || !g->graph) {
            cudaGetLastError();
            g->graph = nullptr;
            g->graph_failed = true;
        }
    }
    for (; it < iterations; it++) {
        if (g->graph && !g->net) {
            cudaError_t e = cudaGraphLaunch(g->graph, g->stream);
            if (e != cudaSuccess) return ffail("graph launch", e);
        } else if (int st = g->iteration()) {
            return st;
        }
    }
    cudaError_t e = cudaStreamSynchronize(g->stream);
    return e == cudaSuccess ? 0 : ffail("iteration", e);
}

// FP64 best responses of both players to the other's average strategies over the whole game
// (flop and turn sweeps in double, river subgames by the batch solver's double best
// response), and exploitability = (BR0 + BR1) / 2 per unit of joint range mass, in chips.
// resolve_iterations > 0 first re-solves the river subgames of the leaves with chips behind
// from zero, for that many CFR iterations, under the reach of the current average flop and
// turn strategies (the net-leaf mode's strategies stop at the turn). In net-leaf mode their
// previous regrets and average sums are replaced; in plain mode, where they are part of the
// solve, they are kept aside and restored afterwards.
int pr_full_exploitability(void *game, int resolve_iterations, double *br0, double *br1, double *expl) {
    prb::TraceRange trace("full game exploitability");
    Game *g = (Game *)game;
    if (!g || resolve_iterations < 0) return 2;
    // In plain mode the river subgames belong to the solve: their rows are kept aside during
    // the re-solve and put back afterwards, so that measuring does not change the solve.
    float *keep = nullptr, *rows_r = nullptr, *rows_a = nullptr;
    size_t row_bytes = 0;
    if (resolve_iterations > 0 && g->batch[0] && !g->net) {
        if (int st = batch_rows(g->batch[0], &rows_r, &rows_a, &row_bytes)) return st;
        cudaError_t e = cudaMalloc(&keep, row_bytes * (rows_a ? 2 : 1));
        if (e == cudaSuccess) e = cudaMemcpyAsync(keep, rows_r, row_bytes, cudaMemcpyDeviceToDevice, g->stream);
        if (e == cudaSuccess && rows_a)
            e = cudaMemcpyAsync((char *)keep + row_bytes, rows_a, row_bytes, cudaMemcpyDeviceToDevice, g->stream);
        if (e != cudaSuccess) {
            cudaFree(keep);
            return ffail("re-solve: keeping the river rows", e);
        }
    }
    const int st = full_exploitability(g, resolve_iterations, br0, br1, expl);
    if (keep) {
        cudaError_t e = cudaMemcpyAsync(rows_r, keep, row_bytes, cudaMemcpyDeviceToDevice, g->stream);
        if (e == cudaSuccess && rows_a)
            e = cudaMemcpyAsync(rows_a, (char *)keep + row_bytes, row_bytes, cudaMemcpyDeviceToDevice, g->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        cudaFree(keep);
        if (e != cudaSuccess) return ffail("re-solve: restoring the river rows", e);
    }
    return st;
}



// Device state, for tests and checkpoints. which: 0 regrets, 1 average sums ([edges][1326]
// floats); 2 reach ([nodes][2][1326] floats), 3 leaf values ([leaves][1326] floats),
// 4 node values ([nodes][1326] floats) of the last CFR pass; 5, 6, 7 the same three in
// double from the last best response; 8, 9 the network inputs (normalised ranges) and reach
// masses of the last net-leaf pass.
int pr_full_read(void *game, int which, void *out) {
    Game *g = (Game *)game;
    if (!g || !out) return 2;
    const void *src = nullptr;
    size_t bytes = 0;
    switch (which) {
        case 0: src = g->d_reg; bytes = sizeof(float) * kH * g->E; break;
        case 1: src = g->d_avg; bytes = sizeof(float) * kH * g->E; break;
        case 2: src = g->d_R; bytes = sizeof(float) * 2 * kH * g->N; break;
        case 3: src = g->d_leafV; bytes = sizeof(float) * kH * g->L; break;
        case 4: src = g->d_V; bytes = sizeof(float) * kH * g->N; break;
        case 5: src = g->d_R64; bytes = sizeof(double) * 2 * kH * g->N; break;
        case 6: src = g->d_leafV64; bytes = sizeof(double) * kH * g->L; break;
        case 7: src = g->d_V64; bytes = sizeof(double) * kH * g->N; break;
        case 8:  // net-leaf inputs of the last pass: ranges [leaves with chips behind][2][1326]
            src = g->d_nin;
            bytes = g->d_nin ? sizeof(float) * 2 * kH * g->slots[0].size() : 0;
            break;
        case 9:  // and the reach masses [..][2] that scale the outputs back
            src = g->d_nmass;
            bytes = g->d_nmass ? sizeof(float) * 2 * g->slots[0].size() : 0;
            break;
        default: return 2;
    }
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e == cudaSuccess && bytes) e = cudaMemcpy(out, src, bytes, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : ffail("read", e);
}

// Back to the start: zero regrets and average sums of the flop and turn and of every river
// subgame.
int pr_full_reset(void *game) {
    Game *g = (Game *)game;
    if (!g) return 2;
    const size_t rows = std::max<size_t>((size_t)g->E * kH * sizeof(float), 4);
    cudaError_t e = cudaMemsetAsync(g->d_reg, 0, rows, g->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(g->d_avg, 0, rows, g->stream);
    if (e != cudaSuccess) return ffail("reset", e);
    for (int b = 0; b < 2; b++)
        if (g->batch[b])
            if (int st = batch_clear(g->batch[b], g->stream)) return st;
    e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return ffail("reset", e);
    return g->set_weight(1.0f);
}

// Replaces the regrets (which 0) or average sums (which 1), [edges][1326] floats.
int pr_full_write(void *game, int which, const void *in) {
    Game *g = (Game *)game;
    if (!g || !in || (which != 0 && which != 1)) return 2;
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e == cudaSuccess && g->E)
        e = cudaMemcpy(which == 0 ? g->d_reg : g->d_avg, in, sizeof(float) * kH * g->E, cudaMemcpyHostToDevice);
    return e == cudaSuccess ? 0 : ffail("write", e);
}

// The river-subgame batch of the leaves with chips behind (which 0) or of the all-in leaves
// (which 1), or null; subgame j * 48 + k is river card k (in card order) of the batch's
// j-th leaf (leaves in pre-order). Owned by the game.
void *pr_full_batch(void *game, int which) {
    Game *g = (Game *)game;
    if (!g || which < 0 || which > 1) return nullptr;
    return g->batch[which];
}

// Leaf node ids of batch `which`, in its order.
int pr_full_batch_leaves(void *game, int which, int *nodes_out) {
    Game *g = (Game *)game;
    if (!g || which < 0 || which > 1) return -1;
    if (nodes_out) memcpy(nodes_out, g->slots[which].data(), sizeof(int) * g->slots[which].size());
    return (int)g->slots[which].size();
}

double pr_full_joint(void *game) { return game ? ((Game *)game)->joint : 0.0; }

}  // extern "C"
