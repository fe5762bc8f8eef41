// C ABI of the batched general-subgame solver (pr_batch_*; no reference counterpart): batch
// construction, CFR iterations replayed as a CUDA graph, per-subgame exploitability in
// single or double precision, strategy evaluation (root values), regret / average access
// and the autotuner that picks the launch configuration per tree-shape class.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <thread>
#include <numeric>
#include <vector>

#include "../../include/pokerrust_b200.h"
#include "batch_internal.h"
#include "batch_solver.h"
#include "device_common.cuh"
#include "trace.h"

namespace prb {
namespace {

// True when every weight of n is finite and, with `nonneg`, not negative (v - v is NaN for NaN
// and infinities).
bool valid_weights(const float *r, size_t n, bool nonneg = true) {
    float bad = 0.0f;
    for (size_t i = 0; i < n; i++) bad += (r[i] - r[i]) + (nonneg && r[i] < 0.0f ? 1.0f : 0.0f);
    return bad == 0.0f;
}

int bfail(const char *what, cudaError_t e = cudaSuccess) {
    if (e != cudaSuccess) fprintf(stderr, "pokerrust_b200: batch: %s: %s\n", what, cudaGetErrorString(e));
    else fprintf(stderr, "pokerrust_b200: batch: %s\n", what);
    fflush(stderr);
    return e != cudaSuccess ? 1 : 2;
}

// Launch configuration of one tree-shape class.
struct ClassCfg {
    int first = 0, count = 0;  // slice of the work queue
    int max_leaves = 0;
    int K = 2;                 // hands per thread
    int per_sm = 1;            // resident CTAs per SM
    int order = 0;             // 0: most work first, 1: input order
};

constexpr int kClasses = 2;    // trees with <= 16 leaves / more

struct Batch {
    int count = 0;
    std::vector<pr_subgame> specs;
    std::vector<BSub> subs;
    std::vector<BNode> nodes;
    std::vector<double> joint;  // sum over clash-free hand pairs of r0(h) r1(o)
    int total_edges = 0;
    int sms = 148;
    ClassCfg cls[kClasses];
    bool avg_on = false;
    bool tuned = false;
    cudaStream_t stream = nullptr;
    BSub *d_subs = nullptr;
    BNode *d_nodes = nullptr;
    BPack *d_packs = nullptr;
    float *d_ranges = nullptr;
    double *d_ranges64 = nullptr;  // [count][2][kBRow] double ranges of best responses inside a larger game
    bool own_weight = false;       // CFR average sums weighted by the updater's range
    const float *avg_weight = nullptr;  // device scalar weighting CFR average-sum terms (null: 1)
    float *d_wt = nullptr;              // the batch's own weight scalar (linear averaging)
    bool linear = false;                // iteration t adds t x its average-sum terms
    float *d_regrets = nullptr, *d_avg = nullptr;
    int *d_order = nullptr, *d_head = nullptr, *d_err = nullptr;
    void *d_sum = nullptr;   // [count] doubles
    void *d_root = nullptr;  // [count][kBRow] doubles, lazily
    void *d_child = nullptr; // [count][8][kBRow] doubles, lazily
    double *d_hands = nullptr;  // [count][10][1326] doubles, lazily: results in hand order for host copies
    double *h_pinned = nullptr;  // pinned host copy of d_hands, lazily (the adjoint's host outputs)
    std::vector<uint16_t> hand;  // [count][kBRow] colex hand of each position
    cudaGraphExec_t graph = nullptr;
    bool graph_avg = false, graph_failed = false;

    ~Batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (h_pinned) cudaFreeHost(h_pinned);
        if (stream) cudaStreamSynchronize(stream);
        for (void *p : {(void *)d_subs, (void *)d_nodes, (void *)d_packs, (void *)d_ranges, (void *)d_ranges64,
                        (void *)d_regrets, (void *)d_avg, (void *)d_order, (void *)d_head, (void *)d_err, d_sum,
                        d_root, d_child, (void *)d_wt, (void *)d_hands})
            cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }

    // the order of the work queue: per class, most work first or input order
    void build_order(std::vector<int> &order) const {
        order.clear();
        for (int c = 0; c < kClasses; c++) {
            std::vector<int> ids;
            for (int s = 0; s < count; s++)
                if ((subs[s].num_leaves > batch_group_leaves(0)) == (c == 1)) ids.push_back(s);
            if (cls[c].order == 0)
                std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) {
                    const long wa = (long)subs[a].num_edges * 4 + subs[a].num_leaves;
                    const long wb = (long)subs[b].num_edges * 4 + subs[b].num_leaves;
                    return wa > wb;
                });
            order.insert(order.end(), ids.begin(), ids.end());
        }
    }

    int upload_order() {
        std::vector<int> order;
        build_order(order);
        cudaError_t e = cudaMemcpy(d_order, order.data(), sizeof(int) * count, cudaMemcpyHostToDevice);
        return e == cudaSuccess ? 0 : bfail("queue upload", e);
    }

    // one pass of `mode` for `player` over every class; heads [slot*kClasses + c] must be zero.
    // `queue` / `heads` replace the batch's own work-queue order and heads when given.
    int pass(int mode, int player, int fp64, int use_average, void *root_out, void *sum_out, int slot,
             void *child_out = nullptr, cudaStream_t on = nullptr, const int *queue = nullptr,
             int *heads = nullptr) {
        for (int c = 0; c < kClasses; c++) {
            const ClassCfg &k = cls[c];
            if (!k.count) continue;
            BLaunch a{};
            a.subs = d_subs;
            a.nodes = d_nodes;
            a.packs = d_packs;
            a.ranges = d_ranges;
            a.regrets = d_regrets;
            a.avg = (avg_on || use_average) ? d_avg : nullptr;
            a.order = (queue ? queue : d_order) + k.first;
            a.head = (heads ? heads : d_head) + slot * kClasses + c;
            a.count = k.count;
            a.player = player;
            a.use_average = use_average;
            a.root_out = root_out;
            a.sum_out = sum_out;
            a.child_out = child_out;
            a.ranges64 = fp64 ? d_ranges64 : nullptr;
            a.own_reach = own_weight;
            a.avg_weight = avg_weight;
            const int ctas = std::min(k.count, std::max(1, k.per_sm) * sms);
            const int dense = mode == kBModeCFR && !fp64 && k.K == 4 && k.per_sm >= 3;
            const int group = dense ? batch_dense_group() : batch_group_leaves(fp64);
            cudaError_t e = launch_batch_pass(mode, k.K, fp64, mode == kBModeCFR && avg_on, a, ctas, group,
                                              on ? on : stream, dense);
            if (e != cudaSuccess) return bfail("pass launch", e);
        }
        return 0;
    }

    // One CFR iteration (both players, then the linear-average weight step). `queue` / `heads`
    // (2 * kClasses ints) replace the batch's own work queue when given.
    int iteration(const int *queue = nullptr, int *heads = nullptr) {
        cudaError_t e = cudaMemsetAsync(heads ? heads : d_head, 0, sizeof(int) * 2 * kClasses, stream);
        if (e != cudaSuccess) return bfail("queue reset", e);
        for (int pl = 0; pl < 2; pl++)
            if (int st = pass(kBModeCFR, pl, 0, 0, nullptr, nullptr, pl, nullptr, nullptr, queue, heads)) return st;
        if (linear) {
            e = launch_weight_step(d_wt, stream);
            if (e != cudaSuccess) return bfail("weight update", e);
        }
        return 0;
    }
};

// Position-order rows [count][rows][kBRow] -> hand-order rows [count][rows][1326] (hands that
// touch the board are 0), times `sign`; with `weight` (position-order ranges [count][2][kBRow])
// each value is first multiplied by player 0's range of the hand.
__global__ void to_hands_kernel(const double *__restrict__ src, const BPack *__restrict__ packs, int rows,
                                double sign, const float *__restrict__ weight, double *__restrict__ dst) {
    const int s = blockIdx.x, r = blockIdx.y;
    const uint16_t *pos_of = packs[s].pos_of;
    const double *row = src + ((size_t)s * rows + r) * kBRow;
    const float *w = weight ? weight + (size_t)s * 2 * kBRow : nullptr;
    double *out = dst + ((size_t)s * rows + r) * 1326;
    for (int h = threadIdx.x; h < 1326; h += blockDim.x) {
        const int p = pos_of[h];
        double v = 0.0;
        if (p != 0xFFFF) {
            v = row[p];
            if (w) v = (double)w[p] * v;
        }
        out[h] = sign * v;
    }
}

// Rows [edge][kBRow] (position order) of subgames [first, first + gridDim.x) -> rows
// [edge - edge_base][1326] (colex order; hands on the board 0), one CTA per subgame.
__global__ void rows_to_hands_kernel(const float *__restrict__ src, const BSub *__restrict__ subs,
                                     const BPack *__restrict__ packs, int first, int edge_base,
                                     float *__restrict__ dst) {
    const int s = first + blockIdx.x;
    const BSub d = subs[s];
    const uint16_t *pos_of = packs[s].pos_of;
    for (int k = 0; k < d.num_edges; k++) {
        const float *row = src + (size_t)(d.edge_off + k) * kBRow;
        float *out = dst + (size_t)(d.edge_off + k - edge_base) * 1326;
        for (int h = threadIdx.x; h < 1326; h += blockDim.x) {
            const int p = pos_of[h];
            out[h] = p != 0xFFFF ? row[p] : 0.0f;
        }
    }
}

int to_hands(Batch *b, const void *src, int rows, double sign, const float *weight, double *dst) {
    to_hands_kernel<<<dim3(b->count, rows), 256, 0, b->stream>>>((const double *)src, b->d_packs, rows, sign, weight,
                                                                dst);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : bfail("hand-order copy", e);
}

int ensure_hands_buffer(Batch *b) {
    if (b->d_hands) return 0;
    cudaError_t e = cudaMalloc(&b->d_hands, sizeof(double) * 10 * 1326 * (size_t)b->count);
    return e == cudaSuccess ? 0 : bfail("hand-order buffer allocation", e);
}

// The two evaluation passes of the adjoint, results in hand order on the device (null outputs
// skipped); see pr_batch_value_grad.
int value_grad_device(Batch *b, int use_average, double *d_r0, double *d_r1, double *d_sigma) {
    cudaError_t e;
    if (!b->d_root && (e = cudaMalloc(&b->d_root, sizeof(double) * kBRow * b->count)) != cudaSuccess)
        return bfail("root value allocation", e);
    if (!b->d_child && (e = cudaMalloc(&b->d_child, sizeof(double) * 8 * kBRow * b->count)) != cudaSuccess)
        return bfail("root value allocation", e);
    for (int pl = 0; pl < 2; pl++) {
        e = cudaMemsetAsync(b->d_head, 0, sizeof(int) * 4 * kClasses, b->stream);
        if (e == cudaSuccess && pl == 0)
            e = cudaMemsetAsync(b->d_child, 0, sizeof(double) * 8 * kBRow * b->count, b->stream);
        if (e != cudaSuccess) return bfail("queue reset", e);
        if (int st = b->pass(kBModeEval, pl, 1, use_average, b->d_root, nullptr, 0, pl == 0 ? b->d_child : nullptr))
            return st;
        double *out = pl == 0 ? d_r0 : d_r1;
        if (out)
            if (int st = to_hands(b, b->d_root, 1, pl == 0 ? 1.0 : -1.0, nullptr, out)) return st;
        if (pl == 0 && d_sigma)
            if (int st = to_hands(b, b->d_child, 8, 1.0, b->d_ranges, d_sigma)) return st;
    }
    e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? 0 : bfail("adjoint", e);
}

// ---- no-allocation iteration ----
// Work-queue scratch of pr_batch_iterate_noalloc: kClasses * 2 queue heads, then the queue
// order of up to kNoAllocMaxSubgames subgames, 256 KB in all. It is a fixed device array of
// the library, so every GPU that loads the library holds it until the process exits, and
// the entry point needs no allocation. Host code only sees a stand-in for this name; the
// device address comes from cudaGetSymbolAddress (noalloc_scratch below).
constexpr int kNoAllocMaxSubgames = 65536;
constexpr int kNoAllocHeads = 2 * kClasses;
static __device__ __align__(256) int g_noalloc_scratch[kNoAllocHeads + kNoAllocMaxSubgames];

std::mutex g_noalloc_mu;
int *g_noalloc_ptr[64] = {};  // per device, looked up once with that device current

int *noalloc_scratch() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            bfail("no-allocation scratch lookup", e);
            return nullptr;
        }
        g_noalloc_ptr[dev] = (int *)p;
    }
    return g_noalloc_ptr[dev];
}

}  // namespace

int batch_view(void *batch, BatchView *v, bool need64) {
    Batch *b = (Batch *)batch;
    if (!b || !v) return 2;
    if (need64 && !b->d_ranges64) {
        const size_t bytes = sizeof(double) * 2 * kBRow * b->count;
        cudaError_t e = cudaMalloc(&b->d_ranges64, bytes);
        if (e == cudaSuccess) e = cudaMemset(b->d_ranges64, 0, bytes);
        if (e != cudaSuccess) return bfail("double range allocation", e);
    }
    v->packs = b->d_packs;
    v->ranges = b->d_ranges;
    v->ranges64 = b->d_ranges64;
    v->count = b->count;
    v->stream = b->stream;
    return 0;
}

int batch_set_own_weight(void *batch, bool on) {
    Batch *b = (Batch *)batch;
    if (!b) return 2;
    if (b->own_weight != on && b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->own_weight = on;
    return 0;
}

int batch_set_avg_weight(void *batch, const float *weight) {
    Batch *b = (Batch *)batch;
    if (!b) return 2;
    if (b->avg_weight != weight && b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->avg_weight = weight;
    return 0;
}

int batch_run_pass(void *batch, int mode, int player, int fp64, int use_average, void *root_out,
                   cudaStream_t on) {
    Batch *b = (Batch *)batch;
    if (!b || (use_average && !b->avg_on) || (mode == kBModeCFR && fp64)) return 2;
    const int slot = 3;  // heads of this slot are reset here, on the caller's stream
    cudaError_t e = cudaMemsetAsync(b->d_head + slot * kClasses, 0, sizeof(int) * kClasses, on);
    if (e != cudaSuccess) return bfail("queue reset", e);
    return b->pass(mode, player, fp64, use_average, root_out, nullptr, slot, nullptr, on);
}

int batch_rows(void *batch, float **regrets, float **avg, size_t *bytes) {
    Batch *b = (Batch *)batch;
    if (!b) return 2;
    *regrets = b->d_regrets;
    *avg = b->d_avg;
    *bytes = (size_t)b->total_edges * kBRow * sizeof(float);
    return 0;
}

int batch_clear(void *batch, cudaStream_t on) {
    Batch *b = (Batch *)batch;
    if (!b) return 2;
    const size_t rows = (size_t)b->total_edges * kBRow * sizeof(float);
    cudaError_t e = cudaMemsetAsync(b->d_regrets, 0, rows, on);
    if (e == cudaSuccess && b->d_avg) e = cudaMemsetAsync(b->d_avg, 0, rows, on);
    return e == cudaSuccess ? 0 : bfail("clear", e);
}

}  // namespace prb

using namespace prb;

extern "C" {

int pr_batch_tree(const pr_subgame *spec, void *nodes_out, int *num_nodes, int *num_edges, int *num_leaves) {
    if (!spec) return 2;
    BTree t;
    if (spec->max_raises < 1 || spec->max_raises > 3) return 2;
    if (!build_bet_tree(spec->pot, spec->stack, spec->sizes, spec->max_raises, &t) || t.depth >= 6) return 2;
    if (nodes_out) memcpy(nodes_out, t.nodes.data(), t.nodes.size() * sizeof(BNode));
    if (num_nodes) *num_nodes = (int)t.nodes.size();
    if (num_edges) *num_edges = t.num_edges;
    if (num_leaves) *num_leaves = t.num_leaves;
    return 0;
}

void *pr_batch_new(const pr_subgame *specs, int count, const float *ranges) {
    if (!specs || count <= 0 || !ranges) {
        bfail("pr_batch_new: bad arguments");
        return nullptr;
    }
    if (!valid_weights(ranges, (size_t)2 * 1326 * count)) {
        bfail("pr_batch_new: a range holds a NaN, an infinity or a negative weight");
        return nullptr;
    }
    Batch *b = new Batch();
    b->count = count;
    b->specs.assign(specs, specs + count);
    b->subs.resize(count);
    b->joint.resize(count);
    int edges = 0;
    for (int s = 0; s < count; s++) {
        const pr_subgame &sp = specs[s];
        BTree t;
        if (__builtin_popcountll(sp.board) != 5 || (sp.board >> 52) || sp.max_raises < 1 || sp.max_raises > 3 ||
            !build_bet_tree(sp.pot, sp.stack, sp.sizes, sp.max_raises, &t) || t.depth >= 6) {
            fprintf(stderr, "pokerrust_b200: batch: subgame %d has a bad board or bet tree\n", s);
            delete b;
            return nullptr;
        }
        BSub &d = b->subs[s];
        d.board = sp.board;
        d.node_off = (int)b->nodes.size();
        d.num_nodes = (int)t.nodes.size();
        d.edge_off = edges;
        d.num_edges = t.num_edges;
        d.num_leaves = t.num_leaves;
        d.pot = sp.pot;
        b->nodes.insert(b->nodes.end(), t.nodes.begin(), t.nodes.end());
        edges += t.num_edges;
        // joint mass of clash-free hand pairs (double)
        const float *r0 = ranges + (size_t)s * 2 * 1326, *r1 = r0 + 1326;
        double tot = 0, card[52] = {0};
        for (int h = 0; h < 1326; h++) {
            int c1, c2;
            hand_cards(h, &c1, &c2);
            if (((1ull << c1) | (1ull << c2)) & sp.board) continue;
            tot += r1[h];
            card[c1] += r1[h];
            card[c2] += r1[h];
        }
        double j = 0;
        for (int h = 0; h < 1326; h++) {
            int c1, c2;
            hand_cards(h, &c1, &c2);
            if (((1ull << c1) | (1ull << c2)) & sp.board) continue;
            j += (double)r0[h] * (tot - card[c1] - card[c2] + r1[h]);
        }
        b->joint[s] = j;
    }
    b->total_edges = edges;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    // shape classes
    int first = 0;
    for (int c = 0; c < kClasses; c++) {
        b->cls[c].first = first;
        b->cls[c].count = 0;
        for (int s = 0; s < count; s++)
            if ((b->subs[s].num_leaves > batch_group_leaves(0)) == (c == 1)) {
                b->cls[c].count++;
                b->cls[c].max_leaves = std::max(b->cls[c].max_leaves, b->subs[s].num_leaves);
            }
        first += b->cls[c].count;
    }
    cudaError_t e;
    const size_t rows = (size_t)edges * kBRow * sizeof(float);
    float *d_in = nullptr;
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_subs, sizeof(BSub) * count)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_nodes, sizeof(BNode) * b->nodes.size())) != cudaSuccess ||
        (e = cudaMalloc(&b->d_packs, sizeof(BPack) * count)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_ranges, sizeof(float) * 2 * kBRow * count)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_regrets, rows)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_order, sizeof(int) * count)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_head, sizeof(int) * 4 * kClasses)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_err, sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_sum, sizeof(double) * count)) != cudaSuccess ||
        (e = cudaMalloc(&d_in, sizeof(float) * 2 * 1326 * count)) != cudaSuccess) {
        bfail("allocation", e);
        cudaFree(d_in);
        delete b;
        return nullptr;
    }
    int err = 0;
    if ((e = cudaMemcpy(b->d_subs, b->subs.data(), sizeof(BSub) * count, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(b->d_nodes, b->nodes.data(), sizeof(BNode) * b->nodes.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(d_in, ranges, sizeof(float) * 2 * 1326 * count, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(b->d_regrets, 0, rows)) != cudaSuccess ||
        (e = cudaMemset(b->d_err, 0, sizeof(int))) != cudaSuccess ||
        (e = launch_batch_setup(b->d_subs, count, b->d_packs, d_in, b->d_ranges, b->d_err, b->stream)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(b->stream)) != cudaSuccess ||
        (e = cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) {
        bfail("setup", e);
        cudaFree(d_in);
        delete b;
        return nullptr;
    }
    cudaFree(d_in);
    if (err) {
        bfail("setup found an inconsistent board");
        delete b;
        return nullptr;
    }
    // the hand of every position, one strided copy out of the packs
    b->hand.resize((size_t)count * kBRow);
    e = cudaMemcpy2D(b->hand.data(), sizeof(uint16_t) * kBRow, (const char *)b->d_packs + offsetof(BPack, hand),
                     sizeof(BPack), sizeof(uint16_t) * kBRow, count, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        bfail("pack download", e);
        delete b;
        return nullptr;
    }
    if (b->upload_order()) {
        delete b;
        return nullptr;
    }
    return b;
}

void pr_batch_free(void *batch) { delete (Batch *)batch; }

int pr_batch_count(void *batch) { return batch ? ((Batch *)batch)->count : 0; }

int pr_batch_shape(void *batch, int s, int *num_nodes, int *num_edges, int *num_leaves) {
    Batch *b = (Batch *)batch;
    if (!b || s < 0 || s >= b->count) return 2;
    if (num_nodes) *num_nodes = b->subs[s].num_nodes;
    if (num_edges) *num_edges = b->subs[s].num_edges;
    if (num_leaves) *num_leaves = b->subs[s].num_leaves;
    return 0;
}

int pr_batch_enable_average(void *batch) {
    Batch *b = (Batch *)batch;
    if (!b) return 2;
    if (b->avg_on) return 0;
    const size_t rows = (size_t)b->total_edges * kBRow * sizeof(float);
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_avg, rows)) != cudaSuccess || (e = cudaMemset(b->d_avg, 0, rows)) != cudaSuccess)
        return bfail("average-strategy allocation", e);
    b->avg_on = true;
    // the average-sum kernels use more registers and shared memory: keep every class's
    // resident CTAs per SM within what now fits
    for (int c = 0; c < kClasses; c++) {
        ClassCfg &k = b->cls[c];
        const bool dense = k.K == 4 && k.per_sm >= 3;
        const int fits = dense ? batch_dense_ctas_per_sm(1) : batch_ctas_per_sm(kBModeCFR, k.K, 0, 1);
        if (k.per_sm > fits) k.per_sm = std::max(1, dense && fits < 3 ? std::min(fits, 2) : fits);
    }
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return 0;
}

// Average sums weighted by the iteration number (on: iteration t of the batch adds t x
// reach x strategy; the weighting usual with regrets clipped at zero) or by 1 (off, the
// default). The weight restarts at 1.
int pr_batch_set_linear_average(void *batch, int on) {
    Batch *b = (Batch *)batch;
    if (!b) return 2;
    cudaError_t e;
    if (!b->d_wt && (e = cudaMalloc(&b->d_wt, sizeof(float))) != cudaSuccess) return bfail("weight allocation", e);
    const float one = 1.0f;
    e = cudaMemcpyAsync(b->d_wt, &one, sizeof(float), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail("weight reset", e);
    b->linear = on != 0;
    return batch_set_avg_weight(b, b->linear ? b->d_wt : nullptr);
}

int pr_batch_iterate(void *batch, int iterations) {
    prb::TraceRange trace("batch iterations");
    Batch *b = (Batch *)batch;
    if (!b || iterations < 0) return 2;
    if (b->graph && b->graph_avg != b->avg_on) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    int it = 0;
    if (!b->graph && !b->graph_failed && iterations > 0) {
        if (int st = b->iteration()) return st;
        it++;
        cudaError_t e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) return bfail("iteration", e);
        cudaGraph_t g = nullptr;
        int st = 0;
        e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            st = b->iteration();
            e = cudaStreamEndCapture(b->stream, &g);
        }
        if (e == cudaSuccess && !st && g) e = cudaGraphInstantiate(&b->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess || st || !b->graph) {
            cudaGetLastError();
            b->graph = nullptr;
            b->graph_failed = true;
        }
        b->graph_avg = b->avg_on;
    }
    for (; it < iterations; it++) {
        if (b->graph) {
            cudaError_t e = cudaGraphLaunch(b->graph, b->stream);
            if (e != cudaSuccess) return bfail("graph launch", e);
        } else if (int st = b->iteration()) {
            return st;
        }
    }
    cudaError_t e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? 0 : bfail("iteration", e);
}

// Best-response sums of both players per subgame, and exploitability = (BR0 + BR1) / 2 per
// unit of joint range mass, in chips.
int pr_batch_exploitability(void *batch, int use_average, int fp64, double *br0, double *br1, double *expl) {
    prb::TraceRange trace("batch exploitability");
    Batch *b = (Batch *)batch;
    if (!b || (use_average && !b->avg_on)) return 2;
    std::vector<double> sums[2];
    std::vector<float> sumsf(b->count);
    cudaError_t e = cudaMemsetAsync(b->d_head, 0, sizeof(int) * 4 * kClasses, b->stream);
    if (e != cudaSuccess) return bfail("queue reset", e);
    for (int pl = 0; pl < 2; pl++) {
        sums[pl].resize(b->count);
        if (int st = b->pass(kBModeBR, pl, fp64, use_average, nullptr, b->d_sum, 2 + pl)) return st;
        if (fp64) {
            e = cudaMemcpyAsync(sums[pl].data(), b->d_sum, sizeof(double) * b->count, cudaMemcpyDeviceToHost, b->stream);
        } else {
            e = cudaMemcpyAsync(sumsf.data(), b->d_sum, sizeof(float) * b->count, cudaMemcpyDeviceToHost, b->stream);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) return bfail("best response", e);
        if (!fp64)
            for (int s = 0; s < b->count; s++) sums[pl][s] = sumsf[s];
    }
    for (int s = 0; s < b->count; s++) {
        if (br0) br0[s] = sums[0][s];
        if (br1) br1[s] = sums[1][s];
        if (expl) expl[s] = (sums[0][s] + sums[1][s]) / 2.0 / b->joint[s];
    }
    return 0;
}

// Root values (counterfactual values of `player` at the root, per colex hand; blocked hands
// 0) under the current or average strategies, in double precision, and their
// range-weighted sums (the subgame value for that player).
int pr_batch_root_values(void *batch, int player, int use_average, double *values, double *sums) {
    Batch *b = (Batch *)batch;
    if (!b || (player != 0 && player != 1) || (use_average && !b->avg_on)) return 2;
    cudaError_t e;
    if (!b->d_root && (e = cudaMalloc(&b->d_root, sizeof(double) * kBRow * b->count)) != cudaSuccess)
        return bfail("root value allocation", e);
    e = cudaMemsetAsync(b->d_head, 0, sizeof(int) * 4 * kClasses, b->stream);
    if (e != cudaSuccess) return bfail("queue reset", e);
    if (int st = b->pass(kBModeEval, player, 1, use_average, b->d_root, b->d_sum, 3)) return st;
    if (values) {
        if (int st = ensure_hands_buffer(b)) return st;
        if (int st = to_hands(b, b->d_root, 1, 1.0, nullptr, b->d_hands)) return st;
        e = cudaMemcpyAsync(values, b->d_hands, sizeof(double) * 1326 * b->count, cudaMemcpyDeviceToHost, b->stream);
    }
    if (e == cudaSuccess && sums)
        e = cudaMemcpyAsync(sums, b->d_sum, sizeof(double) * b->count, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? 0 : bfail("evaluation", e);
}

// CFR iterations like pr_batch_iterate for callers that may not allocate once their solve
// loop runs: a process whose GPU memory belongs to its own caching allocator after start-up,
// or a loop on a shared GPU where a cudaMalloc / cudaFree (which synchronise the device) or
// building a CUDA graph (pr_batch_iterate does that on its first call) would stall other
// work. The passes are launched directly, and the work queue (heads and order) lives in the
// library's fixed device array instead of the batch's buffers.
int pr_batch_iterate_noalloc(void *batch, int iterations) {
    Batch *b = (Batch *)batch;
    if (!b || iterations < 0) return 2;
    if (b->count > kNoAllocMaxSubgames) {
        fprintf(stderr, "pokerrust_b200: pr_batch_iterate_noalloc: %d subgames exceed the limit of %d\n", b->count,
                kNoAllocMaxSubgames);
        return 2;
    }
    int *scratch = noalloc_scratch();
    if (!scratch) return 1;
    int *heads = scratch, *order = scratch + kNoAllocHeads;
    std::vector<int> host_order;
    b->build_order(host_order);
    cudaError_t e = cudaMemcpyAsync(order, host_order.data(), sizeof(int) * b->count, cudaMemcpyHostToDevice,
                                    b->stream);
    if (e != cudaSuccess) return bfail("queue upload", e);
    // the same iteration as pr_batch_iterate (launch configurations, average weights and the
    // linear-average weight step), with the queue in the fixed array; the heads start at zero
    // in every iteration
    for (int it = 0; it < iterations; it++)
        if (int st = b->iteration(order, heads)) return st;
    e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? 0 : bfail("iteration", e);
}

// Subgame value V = r0^T U(sigma) r1 = sum_h r0(h) cfv0(h): player 0's expected chips times
// the joint range mass, under the current or average strategies (double precision).
int pr_batch_value(void *batch, int use_average, double *V) {
    prb::TraceRange trace("batch value");
    Batch *b = (Batch *)batch;
    if (!b || !V || (use_average && !b->avg_on)) return 2;
    cudaError_t e = cudaMemsetAsync(b->d_head, 0, sizeof(int) * 4 * kClasses, b->stream);
    if (e != cudaSuccess) return bfail("queue reset", e);
    if (int st = b->pass(kBModeEval, 0, 1, use_average, nullptr, b->d_sum, 0)) return st;
    e = cudaMemcpyAsync(V, b->d_sum, sizeof(double) * b->count, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? 0 : bfail("value", e);
}

// Adjoint of pr_batch_value: dV/dr0 = cfv0 and dV/dr1 = -cfv1 per colex hand ([count][1326]),
// and dV/dsigma(a, h) = r0(h) cfv0(child a, h) for the root's actions (player 0 acts at the
// root; [count][8][1326], rows past the root's action count are zero). Two evaluation
// passes; reach vectors are recomputed from the strategies, not stored per node.
int pr_batch_value_grad(void *batch, int use_average, double *d_r0, double *d_r1, double *d_sigma) {
    prb::TraceRange trace("batch value gradient");
    Batch *b = (Batch *)batch;
    if (!b || (use_average && !b->avg_on)) return 2;
    if (int st = ensure_hands_buffer(b)) return st;
    const size_t n = (size_t)1326 * b->count;
    double *h0 = b->d_hands, *h1 = h0 + n, *hs = h1 + n;
    if (int st = value_grad_device(b, use_average, d_r0 ? h0 : nullptr, d_r1 ? h1 : nullptr, d_sigma ? hs : nullptr))
        return st;
    // device -> pinned host in one copy, then pinned -> the caller's arrays on host threads
    // (pageable destinations would otherwise be copied through the driver's small staging)
    cudaError_t e = cudaSuccess;
    if (!b->h_pinned) e = cudaHostAlloc(&b->h_pinned, sizeof(double) * 10 * n, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        b->h_pinned = nullptr;
        return bfail("pinned staging allocation", e);
    }
    e = cudaMemcpyAsync(b->h_pinned, b->d_hands, sizeof(double) * 10 * n, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail("adjoint copy", e);
    struct Part { double *dst; const double *src; size_t n; };
    std::vector<Part> parts;
    if (d_r0) parts.push_back({d_r0, b->h_pinned, n});
    if (d_r1) parts.push_back({d_r1, b->h_pinned + n, n});
    if (d_sigma) parts.push_back({d_sigma, b->h_pinned + 2 * n, 8 * n});
    size_t total = 0;
    for (auto &q : parts) total += q.n;
    const int threads = (int)std::min<size_t>(16, std::max<size_t>(1, std::min<unsigned>(std::thread::hardware_concurrency(), total / (1u << 18))));
    auto work = [&](int t) {
        // thread t copies its share [total * t / threads, total * (t + 1) / threads) of the parts
        const size_t lo = total * t / threads, hi = total * (t + 1) / threads;
        size_t at = 0;
        for (auto &q : parts) {
            const size_t a = std::max(lo, at), z = std::min(hi, at + q.n);
            if (a < z) memcpy(q.dst + (a - at), q.src + (a - at), sizeof(double) * (z - a));
            at += q.n;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; t++) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    return e == cudaSuccess ? 0 : bfail("adjoint copy", e);
}

// The same adjoint with device outputs (device pointers, same layouts), for callers that use
// the gradients on the GPU; synchronous.
int pr_batch_value_grad_device(void *batch, int use_average, double *d_r0, double *d_r1, double *d_sigma) {
    Batch *b = (Batch *)batch;
    if (!b || (use_average && !b->avg_on)) return 2;
    return value_grad_device(b, use_average, d_r0, d_r1, d_sigma);
}

// Replaces the ranges of subgame s ([2][1326] floats, colex order).
int pr_batch_set_ranges(void *batch, int s, const float *r) {
    Batch *b = (Batch *)batch;
    if (!b || s < 0 || s >= b->count || !r) return 2;
    // finite weights only; negative ones are allowed here: the subgame value and its adjoint
    // are bilinear in the ranges, and central differences step below zero
    if (!valid_weights(r, 2 * 1326, false)) return bfail("pr_batch_set_ranges: a range holds a NaN or an infinity");
    std::vector<float> rows(2 * kBRow, 0.0f);
    const uint16_t *hand = b->hand.data() + (size_t)s * kBRow;
    for (int pl = 0; pl < 2; pl++)
        for (int p = 0; p < kBLive; p++) rows[pl * kBRow + p] = r[pl * 1326 + hand[p]];
    cudaStreamSynchronize(b->stream);
    cudaError_t e = cudaMemcpy(b->d_ranges + (size_t)s * 2 * kBRow, rows.data(), sizeof(float) * 2 * kBRow,
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return bfail("range upload", e);
    // joint mass of clash-free pairs
    const float *r0 = r, *r1 = r + 1326;
    const uint64_t board = b->subs[s].board;
    double tot = 0, card[52] = {0};
    for (int h = 0; h < 1326; h++) {
        int c1, c2;
        hand_cards(h, &c1, &c2);
        if (((1ull << c1) | (1ull << c2)) & board) continue;
        tot += r1[h];
        card[c1] += r1[h];
        card[c2] += r1[h];
    }
    double j = 0;
    for (int h = 0; h < 1326; h++) {
        int c1, c2;
        hand_cards(h, &c1, &c2);
        if (((1ull << c1) | (1ull << c2)) & board) continue;
        j += (double)r0[h] * (tot - card[c1] - card[c2] + r1[h]);
    }
    b->joint[s] = j;
    return 0;
}

namespace {
// device rows [edge][kBRow] (position order) <-> host rows [edge][1326] (colex order)
int rows_io(Batch *b, float *dev, int s, float *host, bool to_host) {
    const BSub &d = b->subs[s];
    std::vector<float> buf((size_t)d.num_edges * kBRow);
    float *src = dev + (size_t)d.edge_off * kBRow;
    cudaError_t e = cudaSuccess;
    const uint16_t *hand = b->hand.data() + (size_t)s * kBRow;
    if (to_host) {
        e = cudaMemcpy(buf.data(), src, sizeof(float) * buf.size(), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return bfail("row download", e);
        for (int k = 0; k < d.num_edges; k++) {
            float *o = host + (size_t)k * 1326;
            for (int h = 0; h < 1326; h++) o[h] = 0.0f;
            for (int p = 0; p < kBLive; p++) o[hand[p]] = buf[(size_t)k * kBRow + p];
        }
    } else {
        for (int k = 0; k < d.num_edges; k++)
            for (int p = 0; p < kBRow; p++)
                buf[(size_t)k * kBRow + p] = p < kBLive ? host[(size_t)k * 1326 + hand[p]] : 0.0f;
        e = cudaMemcpy(src, buf.data(), sizeof(float) * buf.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return bfail("row upload", e);
    }
    return 0;
}
}  // namespace

int pr_batch_get_regrets(void *batch, int s, float *out) {
    Batch *b = (Batch *)batch;
    if (!b || s < 0 || s >= b->count || !out) return 2;
    cudaStreamSynchronize(b->stream);
    return rows_io(b, b->d_regrets, s, out, true);
}

int pr_batch_set_regrets(void *batch, int s, const float *in) {
    Batch *b = (Batch *)batch;
    if (!b || s < 0 || s >= b->count || !in) return 2;
    cudaStreamSynchronize(b->stream);
    return rows_io(b, b->d_regrets, s, const_cast<float *>(in), false);
}

int pr_batch_get_average(void *batch, int s, float *out) {
    Batch *b = (Batch *)batch;
    if (!b || !b->avg_on || s < 0 || s >= b->count || !out) return 2;
    cudaStreamSynchronize(b->stream);
    return rows_io(b, b->d_avg, s, out, true);
}

int pr_batch_set_average(void *batch, int s, const float *in) {
    Batch *b = (Batch *)batch;
    if (!b || !b->avg_on || s < 0 || s >= b->count || !in) return 2;
    cudaStreamSynchronize(b->stream);
    return rows_io(b, b->d_avg, s, const_cast<float *>(in), false);
}

// All subgames' regret (which 0) or average-sum (which 1) rows at once: out[sum E_s][1326]
// floats, colex order, subgames in batch order and each subgame's edges in its tree order.
// Converted on the device in chunks of subgames and copied out one chunk at a time.
int pr_batch_get_all(void *batch, int which, float *out) {
    Batch *b = (Batch *)batch;
    if (!b || !out || (which != 0 && which != 1) || (which == 1 && !b->avg_on)) return 2;
    const float *src = which ? b->d_avg : b->d_regrets;
    constexpr int kChunkRows = 8192;  // 43 MB of staging; a subgame has at most kBMaxNodes edges
    float *stage = nullptr;
    cudaError_t e = cudaMalloc(&stage, sizeof(float) * 1326 * kChunkRows);
    if (e != cudaSuccess) return bfail("row staging allocation", e);
    int s = 0;
    while (s < b->count && e == cudaSuccess) {
        const int base = b->subs[s].edge_off;
        int t = s;
        while (t < b->count && b->subs[t].edge_off + b->subs[t].num_edges - base <= kChunkRows) t++;
        rows_to_hands_kernel<<<t - s, 256, 0, b->stream>>>(src, b->d_subs, b->d_packs, s, base, stage);
        e = cudaGetLastError();
        const size_t rows = (size_t)(t < b->count ? b->subs[t].edge_off : b->total_edges) - base;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out + (size_t)base * 1326, stage, sizeof(float) * 1326 * rows, cudaMemcpyDeviceToHost,
                                b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        s = t;
    }
    cudaFree(stage);
    return e == cudaSuccess ? 0 : bfail("row download", e);
}

// Configuration of class c: hands per thread, resident CTAs per SM, queue order.
int pr_batch_config(void *batch, int c, int *K, int *per_sm, int *order, int *count) {
    Batch *b = (Batch *)batch;
    if (!b || c < 0 || c >= kClasses) return 2;
    if (K) *K = b->cls[c].K;
    if (per_sm) *per_sm = b->cls[c].per_sm;
    if (order) *order = b->cls[c].order;
    if (count) *count = b->cls[c].count;
    return 0;
}

int pr_batch_set_config(void *batch, int c, int K, int per_sm, int order) {
    Batch *b = (Batch *)batch;
    if (!b || c < 0 || c >= kClasses || (K != 2 && K != 3 && K != 4) || per_sm < 1 || per_sm > 4 ||
        (order != 0 && order != 1))
        return 2;
    const int fits = K == 4 && per_sm >= 3 ? batch_dense_ctas_per_sm(b->avg_on) : batch_ctas_per_sm(kBModeCFR, K, 0, b->avg_on);
    if (per_sm > fits) return 2;
    b->cls[c].K = K;
    b->cls[c].per_sm = per_sm;
    b->cls[c].order = order;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return b->upload_order();
}

// Autotuner: for each shape class, times one CFR pass of every configuration (hands per
// thread 2/3/4, resident CTAs per SM up to what fits, queue order) over the class's share of
// the first (up to) 8192 subgames and keeps the fastest; their regrets and sums are restored
// afterwards, so tuning does not change the solve. Writes the chosen class-0 / class-1 times
// (ms per pass over those subgames).
int pr_batch_tune(void *batch, double *ms_out) {
    Batch *b = (Batch *)batch;
    if (!b) return 2;
    // Passes are timed on the first nt subgames only (at most kTuneSubgames): their rows are
    // contiguous, so only they are saved and restored, and a batch of any size can be tuned
    // beside its own state.
    constexpr int kTuneSubgames = 8192;
    const int nt = std::min(b->count, kTuneSubgames);
    const int rows_nt = nt < b->count ? b->subs[nt].edge_off : b->total_edges;
    const size_t rows = (size_t)rows_nt * kBRow * sizeof(float);
    float *save_r = nullptr, *save_a = nullptr;
    int *tune_order = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&save_r, rows)) != cudaSuccess) return bfail("tuning allocation", e);
    if ((b->avg_on && (e = cudaMalloc(&save_a, rows)) != cudaSuccess) ||
        (e = cudaMalloc(&tune_order, sizeof(int) * nt)) != cudaSuccess) {
        cudaFree(save_r);
        cudaFree(save_a);
        return bfail("tuning allocation", e);
    }
    // the tuning queue: the first nt subgames in the class's queue order; class c starts at
    // sub_first[c] and holds sub_count[c] of them
    int sub_first[kClasses], sub_count[kClasses];
    auto upload_tune_order = [&]() -> int {
        std::vector<int> full, sub;
        b->build_order(full);
        for (int c = 0, at = 0; c < kClasses; c++) {
            sub_first[c] = (int)sub.size();
            for (int i = 0; i < b->cls[c].count; i++)
                if (full[at + i] < nt) sub.push_back(full[at + i]);
            sub_count[c] = (int)sub.size() - sub_first[c];
            at += b->cls[c].count;
        }
        cudaError_t x = cudaMemcpy(tune_order, sub.data(), sizeof(int) * sub.size(), cudaMemcpyHostToDevice);
        return x == cudaSuccess ? 0 : bfail("tuning queue upload", x);
    };
    cudaMemcpyAsync(save_r, b->d_regrets, rows, cudaMemcpyDeviceToDevice, b->stream);
    if (save_a) cudaMemcpyAsync(save_a, b->d_avg, rows, cudaMemcpyDeviceToDevice, b->stream);
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    int status = 0;
    for (int c = 0; c < kClasses && !status; c++) {
        if (!b->cls[c].count) {
            if (ms_out) ms_out[c] = 0.0;
            continue;
        }
        ClassCfg keep[kClasses];
        for (int i = 0; i < kClasses; i++) keep[i] = b->cls[i];
        float best = 1e30f;
        ClassCfg best_cfg = keep[c];
        for (int K : {2, 3, 4}) {
            const int fits = batch_ctas_per_sm(kBModeCFR, K, 0, b->avg_on);
            // per = 1, 2 where they fit; K = 4 also tries the dense configuration (registers
            // capped for 3 CTAs per SM) where three of its CTAs fit
            std::vector<int> pers;
            for (int per = 1; per <= std::min(fits, 2); per++) pers.push_back(per);
            if (K == 4 && batch_dense_ctas_per_sm(b->avg_on) >= 3) pers.push_back(3);
            for (int per : pers) {
                for (int ord = 0; ord < 2; ord++) {
                    for (int i = 0; i < kClasses; i++) b->cls[i] = keep[i];
                    b->cls[c].K = K;
                    b->cls[c].per_sm = per;
                    b->cls[c].order = ord;
                    if ((status = upload_tune_order())) break;
                    // time this class alone, on its share of the tuning queue
                    for (int i = 0; i < kClasses; i++) {
                        b->cls[i].first = sub_first[i];
                        b->cls[i].count = i == c ? sub_count[i] : 0;
                    }
                    if (!b->cls[c].count) break;
                    float ms = 0;
                    for (int rep = 0; rep < 3 && !status; rep++) {
                        cudaMemsetAsync(b->d_head, 0, sizeof(int) * 4 * kClasses, b->stream);
                        cudaEventRecord(t0, b->stream);
                        status = b->pass(kBModeCFR, rep & 1, 0, 0, nullptr, nullptr, 0, nullptr, nullptr, tune_order);
                        cudaEventRecord(t1, b->stream);
                        cudaEventSynchronize(t1);
                        float t = 0;
                        cudaEventElapsedTime(&t, t0, t1);
                        if (rep > 0) ms += t;  // first run warms up
                    }
                    if (status) break;
                    if (ms < best) {
                        best = ms;
                        best_cfg = b->cls[c];
                    }
                }
                if (status) break;
            }
            if (status) break;
        }
        for (int i = 0; i < kClasses; i++) b->cls[i] = keep[i];
        b->cls[c].K = best_cfg.K;
        b->cls[c].per_sm = best_cfg.per_sm;
        b->cls[c].order = best_cfg.order;
        if (ms_out) ms_out[c] = best < 1e29f ? best / 2.0 : 0.0;
    }
    if (!status) status = b->upload_order();
    cudaMemcpyAsync(b->d_regrets, save_r, rows, cudaMemcpyDeviceToDevice, b->stream);
    if (save_a) cudaMemcpyAsync(b->d_avg, save_a, rows, cudaMemcpyDeviceToDevice, b->stream);
    e = cudaStreamSynchronize(b->stream);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(save_r);
    cudaFree(save_a);
    cudaFree(tune_order);
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->tuned = true;
    if (e != cudaSuccess) return bfail("tuning", e);
    return status;
}

// Algorithmic HBM bytes of one CFR iteration (both players): per edge and hand, the
// updater's regret read + write and average read + write, the other player's regret read
// (20 B with averages, 12 B without), plus ranges in and the tables read per pass.
double pr_batch_iteration_bytes(void *batch) {
    Batch *b = (Batch *)batch;
    if (!b) return 0;
    const double per = b->avg_on ? 20.0 : 12.0;
    return (double)b->total_edges * kBLive * per +
           2.0 * b->count * (2.0 * kBRow * 4 + (double)sizeof(BPack) + 64.0);
}

}  // extern "C"
