// C ABI of the solver: the reference's seven symbols (src/cuda/interface.cu:9-122) and the
// pr_* extensions declared in include/pokerrust_b200.h.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/pokerrust_b200.h"
#include "device_common.cuh"
#include "gen_tables.h"
#include "layout.h"
#include "pack_boards.h"
#include "river_cfr.h"
#include "river_tree.h"
#include "trace.h"

namespace prb {
namespace {

enum Status {
    kOk = 0,
    kErrCuda = 1,
    kErrArg = 2,
    kErrTables = 3,
    kErrTree = 4,
    kErrAlloc = 5,
};

std::atomic<int> g_status{0};
std::atomic<int> g_cuda_error{0};

int fail(int status, const char *what, cudaError_t e = cudaSuccess) {
    g_status.store(status);
    if (e != cudaSuccess) {
        g_cuda_error.store((int)e);
        fprintf(stderr, "pokerrust_b200: %s: %s\n", what, cudaGetErrorString(e));
    } else {
        fprintf(stderr, "pokerrust_b200: %s\n", what);
    }
    fflush(stderr);
    return status;
}

// The river tree rebuilt from the reference's builder rules (src/cuda/builder.cu:8-121):
// checks that the compiled tables of river_tree.h describe the same tree.
struct HostState {
    int terminal, action, actor, parent, nchild, child[3], edge[3];
    float sb, bb;
    bool dealt;
};

bool river_tree_matches() {
    enum { Fold, Check, Call, Raise, DealRiver };
    HostState st[kStates];
    int nst = 1, ned = 0;
    st[0] = HostState{kRiver, Call, 0, -1, 0, {-1, -1, -1}, {-1, -1, -1}, 0.f, 0.f, false};
    struct Rec {
        static void build(HostState *st, int *nst, int *ned, int s, int raises) {
            int acts[3], na = 0;
            switch (st[s].action) {
                case Check: acts[0] = Call; acts[1] = Raise; na = 2; break;
                case Call: if (!st[s].dealt) { acts[0] = DealRiver; na = 1; } break;
                case Raise:
                    acts[0] = Fold; acts[1] = Call; na = 2;
                    if (raises < 4) acts[na++] = Raise;
                    break;
                case DealRiver: acts[0] = Check; acts[1] = Raise; na = 2; break;
                default: break;
            }
            for (int i = 0; i < na; i++) {
                if (*nst >= kStates) return;
                HostState t = st[s];
                const int a = acts[i];
                t.actor = st[s].actor == 0 ? 1 : 0;
                t.action = a;
                t.nchild = 0;
                t.parent = s;
                const float other = st[s].actor == 0 ? st[s].bb : st[s].sb;
                switch (a) {
                    case Fold: t.terminal = st[s].actor == 0 ? kBBWins : kSBWins; break;
                    case Check: t.terminal = kNonTerminal; break;
                    case Call: t.terminal = st[s].dealt ? kShowdown : kRiver; t.sb = t.bb = other; break;
                    case Raise:
                        t.terminal = kNonTerminal;
                        if (st[s].actor == 0) t.sb = st[s].bb + 2.0f; else t.bb = st[s].sb + 2.0f;
                        break;
                    case DealRiver: t.actor = 0; t.terminal = kNonTerminal; t.dealt = true; break;
                }
                const int c = (*nst)++;
                st[c] = t;
                build(st, nst, ned, c, a == Raise ? raises + 1 : 0);
                const int k = st[s].nchild++;
                st[s].child[k] = c;
                st[s].edge[k] = st[s].terminal == kNonTerminal ? (*ned)++ : -1;
            }
        }
    };
    Rec::build(st, &nst, &ned, 0, 0);
    if (nst != kStates || ned != kEdges) return false;
    for (int s = 0; s < kStates; s++) {
        if (st[s].terminal != kTerm(s) || st[s].parent != kParent(s) ||
            st[s].nchild != kNChild(s) || st[s].sb != kSbOff(s) || st[s].bb != kBbOff(s))
            return false;
        if (st[s].terminal == kNonTerminal && st[s].actor != kActor(s)) return false;
        for (int k = 0; k < st[s].nchild; k++)
            if (st[s].child[k] != kChild(s, k) || st[s].edge[k] != kEdge(s, k)) return false;
    }
    return true;
}

constexpr int kPipeChunks = 4;  // chunks of a staged pass (copies overlap the kernel)

struct Builder {
    std::vector<SubgameDesc> desc;
    int capacity = 0;
    float *comm = nullptr;  // pinned staging, capacity rows of kRangeStride
    // device state
    int dev_count = 0, dev_capacity = 0;
    SubgameDesc *d_desc = nullptr;
    float *d_regrets = nullptr;
    float *d_ranges = nullptr;
    float *d_results = nullptr;
    // average strategies (pr_enable_average): own-range staging and the sums
    bool avg_on = false;
    float *comm_own = nullptr;      // pinned, capacity rows
    float *d_own = nullptr;
    float *d_avg = nullptr;
    int avg_capacity = 0;
    double *d_ranges64 = nullptr;   // double-precision best response (lazily allocated)
    double *d_results64 = nullptr;
    int cap64 = 0;
    cudaStream_t stream = nullptr;
    // staged passes are pipelined: ranges of chunk k+1 go up (copy_in) and results of chunk
    // k-1 come down (copy_out) while the kernel runs chunk k on `stream`
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    cudaEvent_t ev_in[kPipeChunks] = {}, ev_done[kPipeChunks] = {};
    unsigned long long checked_flop = 0;  // boards validated against this flop
    int checked_count = -1;
};

struct EvalTables {
    unsigned long long flop = 0;
    BoardPack *packs = nullptr;
    uint16_t *d_eval = nullptr;
    uint16_t *d_coll = nullptr;
    uint16_t *d_abstr = nullptr;
    int *d_err = nullptr;  // [0] error bits, [1] max tie groups, [2] max card-list groups
    int status = 0;
    int max_groups = 0, max_card_groups = 0;
};

constexpr size_t kEvalBytes = (size_t)kSlotsPerBoard * (1326 + 512) * sizeof(uint16_t);
constexpr size_t kCollBytes = (size_t)kSlotsPerBoard * 52 * 51 * sizeof(uint16_t);
constexpr size_t kAbstrBytes = (size_t)kSlotsPerBoard * kHands * sizeof(uint16_t);

// One table set kept for reuse: the reference transfers and frees the tables on every
// iteration (game.rs:71,180), so allocations are recycled instead of repeated.
std::mutex g_cache_mu;
EvalTables *g_cache = nullptr;

bool grow_staging(Builder *b, int need) {
    if (need <= b->capacity) return true;
    int cap = b->capacity ? b->capacity : 1024;
    while (cap < need) cap *= 2;
    float *fresh = nullptr;
    cudaError_t e = cudaHostAlloc((void **)&fresh, (size_t)cap * kRangeStride * sizeof(float),
                                  cudaHostAllocPortable);
    if (e != cudaSuccess) {
        fail(kErrAlloc, "pinned staging allocation", e);
        return false;
    }
    memset(fresh, 0, (size_t)cap * kRangeStride * sizeof(float));
    if (b->comm) {
        memcpy(fresh, b->comm, (size_t)b->capacity * kRangeStride * sizeof(float));
        cudaFreeHost(b->comm);
    }
    b->comm = fresh;
    if (b->avg_on) {
        float *own = nullptr;
        e = cudaHostAlloc((void **)&own, (size_t)cap * kRangeStride * sizeof(float), cudaHostAllocPortable);
        if (e != cudaSuccess) {
            fail(kErrAlloc, "pinned staging allocation", e);
            return false;
        }
        memset(own, 0, (size_t)cap * kRangeStride * sizeof(float));
        if (b->comm_own) {
            memcpy(own, b->comm_own, (size_t)b->capacity * kRangeStride * sizeof(float));
            cudaFreeHost(b->comm_own);
        }
        b->comm_own = own;
    }
    b->capacity = cap;
    return true;
}

// Device arrays of the average-strategy sums, grown with the subgames (new rows zero).
int sync_average(Builder *b) {
    if (b->avg_capacity >= b->dev_capacity) return kOk;
    cudaError_t e;
    float *own = nullptr, *avg = nullptr;
    const size_t rows = (size_t)b->dev_capacity * kRangeStride * sizeof(float);
    const size_t sums = (size_t)b->dev_capacity * kEdges * kBuckets * sizeof(float);
    if ((e = cudaMalloc(&own, rows)) != cudaSuccess || (e = cudaMalloc(&avg, sums)) != cudaSuccess) {
        cudaFree(own);
        return fail(kErrAlloc, "average-strategy allocation", e);
    }
    cudaMemsetAsync(avg, 0, sums, b->stream);
    if (b->d_avg)
        cudaMemcpyAsync(avg, b->d_avg, (size_t)b->avg_capacity * kEdges * kBuckets * sizeof(float),
                        cudaMemcpyDeviceToDevice, b->stream);
    e = cudaStreamSynchronize(b->stream);
    cudaFree(b->d_own);
    cudaFree(b->d_avg);
    b->d_own = own;
    b->d_avg = avg;
    b->avg_capacity = b->dev_capacity;
    return e == cudaSuccess ? kOk : fail(kErrCuda, "average-strategy allocation", e);
}

// Brings the device arrays up to the host's subgame count; new regrets start at zero
// (interface.cu:78 zeroes them once at start-up).
int sync_device(Builder *b) {
    const int n = (int)b->desc.size();
    cudaError_t e;
    if (!b->stream) {
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(kErrCuda, "stream creation", e);
    }
    if (n > b->dev_capacity) {
        int cap = b->dev_capacity ? b->dev_capacity : 1024;
        while (cap < n) cap *= 2;
        SubgameDesc *nd = nullptr;
        float *nr = nullptr, *nrg = nullptr, *nres = nullptr;
        const size_t rows = (size_t)cap * kRangeStride * sizeof(float);
        const size_t regb = (size_t)cap * kEdges * kBuckets * sizeof(float);
        if ((e = cudaMalloc(&nd, (size_t)cap * sizeof(SubgameDesc))) != cudaSuccess ||
            (e = cudaMalloc(&nr, rows)) != cudaSuccess || (e = cudaMalloc(&nres, rows)) != cudaSuccess ||
            (e = cudaMalloc(&nrg, regb)) != cudaSuccess) {
            cudaFree(nd);
            cudaFree(nr);
            cudaFree(nres);
            cudaFree(nrg);
            return fail(kErrAlloc, "device allocation", e);
        }
        cudaMemsetAsync(nrg, 0, regb, b->stream);
        if (b->d_regrets)
            cudaMemcpyAsync(nrg, b->d_regrets, (size_t)b->dev_count * kEdges * kBuckets * sizeof(float),
                            cudaMemcpyDeviceToDevice, b->stream);
        cudaStreamSynchronize(b->stream);
        cudaFree(b->d_desc);
        cudaFree(b->d_ranges);
        cudaFree(b->d_results);
        cudaFree(b->d_regrets);
        b->d_desc = nd;
        b->d_ranges = nr;
        b->d_results = nres;
        b->d_regrets = nrg;
        b->dev_capacity = cap;
    }
    if (n != b->dev_count) {
        e = cudaMemcpyAsync(b->d_desc, b->desc.data(), (size_t)n * sizeof(SubgameDesc),
                            cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) return fail(kErrCuda, "descriptor upload", e);
        b->dev_count = n;
    }
    return kOk;
}

int evaluate_impl(Builder *b, EvalTables *t, int player, int exploit, const float *d_in, float *d_out,
                  cudaStream_t stream, bool staged, const float *d_own = nullptr) {
    prb::TraceRange trace(exploit ? "river pass (best response)" : "river pass (CFR)");
    if (!b || !t) return fail(kErrArg, "evaluate: null builder or tables");
    if (t->status) return fail(kErrTables, "evaluate: tables failed validation on upload");
    if (player != 0 && player != 1) return fail(kErrArg, "evaluate: updating_player must be 0 or 1");
    if (b->checked_flop != t->flop || b->checked_count != (int)b->desc.size()) {
        // every river root must extend the tables' flop by one turn card, so that each
        // {turn, river} slot the kernel reads is one the re-pack filled
        for (const SubgameDesc &d : b->desc)
            if ((d.board4 & t->flop) != t->flop || __builtin_popcountll(d.board4) != 4)
                return fail(kErrArg, "evaluate: a river root's board does not contain the flop");
        b->checked_flop = t->flop;
        b->checked_count = (int)b->desc.size();
    }
    int st = sync_device(b);
    if (st) return st;
    const int n = b->dev_count;
    if (n == 0) return kOk;
    cudaStream_t s = stream ? stream : b->stream;
    cudaError_t e;
    const bool avg = (staged || d_own) && b->avg_on && !exploit;
    if (avg) {
        if ((st = sync_average(b))) return st;
        if (staged && n < 4 * kPipeChunks * 148) {
            e = cudaMemcpyAsync(b->d_own, b->comm_own, (size_t)n * kRangeStride * sizeof(float),
                                cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) return fail(kErrCuda, "own range upload", e);
        }
    }
    if (staged && n >= 4 * kPipeChunks * 148) {
        // pipelined: copy-in / kernel / copy-out of kPipeChunks chunks on three streams
        if (!b->copy_in) {
            if ((e = cudaStreamCreateWithFlags(&b->copy_in, cudaStreamNonBlocking)) != cudaSuccess ||
                (e = cudaStreamCreateWithFlags(&b->copy_out, cudaStreamNonBlocking)) != cudaSuccess)
                return fail(kErrCuda, "stream creation", e);
            for (int k = 0; k < kPipeChunks; k++)
                if ((e = cudaEventCreateWithFlags(&b->ev_in[k], cudaEventDisableTiming)) != cudaSuccess ||
                    (e = cudaEventCreateWithFlags(&b->ev_done[k], cudaEventDisableTiming)) != cudaSuccess)
                    return fail(kErrCuda, "event creation", e);
        }
        // the copies may only start once earlier work on the pass stream is done
        if ((e = cudaEventRecord(b->ev_done[0], s)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(b->copy_in, b->ev_done[0], 0)) != cudaSuccess)
            return fail(kErrCuda, "pass ordering", e);
        for (int k = 0; k < kPipeChunks; k++) {
            const int lo = (int)((long long)n * k / kPipeChunks), hi = (int)((long long)n * (k + 1) / kPipeChunks);
            const size_t row0 = (size_t)lo * kRangeStride, rows = (size_t)(hi - lo) * kRangeStride;
            e = cudaMemcpyAsync(b->d_ranges + row0, b->comm + row0, rows * sizeof(float), cudaMemcpyHostToDevice,
                                b->copy_in);
            if (e == cudaSuccess && avg)
                e = cudaMemcpyAsync(b->d_own + row0, b->comm_own + row0, rows * sizeof(float), cudaMemcpyHostToDevice,
                                    b->copy_in);
            if (e == cudaSuccess) e = cudaEventRecord(b->ev_in[k], b->copy_in);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->ev_in[k], 0);
            if (e != cudaSuccess) return fail(kErrCuda, "range upload", e);
            e = launch_river(exploit ? kModeBR : kModeCFR, b->d_desc + lo, hi - lo, b->d_ranges + row0,
                             b->d_results + row0, b->d_regrets + (size_t)lo * kEdges * kBuckets, t->packs, t->flop,
                             player, t->max_groups, t->max_card_groups, avg ? b->d_own + row0 : nullptr,
                             avg ? b->d_avg + (size_t)lo * kEdges * kBuckets : nullptr, s);
            if (e != cudaSuccess) return fail(kErrCuda, "river kernel launch", e);
            if ((e = cudaEventRecord(b->ev_done[k], s)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(b->copy_out, b->ev_done[k], 0)) != cudaSuccess)
                return fail(kErrCuda, "pass ordering", e);
            e = cudaMemcpyAsync(b->comm + row0, b->d_results + row0, rows * sizeof(float), cudaMemcpyDeviceToHost,
                                b->copy_out);
            if (e != cudaSuccess) return fail(kErrCuda, "result download", e);
        }
        e = cudaStreamSynchronize(b->copy_out);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return fail(kErrCuda, "river pass", e);
        return kOk;
    }
    if (staged) {
        e = cudaMemcpyAsync(b->d_ranges, b->comm, (size_t)n * kRangeStride * sizeof(float),
                            cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return fail(kErrCuda, "range upload", e);
        d_in = b->d_ranges;
        d_out = b->d_results;
    }
    e = launch_river(exploit ? kModeBR : kModeCFR, b->d_desc, n, d_in, d_out, b->d_regrets, t->packs,
                     t->flop, player, t->max_groups, t->max_card_groups, avg ? (staged ? b->d_own : d_own) : nullptr,
                     avg ? b->d_avg : nullptr, s);
    if (e != cudaSuccess) return fail(kErrCuda, "river kernel launch", e);
    if (staged) {
        e = cudaMemcpyAsync(b->comm, b->d_results, (size_t)n * kRangeStride * sizeof(float),
                            cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) return fail(kErrCuda, "result download", e);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return fail(kErrCuda, "river pass", e);
    }
    return kOk;
}

bool card_order_ok(const uint64_t *card_order, const uint16_t *card_indexes) {
    // The kernels index hands by the colex order of their two cards (evaluator.rs:29-40)
    // and the per-card lists by card_indexes (evaluator.rs:159-172).
    int n = 0, fill[52] = {0};
    for (int hi = 1; hi < 52; hi++)
        for (int lo = 0; lo < hi; lo++, n++)
            if (card_order[n] != ((1ull << lo) | (1ull << hi))) return false;
    for (int i = 0; i < kHands; i++) {
        const int lo = ctz64(card_order[i]);
        const int hi = ctz64(card_order[i] & (card_order[i] - 1));
        if (card_indexes[lo * 51 + fill[lo]++] != i) return false;
        if (card_indexes[hi * 51 + fill[hi]++] != i) return false;
    }
    return true;
}

// A table set with device buffers, recycled from the last free_eval_cuda when possible.
EvalTables *acquire_tables() {
    EvalTables *t = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        t = g_cache;
        g_cache = nullptr;
    }
    if (t) {
        t->status = 0;
        return t;
    }
    t = new EvalTables();
    cudaError_t e;
    if ((e = cudaMalloc(&t->packs, (size_t)kSlotsPerBoard * sizeof(BoardPack))) != cudaSuccess ||
        (e = cudaMalloc(&t->d_eval, kEvalBytes)) != cudaSuccess ||
        (e = cudaMalloc(&t->d_coll, kCollBytes)) != cudaSuccess ||
        (e = cudaMalloc(&t->d_abstr, kAbstrBytes)) != cudaSuccess ||
        (e = cudaMalloc(&t->d_err, 4 * sizeof(int))) != cudaSuccess) {
        fail(kErrAlloc, "table allocation", e);
        t->status = -1;
        return t;
    }
    // slots the re-pack never writes (pairs that overlap the flop) stay all-zero
    if ((e = cudaMemset(t->packs, 0, (size_t)kSlotsPerBoard * sizeof(BoardPack))) != cudaSuccess ||
        (e = cudaMemset(t->d_coll, 0, kCollBytes)) != cudaSuccess) {
        fail(kErrCuda, "table initialisation", e);
        t->status = -1;
    }
    return t;
}

// Validates the reference-layout tables in d_eval / d_abstr and re-packs them into BoardPack.
void repack_tables(EvalTables *t) {
    cudaError_t e;
    if ((e = cudaMemset(t->d_err, 0, 4 * sizeof(int))) != cudaSuccess) {
        fail(kErrCuda, "table re-pack", e);
        t->status = -1;
        return;
    }
    launch_pack_boards(t->flop, t->d_eval, t->d_abstr, t->packs, t->d_err, 0);
    int err[4] = {0, 0, 0, 0};
    if ((e = cudaMemcpy(err, t->d_err, 4 * sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) {
        fail(kErrCuda, "table re-pack", e);
        t->status = -1;
        return;
    }
    if (err[0]) {
        fail(kErrTables, "hand-rank tables are not a consistent rank order");
        t->status = err[0];
        return;
    }
    t->max_groups = err[1];
    t->max_card_groups = err[2];
    if (river_smem_bytes(kModeCFR, 0, t->max_groups, t->max_card_groups) > 227 * 1024 ||
        river_smem_bytes(kModeBR, 1, t->max_groups, t->max_card_groups) > 227 * 1024) {
        fail(kErrTables, "a board of this flop has more tie groups than shared memory holds");
        t->status = 128;
    }
}

}  // namespace
}  // namespace prb

using namespace prb;

extern "C" {

void *init_builder(void) {
    if (!river_tree_matches()) {
        fail(kErrTree, "river tree tables disagree with the builder rules");
        return nullptr;
    }
    Builder *b = new Builder();
    if (!grow_staging(b, 1)) {
        delete b;
        return nullptr;
    }
    return b;
}

void upload_c(void *builder, int index, const float *v) {
    Builder *b = (Builder *)builder;
    if (!b || index < 0 || index >= (int)b->desc.size() || !v) {
        fail(kErrArg, "upload_c: bad builder or index");
        return;
    }
    // a range is a vector of finite, non-negative weights: refuse anything else (the slot
    // keeps its previous contents); v - v is NaN exactly for NaN and infinities
    float bad = 0.0f;
    for (int i = 0; i < kHands; i++) bad += (v[i] - v[i]) + (v[i] < 0.0f ? 1.0f : 0.0f);
    if (bad != 0.0f) {
        fail(kErrArg, "upload_c: a range holds a NaN, an infinity or a negative weight");
        return;
    }
    memcpy(b->comm + (size_t)index * kRangeStride, v, kHands * sizeof(float));
}

void download_c(void *builder, int index, float *v) {
    Builder *b = (Builder *)builder;
    if (!b || index < 0 || index >= (int)b->desc.size() || !v) {
        fail(kErrArg, "download_c: bad builder or index");
        return;
    }
    memcpy(v, b->comm + (size_t)index * kRangeStride, kHands * sizeof(float));
}

int build_river_cuda(uint64_t cards, float bet, void *builder) {
    Builder *b = (Builder *)builder;
    if (!b) {
        fail(kErrArg, "build_river_cuda: null builder");
        return -1;
    }
    if (__builtin_popcountll(cards) != 4 || (cards >> 52)) {
        fail(kErrArg, "build_river_cuda: a river root needs a 4-card board");
        return -1;
    }
    const int idx = (int)b->desc.size();
    if (!grow_staging(b, idx + 1)) return -1;
    SubgameDesc d;
    d.board4 = cards;
    d.bet = bet;
    d.pad = 0;
    b->desc.push_back(d);
    return idx;
}

void *transfer_flop_eval_cuda(uint64_t flop, const uint64_t *card_order, const uint16_t *card_indexes,
                              const uint16_t *eval, const uint16_t *coll_vec, const uint16_t *abstractions) {
    // coll_vec is kept for pr_tables_export; the kernels derive the card lists from the
    // sort order instead of reading it
    EvalTables *t = acquire_tables();
    if (t->status) return t;
    cudaError_t e;
    t->flop = flop;
    t->status = 0;
    if (__builtin_popcountll(flop) != 3 || (flop >> 52) || !card_order || !card_indexes || !eval ||
        !abstractions) {
        fail(kErrArg, "transfer_flop_eval_cuda: bad flop or null table");
        t->status = 32;
        return t;
    }
    if (!card_order_ok(card_order, card_indexes)) {
        fail(kErrTables, "transfer_flop_eval_cuda: card_order / card_indexes not in colex order");
        t->status = 64;
        return t;
    }
    if ((e = cudaMemcpy(t->d_eval, eval, kEvalBytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (coll_vec && (e = cudaMemcpy(t->d_coll, coll_vec, kCollBytes, cudaMemcpyHostToDevice)) != cudaSuccess) ||
        (e = cudaMemcpy(t->d_abstr, abstractions, kAbstrBytes, cudaMemcpyHostToDevice)) != cudaSuccess) {
        fail(kErrCuda, "table upload", e);
        t->status = -1;
        return t;
    }
    repack_tables(t);
    return t;
}

void free_eval_cuda(void *eval) {
    EvalTables *t = (EvalTables *)eval;
    if (!t) return;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (!g_cache && t->packs) {
        g_cache = t;
        return;
    }
    cudaFree(t->packs);
    cudaFree(t->d_eval);
    cudaFree(t->d_coll);
    cudaFree(t->d_abstr);
    cudaFree(t->d_err);
    delete t;
}

void evaluate_cuda(void *builder, void *eval, uint16_t updating_player, bool calc_exploit) {
    evaluate_impl((Builder *)builder, (EvalTables *)eval, (int)updating_player, calc_exploit ? 1 : 0,
                  nullptr, nullptr, nullptr, true);
}

int pr_last_error(void) { return g_status.load(); }

void pr_clear_error(void) {
    g_status.store(0);
    g_cuda_error.store(0);
}

const char *pr_error_string(int status) {
    switch (status) {
        case kOk: return "ok";
        case kErrCuda: return cudaGetErrorString((cudaError_t)g_cuda_error.load());
        case kErrArg: return "invalid argument";
        case kErrTables: return "inconsistent hand-rank tables";
        case kErrTree: return "river tree tables disagree with the builder rules";
        case kErrAlloc: return "allocation failed";
        default: return "unknown status";
    }
}

int pr_evaluate(void *builder, void *eval, int updating_player, int calc_exploit) {
    return evaluate_impl((Builder *)builder, (EvalTables *)eval, updating_player, calc_exploit, nullptr,
                         nullptr, nullptr, true);
}

int pr_evaluate_device(void *builder, void *eval, int updating_player, int calc_exploit,
                       const float *d_ranges, float *d_results, void *stream) {
    if (!d_ranges || !d_results) return fail(kErrArg, "pr_evaluate_device: null buffer");
    return evaluate_impl((Builder *)builder, (EvalTables *)eval, updating_player, calc_exploit, d_ranges,
                         d_results, (cudaStream_t)stream, false);
}

int pr_evaluate_device_own(void *builder, void *eval, int updating_player, const float *d_ranges,
                           const float *d_own, float *d_results, void *stream) {
    Builder *b = (Builder *)builder;
    if (!d_ranges || !d_results || !d_own) return fail(kErrArg, "pr_evaluate_device_own: null buffer");
    if (!b || !b->avg_on) return fail(kErrArg, "pr_evaluate_device_own: average strategies are not enabled");
    return evaluate_impl(b, (EvalTables *)eval, updating_player, 0, d_ranges, d_results, (cudaStream_t)stream,
                         false, d_own);
}

namespace {
// Row copies between caller rows of 1326 and staging rows of kRangeStride, split over host
// threads for large batches (one thread copies ~25 MB/s per row call otherwise idle cores).
// With `checked`, rows that hold a NaN, an infinity or a negative weight are not copied; the
// return value counts them.
int copy_rows(float *dst, size_t dst_stride, const float *src, size_t src_stride, int count, bool checked = false) {
    std::atomic<int> rejected{0};
    auto part = [&](int lo, int hi) {
        for (int i = lo; i < hi; i++) {
            const float *row = src + (size_t)i * src_stride;
            if (checked) {
                float bad = 0.0f;
                for (int h = 0; h < kHands; h++) bad += (row[h] - row[h]) + (row[h] < 0.0f ? 1.0f : 0.0f);
                if (bad != 0.0f) {
                    rejected++;
                    continue;
                }
            }
            memcpy(dst + (size_t)i * dst_stride, row, kHands * sizeof(float));
        }
    };
    const int threads = count >= 4096 ? (int)std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    if (threads <= 1) {
        part(0, count);
        return rejected.load();
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
        pool.emplace_back(part, (int)((long long)count * t / threads), (int)((long long)count * (t + 1) / threads));
    for (auto &th : pool) th.join();
    return rejected.load();
}
}  // namespace

int pr_upload_batch(void *builder, int first, int count, const float *v) {
    Builder *b = (Builder *)builder;
    if (!b || !v || first < 0 || count < 0 || first + count > (int)b->desc.size())
        return fail(kErrArg, "pr_upload_batch: bad builder or range");
    if (copy_rows(b->comm + (size_t)first * kRangeStride, kRangeStride, v, kHands, count, true))
        return fail(kErrArg, "pr_upload_batch: a range holds a NaN, an infinity or a negative weight (row not copied)");
    return kOk;
}

int pr_download_batch(void *builder, int first, int count, float *v) {
    Builder *b = (Builder *)builder;
    if (!b || !v || first < 0 || count < 0 || first + count > (int)b->desc.size())
        return fail(kErrArg, "pr_download_batch: bad builder or range");
    copy_rows(v, kHands, b->comm + (size_t)first * kRangeStride, kRangeStride, count);
    return kOk;
}

int pr_enable_average(void *builder) {
    Builder *b = (Builder *)builder;
    if (!b) return fail(kErrArg, "pr_enable_average: null builder");
    if (b->avg_on) return kOk;
    b->avg_on = true;
    const int cap = b->capacity;
    b->capacity = 0;  // re-allocate both staging areas at the current capacity
    float *old = b->comm;
    b->comm = nullptr;
    if (!grow_staging(b, cap)) return kErrAlloc;
    memcpy(b->comm, old, (size_t)cap * kRangeStride * sizeof(float));
    cudaFreeHost(old);
    return kOk;
}

void pr_upload_own(void *builder, int index, const float *v) {
    Builder *b = (Builder *)builder;
    if (!b || !b->avg_on || index < 0 || index >= (int)b->desc.size() || !v) {
        fail(kErrArg, "pr_upload_own: bad builder or index, or averages not enabled");
        return;
    }
    memcpy(b->comm_own + (size_t)index * kRangeStride, v, kHands * sizeof(float));
}

int pr_get_average(void *builder, float *out) {
    Builder *b = (Builder *)builder;
    if (!b || !out || !b->avg_on) return fail(kErrArg, "pr_get_average: averages not enabled");
    int st = sync_device(b);
    if (st) return st;
    if ((st = sync_average(b))) return st;
    cudaError_t e = cudaMemcpyAsync(out, b->d_avg, (size_t)b->dev_count * kEdges * kBuckets * sizeof(float),
                                    cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? kOk : fail(kErrCuda, "average download", e);
}

int pr_set_average(void *builder, const float *in) {
    Builder *b = (Builder *)builder;
    if (!b || !in || !b->avg_on) return fail(kErrArg, "pr_set_average: averages not enabled");
    int st = sync_device(b);
    if (st) return st;
    if ((st = sync_average(b))) return st;
    cudaError_t e = cudaMemcpyAsync(b->d_avg, in, (size_t)b->dev_count * kEdges * kBuckets * sizeof(float),
                                    cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? kOk : fail(kErrCuda, "average upload", e);
}

int pr_builder_count(void *builder) { return builder ? (int)((Builder *)builder)->desc.size() : 0; }

int pr_range_stride(void) { return kRangeStride; }

int pr_get_regrets(void *builder, float *out) {
    Builder *b = (Builder *)builder;
    if (!b || !out) return fail(kErrArg, "pr_get_regrets: null argument");
    int st = sync_device(b);
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync(out, b->d_regrets, (size_t)b->dev_count * kEdges * kBuckets * sizeof(float),
                                    cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return fail(kErrCuda, "regret download", e);
    return kOk;
}

int pr_set_regrets(void *builder, const float *in) {
    Builder *b = (Builder *)builder;
    if (!b || !in) return fail(kErrArg, "pr_set_regrets: null argument");
    int st = sync_device(b);
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync(b->d_regrets, in, (size_t)b->dev_count * kEdges * kBuckets * sizeof(float),
                                    cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return fail(kErrCuda, "regret upload", e);
    return kOk;
}

void pr_free_builder(void *builder) {
    Builder *b = (Builder *)builder;
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    cudaFree(b->d_desc);
    cudaFree(b->d_ranges);
    cudaFree(b->d_results);
    cudaFree(b->d_regrets);
    cudaFree(b->d_ranges64);
    cudaFree(b->d_results64);
    cudaFree(b->d_own);
    cudaFree(b->d_avg);
    if (b->comm_own) cudaFreeHost(b->comm_own);
    if (b->comm) cudaFreeHost(b->comm);
    if (b->copy_in) cudaStreamSynchronize(b->copy_in);
    if (b->copy_out) cudaStreamSynchronize(b->copy_out);
    for (int k = 0; k < kPipeChunks; k++) {
        if (b->ev_in[k]) cudaEventDestroy(b->ev_in[k]);
        if (b->ev_done[k]) cudaEventDestroy(b->ev_done[k]);
    }
    if (b->copy_in) cudaStreamDestroy(b->copy_in);
    if (b->copy_out) cudaStreamDestroy(b->copy_out);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

void *pr_tables_build(uint64_t flop) {
    EvalTables *t = acquire_tables();
    if (t->status) return t;
    t->flop = flop;
    if (__builtin_popcountll(flop) != 3 || (flop >> 52)) {
        fail(kErrArg, "pr_tables_build: a flop is three cards");
        t->status = 32;
        return t;
    }
    cudaError_t e = launch_gen_tables(flop, t->d_eval, t->d_coll, t->d_abstr, 0);
    if (e != cudaSuccess) {
        fail(kErrCuda, "table generation", e);
        t->status = -1;
        return t;
    }
    repack_tables(t);
    return t;
}

int pr_tables_export(void *eval, uint16_t *eval_out, uint16_t *coll_out, uint16_t *abstr_out) {
    EvalTables *t = (EvalTables *)eval;
    if (!t || t->status) return fail(kErrArg, "pr_tables_export: invalid table handle");
    cudaError_t e;
    if ((eval_out && (e = cudaMemcpy(eval_out, t->d_eval, kEvalBytes, cudaMemcpyDeviceToHost)) != cudaSuccess) ||
        (coll_out && (e = cudaMemcpy(coll_out, t->d_coll, kCollBytes, cudaMemcpyDeviceToHost)) != cudaSuccess) ||
        (abstr_out && (e = cudaMemcpy(abstr_out, t->d_abstr, kAbstrBytes, cudaMemcpyDeviceToHost)) != cudaSuccess))
        return fail(kErrCuda, "table export", e);
    return kOk;
}

int pr_eval_status(void *eval) { return eval ? ((EvalTables *)eval)->status : -1; }

// ---- table files ---------------------------------------------------------------------
// Layout (little endian): magic "PRBTABL1" | u32 version (1) | u32 reserved | u64 flop |
// u64 FNV-1a 64 hash of the three arrays | eval u16[1326 * 1838] | coll u16[1326 * 2652] |
// buckets u16[1326 * 1326] -- the packed form transfer_flop_eval_cuda takes.
namespace {
struct TablesHeader {
    char magic[8];
    uint32_t version, reserved;
    uint64_t flop, hash;
};
uint64_t fnv1a64(const void *p, size_t n, uint64_t h) {
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < n; i++) h = (h ^ c[i]) * 1099511628211ull;
    return h;
}
}  // namespace

int pr_tables_save(void *eval, const char *path) {
    EvalTables *t = (EvalTables *)eval;
    if (!t || t->status || !path) return fail(kErrArg, "pr_tables_save: invalid table handle or path");
    std::vector<uint16_t> e(kEvalBytes / 2), c(kCollBytes / 2), a(kAbstrBytes / 2);
    if (int st = pr_tables_export(eval, e.data(), c.data(), a.data())) return st;
    TablesHeader h{};
    memcpy(h.magic, "PRBTABL1", 8);
    h.version = 1;
    h.flop = t->flop;
    uint64_t x = 1469598103934665603ull;
    x = fnv1a64(e.data(), kEvalBytes, x);
    x = fnv1a64(c.data(), kCollBytes, x);
    x = fnv1a64(a.data(), kAbstrBytes, x);
    h.hash = x;
    FILE *f = fopen(path, "wb");
    if (!f) return fail(kErrArg, "pr_tables_save: cannot open the file");
    bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && fwrite(e.data(), 1, kEvalBytes, f) == kEvalBytes &&
              fwrite(c.data(), 1, kCollBytes, f) == kCollBytes && fwrite(a.data(), 1, kAbstrBytes, f) == kAbstrBytes;
    ok = (fclose(f) == 0) && ok;
    return ok ? kOk : fail(kErrArg, "pr_tables_save: write failed");
}

// Reads a table file and uploads it as transfer_flop_eval_cuda does (the same validation);
// null if the file is missing, truncated or corrupted.
void *pr_tables_load(const char *path) {
    if (!path) return nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) {
        fail(kErrArg, "pr_tables_load: cannot open the file");
        return nullptr;
    }
    TablesHeader h{};
    std::vector<uint16_t> e(kEvalBytes / 2), c(kCollBytes / 2), a(kAbstrBytes / 2);
    bool ok = fread(&h, sizeof(h), 1, f) == 1 && memcmp(h.magic, "PRBTABL1", 8) == 0 && h.version == 1 &&
              fread(e.data(), 1, kEvalBytes, f) == kEvalBytes && fread(c.data(), 1, kCollBytes, f) == kCollBytes &&
              fread(a.data(), 1, kAbstrBytes, f) == kAbstrBytes;
    fclose(f);
    if (ok) {
        uint64_t x = 1469598103934665603ull;
        x = fnv1a64(e.data(), kEvalBytes, x);
        x = fnv1a64(c.data(), kCollBytes, x);
        x = fnv1a64(a.data(), kAbstrBytes, x);
        ok = x == h.hash;
    }
    if (!ok) {
        fail(kErrTables, "pr_tables_load: not a table file, truncated or corrupted");
        return nullptr;
    }
    std::vector<uint64_t> order(kHands);
    std::vector<uint16_t> indexes(52 * 51);
    int fill[52] = {0};
    for (int hi = 1, n = 0; hi < 52; hi++)
        for (int lo = 0; lo < hi; lo++, n++) {
            order[n] = (1ull << lo) | (1ull << hi);
            indexes[lo * 51 + fill[lo]++] = (uint16_t)n;
            indexes[hi * 51 + fill[hi]++] = (uint16_t)n;
        }
    return transfer_flop_eval_cuda(h.flop, order.data(), indexes.data(), e.data(), c.data(), a.data());
}

size_t pr_river_smem_bytes(void *eval, int calc_exploit, int fp64) {
    EvalTables *t = (EvalTables *)eval;
    if (!t || t->status) return 0;
    return river_smem_bytes(calc_exploit ? kModeBR : kModeCFR, fp64, t->max_groups, t->max_card_groups);
}

namespace {
// Double-precision best response: host rows of 1326 (staged through the builder's device
// buffers) or device rows of kRangeStride on the caller's stream.
int br64_impl(Builder *b, EvalTables *t, int updating_player, const double *ranges, double *results,
              bool staged, cudaStream_t stream) {
    if (!b || !t || !ranges || !results) return fail(kErrArg, "pr_evaluate_br64: null argument");
    if (t->status) return fail(kErrTables, "pr_evaluate_br64: tables failed validation");
    if (updating_player != 0 && updating_player != 1) return fail(kErrArg, "pr_evaluate_br64: bad player");
    for (const SubgameDesc &d : b->desc)
        if ((d.board4 & t->flop) != t->flop || __builtin_popcountll(d.board4) != 4)
            return fail(kErrArg, "pr_evaluate_br64: a river root's board does not contain the flop");
    int st = sync_device(b);
    if (st) return st;
    const int n = b->dev_count;
    if (n == 0) return kOk;
    cudaError_t e;
    if (!staged) {
        e = launch_river_br64(b->d_desc, n, ranges, results, b->d_regrets, t->packs, t->flop, updating_player,
                              t->max_groups, t->max_card_groups, stream ? stream : b->stream);
        return e == cudaSuccess ? kOk : fail(kErrCuda, "double best-response launch", e);
    }
    if (b->cap64 < b->dev_capacity) {
        cudaFree(b->d_ranges64);
        cudaFree(b->d_results64);
        b->d_ranges64 = b->d_results64 = nullptr;
        b->cap64 = 0;
        const size_t bytes = (size_t)b->dev_capacity * kRangeStride * sizeof(double);
        if ((e = cudaMalloc(&b->d_ranges64, bytes)) != cudaSuccess ||
            (e = cudaMalloc(&b->d_results64, bytes)) != cudaSuccess)
            return fail(kErrAlloc, "double-precision buffers", e);
        cudaMemset(b->d_ranges64, 0, bytes);
        b->cap64 = b->dev_capacity;
    }
    // host rows of 1326 -> device rows of kRangeStride
    e = cudaMemcpy2DAsync(b->d_ranges64, kRangeStride * sizeof(double), ranges, kHands * sizeof(double),
                          kHands * sizeof(double), n, cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return fail(kErrCuda, "double range upload", e);
    e = launch_river_br64(b->d_desc, n, b->d_ranges64, b->d_results64, b->d_regrets, t->packs, t->flop,
                          updating_player, t->max_groups, t->max_card_groups, b->stream);
    if (e != cudaSuccess) return fail(kErrCuda, "double best-response launch", e);
    e = cudaMemcpy2DAsync(results, kHands * sizeof(double), b->d_results64, kRangeStride * sizeof(double),
                          kHands * sizeof(double), n, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return fail(kErrCuda, "double best-response pass", e);
    return kOk;
}
}  // namespace

int pr_evaluate_br64(void *builder, void *eval, int updating_player, const double *ranges, double *results) {
    return br64_impl((Builder *)builder, (EvalTables *)eval, updating_player, ranges, results, true, nullptr);
}

int pr_evaluate_br64_device(void *builder, void *eval, int updating_player, const double *d_ranges,
                            double *d_results, void *stream) {
    return br64_impl((Builder *)builder, (EvalTables *)eval, updating_player, d_ranges, d_results, false,
                     (cudaStream_t)stream);
}

}  // extern "C"
