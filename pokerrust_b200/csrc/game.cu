// Host driver of the whole fixed-flop game over the C ABI: the part of the reference's
// `--features GPU` program above the river solver (src/builder.rs, src/state.rs,
// src/strategy.rs:37-82, src/permutation_handler.rs, src/game.rs), as a C++ library.
//
// The preflop, flop and turn tree is built from the reference's rules (builder.rs:13-79,
// state.rs:66-217) into flat node arrays; the river roots it reaches are registered with
// build_river_cuda in the same order the reference registers them. A half-iteration is the
// reference's GPU protocol (game.rs:68-119): an upload pass that stores every river root's
// opponent range in the staging (state.rs:379-387), one evaluate_cuda, and a download pass
// that reads the river values back and updates the upper-tree regrets (state.rs:219-296,
// strategy.rs:57-66). Turn children run on a thread pool (state.rs:340-341 uses rayon).
// The upload pass only propagates ranges: in the reference its utilities are discarded.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <limits>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "../../include/pokerrust_b200.h"
#include "layout.h"
#include "trace.h"
#include "upper_tree.h"

namespace prb {
namespace {

constexpr int H = 1326;
enum Kind : int8_t { kDecide = 0, kSBWins = 1, kBBWins = 2, kFlop = 4, kTurn = 5, kRiverRoot = 6 };
enum Act : int8_t { Fold, Check, Call, Raise, DealHole, DealFlop, DealTurn, DealRiver };

struct UNode {
    int8_t kind, actor, action, nchild;
    int32_t first;       // first child in `kids`
    uint64_t cards;
    float sb, bb;
    int64_t regret;      // offset of nchild * H regrets (decision nodes)
    int32_t river;       // river root index (kRiverRoot)
    int32_t perm_first;  // flop nodes: suit permutations [perm_first, perm_first + nperm)
    int32_t nperm;
};

// Thread pool with a blocking parallel-for; the caller works too.
class Pool {
  public:
    explicit Pool(int n) {
        for (int i = 0; i < n; i++) workers_.emplace_back([this] { loop(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : workers_) t.join();
    }
    void run(int n, const std::function<void(int)> &f) {
        if (workers_.empty() || n <= 1) {
            for (int i = 0; i < n; i++) f(i);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &f;
            n_ = n;
            next_.store(0);
            active_ = (int)workers_.size();
            gen_++;
        }
        cv_.notify_all();
        for (int i; (i = next_.fetch_add(1)) < n;) f(i);
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return active_ == 0; });
        job_ = nullptr;
    }
  private:
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(int)> *job;
            int n;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                job = job_;
                n = n_;
            }
            for (int i; (i = next_.fetch_add(1)) < n;) (*job)(i);
            std::lock_guard<std::mutex> lk(mu_);
            if (--active_ == 0) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)> *job_ = nullptr;
    int n_ = 0, active_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
    std::atomic<int> next_{0};
};

// Per-thread scratch: vectors of H values per recursion depth.
template <typename T>
struct Scratch {
    static constexpr int kSlots = 9;  // avg, 3 strategies, child range, 3 results, misc
    std::vector<T> buf;
    explicit Scratch(int depth) : buf((size_t)depth * kSlots * H) {}
    T *at(int depth, int slot) { return buf.data() + ((size_t)depth * kSlots + slot) * H; }
};

enum Pass { kUpload = 0, kDownload = 1 };

// Device copy of the upper tree (upper_tree.cu): nodes, the level lists of the two sweeps,
// regrets and average sums, reach vectors and values of every node, the river rows.
struct DevTree {
    cudaStream_t stream = nullptr;
    DevNode *nodes = nullptr;
    int32_t *kids = nullptr, *perm_maps = nullptr, *levels = nullptr;
    std::vector<int> level_off;  // level d = levels[level_off[d], level_off[d + 1])
    float *regrets = nullptr, *avg = nullptr;
    float *Rf = nullptr, *Vf = nullptr;   // [node][2][kRangeStride], [node][kRangeStride]
    double *Rd = nullptr, *Vd = nullptr;  // double-precision best response (lazily allocated)
    float *opp = nullptr, *val = nullptr, *own = nullptr;  // [river][kRangeStride]
    double *opp64 = nullptr, *val64 = nullptr;
    float *root_vals = nullptr;           // [2][kRangeStride]: the root's values of the last CFR pass per updater
    cudaGraphExec_t graph = nullptr;      // one CFR iteration, replayed
    bool graph_avg = false, graph_failed = false;
    bool ready = false;
};

struct Game {
    uint64_t flop = 0;
    void *tables = nullptr;
    void *builder = nullptr;
    std::vector<UNode> nodes;
    std::vector<int32_t> kids;
    std::vector<float> regrets;
    std::vector<float> avg_upper;                 // average-strategy sums, same layout as regrets
    bool avg_on = false;
    std::vector<std::array<int, 4>> perms;
    std::vector<std::vector<int32_t>> perm_maps;  // hand index -> permuted hand index
    std::vector<uint64_t> card_order;
    std::vector<uint64_t> river_board;
    std::vector<float> river_bet;
    std::vector<double> ranges64, results64;      // double-precision best-response staging
    Pool *pool = nullptr;
    int max_depth = 0;
    double t_host = 0, t_gpu = 0;
    int status = 0;
    bool device_tree = true;
    DevTree dt;
    std::vector<float> root_host[2];  // the root's values of the host traversal's last CFR pass per updater
    int root_where = 0;               // 0: no CFR pass yet, 1: root_host, 2: dt.root_vals
    bool host_stale = false;  // the device holds newer upper regrets / sums than the host
    bool dev_stale = true;    // the host holds newer ones than the device

    // ---- tree construction (builder.rs:34-79, state.rs:66-217) ----
    static int popc(uint64_t x) { return __builtin_popcountll(x); }

    void possible(const UNode &s, int raises, std::vector<int> &out) const {
        out.clear();
        switch (s.action) {
            case Fold: break;
            case Check: out = {Call, Raise}; break;
            case Call:
                if (popc(s.cards) == 0) out = {DealFlop};
                else if (popc(s.cards) == 3) out = {DealTurn};
                break;  // 4 cards: a river root, solved on the device
            case Raise:
                out = {Fold, Call};
                if (raises < 4) out.push_back(Raise);
                break;
            case DealHole: out = {Fold, Check, Raise}; break;
            default: out = {Check, Raise}; break;
        }
    }

    static uint64_t permute_cards(uint64_t cards, const std::array<int, 4> &p) {
        uint64_t o = 0;
        while (cards) {
            const int c = __builtin_ctzll(cards);
            cards &= cards - 1;
            o |= 1ull << (13 * p[c / 13] + c % 13);
        }
        return o;
    }

    static int colex2(uint64_t set) {
        const int a = __builtin_ctzll(set);
        set &= set - 1;
        const int b = __builtin_ctzll(set);
        return a + b * (b - 1) / 2;
    }

    // children states of `s` for `action` (state.rs:66-217)
    void children_of(const UNode &s, int action, std::vector<UNode> &out) {
        out.clear();
        UNode t{};
        t.kind = s.kind;
        t.action = (int8_t)action;
        t.cards = s.cards;
        t.sb = s.sb;
        t.bb = s.bb;
        t.actor = s.actor == 0 ? 1 : 0;
        t.river = -1;
        const float other = s.actor == 0 ? s.bb : s.sb;
        switch (action) {
            case Fold: t.kind = s.actor == 0 ? kBBWins : kSBWins; break;
            case Check:
                t.kind = kDecide;
                t.sb = s.bb;
                break;
            case Call:
                t.sb = t.bb = other;
                if (popc(s.cards) == 0) {
                    t.kind = kFlop;
                } else if (popc(s.cards) == 3) {
                    t.kind = kTurn;
                } else {
                    t.kind = kRiverRoot;
                    t.river = (int)river_board.size();
                    river_board.push_back(s.cards);
                    river_bet.push_back(other);
                }
                break;
            case Raise: {
                const float amount = popc(s.cards) < 4 ? 1.0f : 2.0f;
                t.kind = kDecide;
                if (s.actor == 0) t.sb = s.bb + amount;
                else t.bb = s.sb + amount;
                break;
            }
            case DealFlop: {
                // the one fixed flop and the suit permutations of [C, H, S, D], in
                // lexicographic order, that reach a flop not seen before (state.rs:146-172)
                std::set<uint64_t> seen;
                std::array<int, 4> p = {0, 1, 2, 3};
                t.perm_first = (int)perms.size();
                t.nperm = 0;
                do {
                    if (seen.insert(permute_cards(flop, p)).second) {
                        perms.push_back(p);
                        t.nperm++;
                    }
                } while (std::next_permutation(p.begin(), p.end()));
                t.kind = kDecide;
                t.cards = flop;
                t.actor = 0;
                break;
            }
            case DealTurn:
                for (int c = 0; c < 52; c++) {
                    if ((s.cards >> c) & 1) continue;
                    UNode n = t;
                    n.kind = kDecide;
                    n.cards = s.cards | (1ull << c);
                    n.actor = 0;
                    out.push_back(n);
                }
                return;
        }
        out.push_back(t);
    }

    int build(int si, int raises, int depth) {
        max_depth = std::max(max_depth, depth + 1);
        std::vector<int> acts;
        possible(nodes[si], raises, acts);
        std::vector<int> kids_here;
        std::vector<UNode> ch;
        for (int a : acts) {
            const int nr = a == Raise ? raises + 1 : (a == DealFlop || a == DealTurn) ? 0 : raises;
            children_of(nodes[si], a, ch);
            for (UNode &c : ch) {
                const int ci = (int)nodes.size();
                nodes.push_back(c);
                build(ci, nr, depth + 1);
                kids_here.push_back(ci);
            }
        }
        UNode &s = nodes[si];
        s.first = (int)kids.size();
        s.nchild = (int8_t)kids_here.size();
        kids.insert(kids.end(), kids_here.begin(), kids_here.end());
        if (s.kind == kDecide && s.nchild > 0) {
            s.regret = (int64_t)regrets.size();
            regrets.resize(regrets.size() + (size_t)s.nchild * H, 0.0f);
        }
        return si;
    }

    bool init(uint64_t f, int nthreads) {
        flop = f;
        card_order.resize(H);
        for (int hi = 1, n = 0; hi < 52; hi++)
            for (int lo = 0; lo < hi; lo++) card_order[n++] = (1ull << lo) | (1ull << hi);
        UNode root{};
        root.kind = kDecide;
        root.action = DealHole;
        root.sb = 0.5f;
        root.bb = 1.0f;
        root.actor = 0;
        root.river = -1;
        nodes.reserve(1 << 18);
        nodes.push_back(root);
        build(0, 1, 0);
        perm_maps.resize(perms.size());
        for (size_t i = 0; i < perms.size(); i++) {
            perm_maps[i].resize(H);
            for (int h = 0; h < H; h++) perm_maps[i][h] = colex2(permute_cards(card_order[h], perms[i]));
        }
        tables = pr_tables_build(flop);
        if (!tables || pr_eval_status(tables) != 0) return false;
        builder = init_builder();
        if (!builder) return false;
        for (size_t i = 0; i < river_board.size(); i++)
            if (build_river_cuda(river_board[i], river_bet[i], builder) != (int)i) return false;
        if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
        pool = new Pool(std::max(0, nthreads - 1));
        return true;
    }

    ~Game() {
        delete pool;
        dt_release();
        if (builder) pr_free_builder(builder);
        if (tables) free_eval_cuda(tables);
    }

    // ---- device upper tree ----
    void dt_release() {
        if (dt.graph) cudaGraphExecDestroy(dt.graph);
        if (dt.stream) cudaStreamSynchronize(dt.stream);
        for (void *p : {(void *)dt.nodes, (void *)dt.kids, (void *)dt.perm_maps, (void *)dt.levels,
                        (void *)dt.regrets, (void *)dt.avg, (void *)dt.Rf, (void *)dt.Vf, (void *)dt.Rd,
                        (void *)dt.Vd, (void *)dt.opp, (void *)dt.val, (void *)dt.own, (void *)dt.opp64,
                        (void *)dt.val64, (void *)dt.root_vals})
            cudaFree(p);
        if (dt.stream) cudaStreamDestroy(dt.stream);
        dt = DevTree();
    }

    static int cuda_fail(const char *what, cudaError_t e) {
        fprintf(stderr, "pokerrust_b200: device upper tree: %s: %s\n", what, cudaGetErrorString(e));
        return 1;
    }

    template <typename X>
    static cudaError_t upload(X **dst, const X *src, size_t n) {
        cudaError_t e = cudaMalloc((void **)dst, n * sizeof(X));
        if (e == cudaSuccess && src) e = cudaMemcpy(*dst, src, n * sizeof(X), cudaMemcpyHostToDevice);
        return e;
    }

    int dt_init() {
        if (dt.ready) return 0;
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&dt.stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail("stream", e);
        const size_t N = nodes.size(), R = river_board.size();
        std::vector<DevNode> dn(N);
        std::vector<int> depth(N, 0);
        int D = 1;
        for (size_t i = 0; i < N; i++) {
            const UNode &u = nodes[i];
            DevNode &d = dn[i];
            d = DevNode{};
            d.kind = u.kind;
            d.actor = u.actor;
            d.nchild = u.nchild;
            d.first = u.first;
            d.cards = u.cards;
            d.sb = u.sb;
            d.bb = u.bb;
            d.regret = u.regret;
            d.river = u.river;
            d.perm_first = u.perm_first;
            d.nperm = u.nperm;
            for (int k = 0; k < u.nchild; k++) {  // children follow their parent in `nodes`
                depth[kids[u.first + k]] = depth[i] + 1;
                D = std::max(D, depth[i] + 2);
            }
        }
        std::vector<int32_t> lv;
        dt.level_off.assign(1, 0);
        for (int d = 0; d < D; d++) {
            for (size_t i = 0; i < N; i++)
                if (depth[i] == d) lv.push_back((int32_t)i);
            dt.level_off.push_back((int)lv.size());
        }
        std::vector<int32_t> pm;
        for (auto &m : perm_maps) pm.insert(pm.end(), m.begin(), m.end());
        if ((e = upload(&dt.nodes, dn.data(), N)) != cudaSuccess || (e = upload(&dt.kids, kids.data(), kids.size())) ||
            (e = upload(&dt.perm_maps, pm.data(), pm.size())) || (e = upload(&dt.levels, lv.data(), lv.size())) ||
            (e = upload(&dt.regrets, regrets.data(), regrets.size())) ||
            (e = upload<float>(&dt.Rf, nullptr, N * 2 * kRangeStride)) ||
            (e = upload<float>(&dt.Vf, nullptr, N * kRangeStride)) ||
            (e = upload<float>(&dt.opp, nullptr, R * kRangeStride)) ||
            (e = upload<float>(&dt.val, nullptr, R * kRangeStride)) ||
            (e = upload<float>(&dt.root_vals, nullptr, 2 * kRangeStride)))
            return cuda_fail("allocation", e);
        dt.ready = true;
        dev_stale = true;
        return 0;
    }

    int dt_alloc64() {
        if (dt.Rd) return 0;
        const size_t N = nodes.size(), R = river_board.size();
        cudaError_t e;
        if ((e = upload<double>(&dt.Rd, nullptr, N * 2 * kRangeStride)) ||
            (e = upload<double>(&dt.Vd, nullptr, N * kRangeStride)) ||
            (e = upload<double>(&dt.opp64, nullptr, R * kRangeStride)) ||
            (e = upload<double>(&dt.val64, nullptr, R * kRangeStride)))
            return cuda_fail("double-precision allocation", e);
        return 0;
    }

    // host -> device copies of the upper regrets and sums when the host changed them
    int dt_push() {
        if (int st = dt_init()) return st;
        if (!dev_stale) return 0;
        cudaError_t e = cudaMemcpy(dt.regrets, regrets.data(), regrets.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && avg_on) {
            const size_t rows = (size_t)river_board.size() * kRangeStride;
            if (!dt.avg && (e = cudaMalloc(&dt.avg, avg_upper.size() * 4)) == cudaSuccess)
                e = cudaMalloc(&dt.own, rows * 4);
            if (e == cudaSuccess) e = cudaMemset(dt.own, 0, rows * 4);
            if (e == cudaSuccess) e = cudaMemcpy(dt.avg, avg_upper.data(), avg_upper.size() * 4, cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) return cuda_fail("regret upload", e);
        dev_stale = false;
        return 0;
    }

    // device -> host copies when the device changed them
    int dt_pull() {
        if (!host_stale) return 0;
        cudaError_t e = cudaStreamSynchronize(dt.stream);
        if (e == cudaSuccess)
            e = cudaMemcpy(regrets.data(), dt.regrets, regrets.size() * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && avg_on && dt.avg)
            e = cudaMemcpy(avg_upper.data(), dt.avg, avg_upper.size() * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail("regret download", e);
        host_stale = false;
        return 0;
    }

    // One half-iteration or best-response pass on the device, enqueued on dt.stream:
    // root ranges, top-down levels, the river pass, bottom-up levels.
    template <typename T>
    int dt_half(int upd, bool br) {
        const bool f64 = sizeof(T) == 8;
        T *R = f64 ? (T *)dt.Rd : (T *)dt.Rf;
        T *V = f64 ? (T *)dt.Vd : (T *)dt.Vf;
        T *opp = f64 ? (T *)dt.opp64 : (T *)dt.opp;
        T *val = f64 ? (T *)dt.val64 : (T *)dt.val;
        const bool avg = avg_on && !br;
        UpperView v{dt.nodes, dt.kids, dt.perm_maps, dt.regrets};
        cudaError_t e = upper_set_root(f64 ? nullptr : dt.Rf, f64 ? dt.Rd : nullptr, dt.stream);
        const int D = (int)dt.level_off.size() - 1;
        for (int d = 0; d < D && e == cudaSuccess; d++)
            e = upper_down<T>(v, dt.levels + dt.level_off[d], dt.level_off[d + 1] - dt.level_off[d], upd, R,
                              opp, avg ? dt.own : nullptr, dt.stream);
        if (e != cudaSuccess) return cuda_fail("top-down sweep", e);
        int st;
        if (f64) st = pr_evaluate_br64_device(builder, tables, upd, dt.opp64, dt.val64, dt.stream);
        else if (avg) st = pr_evaluate_device_own(builder, tables, upd, dt.opp, dt.own, dt.val, dt.stream);
        else st = pr_evaluate_device(builder, tables, upd, br ? 1 : 0, dt.opp, dt.val, dt.stream);
        if (st) return st;
        for (int d = D - 1; d >= 0 && e == cudaSuccess; d--)
            e = upper_up<T>(v, dt.levels + dt.level_off[d], dt.level_off[d + 1] - dt.level_off[d], upd, br ? 1 : 0,
                            R, V, val, dt.regrets, avg ? dt.avg : nullptr, dt.stream);
        if (e != cudaSuccess) return cuda_fail("bottom-up sweep", e);
        if (!f64 && !br) {  // keep the root's values of this CFR pass (node 0 is the root)
            e = cudaMemcpyAsync(dt.root_vals + (size_t)upd * kRangeStride, V, sizeof(float) * H,
                                cudaMemcpyDeviceToDevice, dt.stream);
            if (e != cudaSuccess) return cuda_fail("root values", e);
        }
        return 0;
    }

    // A CFR iteration as one graph: captured after an eager first iteration (which sets up
    // everything the river pass allocates lazily); eager launches if capture is refused.
    int dt_iterate(int iterations) {
        using clk = std::chrono::steady_clock;
        auto t0 = clk::now();
        if (int st = dt_push()) return st;
        if (dt.graph && dt.graph_avg != avg_on) {
            cudaGraphExecDestroy(dt.graph);
            dt.graph = nullptr;
        }
        int it = 0;
        if (!dt.graph && !dt.graph_failed && iterations > 0) {
            for (int upd = 0; upd < 2; upd++)
                if (int st = dt_half<float>(upd, false)) return st;
            it++;
            cudaError_t e = cudaStreamSynchronize(dt.stream);
            if (e != cudaSuccess) return cuda_fail("iteration", e);
            cudaGraph_t g = nullptr;
            int st = 0;
            e = cudaStreamBeginCapture(dt.stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                for (int upd = 0; upd < 2 && !st; upd++) st = dt_half<float>(upd, false);
                e = cudaStreamEndCapture(dt.stream, &g);
            }
            if (e == cudaSuccess && !st && g) e = cudaGraphInstantiate(&dt.graph, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess || st || !dt.graph) {
                cudaGetLastError();
                dt.graph = nullptr;
                dt.graph_failed = true;
                pr_clear_error();
            }
            dt.graph_avg = avg_on;
        }
        for (; it < iterations; it++) {
            if (dt.graph) {
                cudaError_t e = cudaGraphLaunch(dt.graph, dt.stream);
                if (e != cudaSuccess) return cuda_fail("graph launch", e);
            } else {
                for (int upd = 0; upd < 2; upd++)
                    if (int st = dt_half<float>(upd, false)) return st;
            }
        }
        cudaError_t e = cudaStreamSynchronize(dt.stream);
        if (e != cudaSuccess) return cuda_fail("iteration", e);
        host_stale = true;
        if (iterations > 0) root_where = 2;
        t_gpu += std::chrono::duration<double>(clk::now() - t0).count();
        return 0;
    }

    // Best-response values of both players at the root, on the device.
    template <typename T>
    int dt_exploit(T *sb, T *bb) {
        using clk = std::chrono::steady_clock;
        auto t0 = clk::now();
        if (int st = dt_push()) return st;
        if (sizeof(T) == 8)
            if (int st = dt_alloc64()) return st;
        T *V = sizeof(T) == 8 ? (T *)dt.Vd : (T *)dt.Vf;
        for (int upd = 0; upd < 2; upd++) {
            if (int st = dt_half<T>(upd, true)) return st;
            cudaError_t e = cudaMemcpyAsync(upd == 0 ? sb : bb, V, sizeof(T) * H, cudaMemcpyDeviceToHost, dt.stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(dt.stream);
            if (e != cudaSuccess) return cuda_fail("best response", e);
        }
        t_gpu += std::chrono::duration<double>(clk::now() - t0).count();
        return 0;
    }

    // ---- traversal (state.rs:219-376) ----
    template <typename T>
    void strategy(const UNode &s, T *probs) const {
        // RegularStrategy::get_strategy (strategy.rs:68-81)
        const float *r = regrets.data() + s.regret;
        const int n = s.nchild;
        for (int i = 0; i < H; i++) {
            T sum = T(0);
            for (int k = 0; k < n; k++) sum += T(r[(size_t)k * H + i]);
            for (int k = 0; k < n; k++)
                probs[(size_t)k * H + i] = sum <= T(1e-4f) ? T(1) / T(n) : T(r[(size_t)k * H + i]) / sum;
        }
    }

    template <typename T>
    void fold(const UNode &s, const T *opp, int upd, int folding, T *out) const {
        // evaluate_fold (state.rs:456-492)
        T total = T(0);
        T coll[52] = {};
        for (int i = 0; i < H; i++) {
            total += opp[i];
            coll[__builtin_ctzll(card_order[i])] += opp[i];
            coll[63 - __builtin_clzll(card_order[i])] += opp[i];
        }
        const T b = T(folding == 0 ? s.sb : s.bb);
        const T m = b * (upd == folding ? T(-1) : T(1));
        for (int i = 0; i < H; i++) {
            T v = total + opp[i];
            v -= coll[__builtin_ctzll(card_order[i])];
            v -= coll[63 - __builtin_clzll(card_order[i])];
            out[i] = v * m;
        }
    }

    template <typename T>
    void river(const UNode &s, const T *opp, const T *own, int pass, T *out);

    template <typename T>
    void eval(int si, const T *sb, const T *bb, int upd, bool br, int pass, T *out, int depth,
              Scratch<T> &sc) {
        const UNode &s = nodes[si];
        const T *opp = upd == 0 ? bb : sb;
        switch (s.kind) {
            case kDecide: {
                T *avg = sc.at(depth, 0);
                T *probs = sc.at(depth, 1);  // slots 1..3
                T *child = sc.at(depth, 4);
                T *res = sc.at(depth, 5);    // slots 5..7
                T *u = sc.at(depth, 8);
                strategy(s, probs);
                const bool mine = upd == s.actor;
                const T init = (mine && br) ? -std::numeric_limits<T>::infinity() : T(0);
                for (int i = 0; i < H; i++) avg[i] = init;
                for (int k = 0; k < s.nchild; k++) {
                    const T *p = probs + (size_t)k * H;
                    const T *own = s.actor == 0 ? sb : bb;
                    for (int i = 0; i < H; i++) child[i] = own[i] * p[i];
                    T *uk = (mine && !br) ? res + (size_t)k * H : u;
                    if (s.actor == 0) eval(kids[s.first + k], child, bb, upd, br, pass, uk, depth + 1, sc);
                    else eval(kids[s.first + k], sb, child, upd, br, pass, uk, depth + 1, sc);
                    if (pass == kUpload) continue;  // no utilities in the upload pass
                    if (mine) {
                        if (!br) for (int i = 0; i < H; i++) avg[i] += uk[i] * p[i];
                        else for (int i = 0; i < H; i++) avg[i] = std::fmax(avg[i], uk[i]);
                    } else {
                        for (int i = 0; i < H; i++) avg[i] += uk[i];
                    }
                }
                if (pass == kDownload && mine && !br && avg_on) {
                    // average-strategy sums: own reach into the node times the action probability
                    const T *own = s.actor == 0 ? sb : bb;
                    float *a = avg_upper.data() + s.regret;
                    for (int k = 0; k < s.nchild; k++)
                        for (int i = 0; i < H; i++) a[(size_t)k * H + i] += float(own[i] * probs[(size_t)k * H + i]);
                }
                if (pass == kDownload && mine && !br) {
                    // RegularStrategy::update_add (strategy.rs:57-66)
                    float *r = regrets.data() + s.regret;
                    for (int k = 0; k < s.nchild; k++)
                        for (int i = 0; i < H; i++) {
                            float &x = r[(size_t)k * H + i];
                            x = std::fmax(x + float(res[(size_t)k * H + i] - avg[i]), 0.0f);
                        }
                }
                memcpy(out, avg, sizeof(T) * H);
                return;
            }
            case kSBWins:
                if (pass == kDownload) fold(s, opp, upd, 1, out);
                return;
            case kBBWins:
                if (pass == kDownload) fold(s, opp, upd, 0, out);
                return;
            case kFlop: {
                // state.rs:301-336: mask, evaluate, mask, average over suit permutations
                T *nsb = sc.at(depth, 0), *nbb = sc.at(depth, 1), *r = sc.at(depth, 2);
                T *tot = sc.at(depth, 3);
                for (int i = 0; i < H; i++) tot[i] = T(0);
                T count = T(0);
                for (int k = 0; k < s.nchild; k++) {
                    const UNode &c = nodes[kids[s.first + k]];
                    for (int i = 0; i < H; i++) {
                        const bool blocked = card_order[i] & c.cards;
                        nsb[i] = blocked ? T(0) : sb[i];
                        nbb[i] = blocked ? T(0) : bb[i];
                    }
                    eval(kids[s.first + k], nsb, nbb, upd, br, pass, r, depth + 1, sc);
                    if (pass == kUpload) continue;
                    for (int i = 0; i < H; i++)
                        if (card_order[i] & c.cards) r[i] = T(0);
                    for (int p = 0; p < c.nperm; p++) {
                        count += T(1);
                        const int32_t *map = perm_maps[c.perm_first + p].data();
                        for (int i = 0; i < H; i++) tot[map[i]] += r[i];
                    }
                }
                if (pass == kDownload) {
                    const T scale = T(1) / count;
                    for (int i = 0; i < H; i++) out[i] = tot[i] * scale;
                }
                return;
            }
            case kTurn: {
                // state.rs:337-376: the 49 turn cards in parallel, then their mean
                const int n = s.nchild;
                std::vector<T> res((size_t)n * H);
                pool->run(n, [&](int k) {
                    thread_local Scratch<T> *tsc = nullptr;
                    thread_local int tsc_depth = 0;
                    if (!tsc || tsc_depth < max_depth + 2) {
                        delete tsc;
                        tsc = new Scratch<T>(max_depth + 2);
                        tsc_depth = max_depth + 2;
                    }
                    const UNode &c = nodes[kids[s.first + k]];
                    T *nsb = tsc->at(depth, 0), *nbb = tsc->at(depth, 1);
                    for (int i = 0; i < H; i++) {
                        const bool blocked = card_order[i] & c.cards;
                        nsb[i] = blocked ? T(0) : sb[i];
                        nbb[i] = blocked ? T(0) : bb[i];
                    }
                    T *r = res.data() + (size_t)k * H;
                    eval(kids[s.first + k], nsb, nbb, upd, br, pass, r, depth + 1, *tsc);
                    if (pass == kDownload)
                        for (int i = 0; i < H; i++)
                            if (card_order[i] & c.cards) r[i] = T(0);
                });
                if (pass == kDownload) {
                    for (int i = 0; i < H; i++) out[i] = T(0);
                    for (int k = 0; k < n; k++)
                        for (int i = 0; i < H; i++) out[i] += res[(size_t)k * H + i];
                    const T scale = T(1) / T(n);
                    for (int i = 0; i < H; i++) out[i] *= scale;
                }
                return;
            }
            case kRiverRoot:
                river(s, opp, upd == 0 ? sb : bb, pass, out);
                return;
        }
    }

    // One half-iteration or best-response pass of `upd` (game.rs:73-96 / 122-168).
    template <typename T>
    int half(int upd, bool br, T *out) {
        if (int st = dt_pull()) return st;
        if (!br) dev_stale = true;
        using clk = std::chrono::steady_clock;
        Scratch<T> sc(max_depth + 2);
        std::vector<T> ones(H, T(1));
        auto t0 = clk::now();
        eval<T>(0, ones.data(), ones.data(), upd, br, kUpload, out, 0, sc);
        auto t1 = clk::now();
        int st;
        if (sizeof(T) == 8) {
            st = pr_evaluate_br64(builder, tables, upd, ranges64.data(), results64.data());
        } else {
            st = pr_evaluate(builder, tables, upd, br ? 1 : 0);
        }
        auto t2 = clk::now();
        if (st) return st;
        eval<T>(0, ones.data(), ones.data(), upd, br, kDownload, out, 0, sc);
        auto t3 = clk::now();
        t_host += std::chrono::duration<double>((t1 - t0) + (t3 - t2)).count();
        t_gpu += std::chrono::duration<double>(t2 - t1).count();
        return 0;
    }
};

template <>
void Game::river<float>(const UNode &s, const float *opp, const float *own, int pass, float *out) {
    // state.rs:378-389: stage the opponent range, or read the device's values back
    if (pass == kUpload) {
        upload_c(builder, s.river, opp);
        if (avg_on) pr_upload_own(builder, s.river, own);
    } else {
        download_c(builder, s.river, out);
    }
}

template <>
void Game::river<double>(const UNode &s, const double *opp, const double *, int pass, double *out) {
    if (pass == kUpload) memcpy(ranges64.data() + (size_t)s.river * H, opp, sizeof(double) * H);
    else memcpy(out, results64.data() + (size_t)s.river * H, sizeof(double) * H);
}

}  // namespace
}  // namespace prb

using prb::Game;

extern "C" {

void *pr_game_new(uint64_t flop, int nthreads) {
    Game *g = new Game();
    if (!g->init(flop, nthreads)) {
        delete g;
        return nullptr;
    }
    return g;
}

void pr_game_free(void *game) { delete (Game *)game; }

int pr_game_num_rivers(void *game) { return game ? (int)((Game *)game)->river_board.size() : 0; }

int pr_game_river_roots(void *game, uint64_t *boards, float *bets) {
    Game *g = (Game *)game;
    if (!g || !boards || !bets) return 2;
    for (size_t i = 0; i < g->river_board.size(); i++) {
        boards[i] = g->river_board[i];
        bets[i] = g->river_bet[i];
    }
    return 0;
}

void *pr_game_builder(void *game) { return game ? ((Game *)game)->builder : nullptr; }
void *pr_game_tables(void *game) { return game ? ((Game *)game)->tables : nullptr; }

int pr_game_iterate(void *game, int iterations) {
    prb::TraceRange trace("game iterations");
    Game *g = (Game *)game;
    if (!g) return 2;
    if (g->device_tree) return g->dt_iterate(iterations);
    for (int it = 0; it < iterations; it++) {
        for (int upd = 0; upd < 2; upd++) {
            g->root_host[upd].resize(prb::H);
            const int st = g->half<float>(upd, false, g->root_host[upd].data());
            if (st) return st;
            g->root_where = 1;
        }
    }
    return 0;
}

int pr_game_root_values(void *game, float *sb, float *bb) {
    Game *g = (Game *)game;
    if (!g || !sb || !bb || !g->root_where) return 2;
    if (g->root_where == 1) {
        memcpy(sb, g->root_host[0].data(), sizeof(float) * prb::H);
        memcpy(bb, g->root_host[1].data(), sizeof(float) * prb::H);
        return 0;
    }
    cudaError_t e = cudaStreamSynchronize(g->dt.stream);
    if (e == cudaSuccess) e = cudaMemcpy(sb, g->dt.root_vals, sizeof(float) * prb::H, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(bb, g->dt.root_vals + prb::kRangeStride, sizeof(float) * prb::H, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : Game::cuda_fail("root values", e);
}

int pr_game_exploitability(void *game, int fp64, double *sum_sb, double *sum_bb, double *mbh) {
    prb::TraceRange trace("game exploitability");
    Game *g = (Game *)game;
    if (!g) return 2;
    if (fp64) {
        if (!g->device_tree) {
            const size_t n = g->river_board.size() * prb::H;
            g->ranges64.assign(n, 0.0);
            g->results64.assign(n, 0.0);
        }
        std::vector<double> sb(prb::H), bb(prb::H);
        int st;
        if (g->device_tree) {
            st = g->dt_exploit<double>(sb.data(), bb.data());
        } else {
            st = g->half<double>(0, true, sb.data());
            if (!st) st = g->half<double>(1, true, bb.data());
        }
        if (st) return st;
        double s1 = 0, s2 = 0;
        for (int i = 0; i < prb::H; i++) {
            s1 += sb[i];
            s2 += bb[i];
        }
        *sum_sb = s1;
        *sum_bb = s2;
        *mbh = (s1 + s2) * 1000.0 / 1326.0 / 1255.0 / 2.0;
        return 0;
    }
    std::vector<float> sb(prb::H), bb(prb::H);
    int st;
    if (g->device_tree) {
        st = g->dt_exploit<float>(sb.data(), bb.data());
    } else {
        st = g->half<float>(0, true, sb.data());
        if (!st) st = g->half<float>(1, true, bb.data());
    }
    if (st) return st;
    float s1 = 0, s2 = 0;
    for (int i = 0; i < prb::H; i++) {
        s1 += sb[i];
        s2 += bb[i];
    }
    *sum_sb = s1;
    *sum_bb = s2;
    *mbh = (double)((s1 + s2) * 1000.0f / 1326.0f / 1255.0f / 2.0f);  // game.rs:175
    return 0;
}

int pr_game_timings(void *game, double *host_seconds, double *device_seconds) {
    Game *g = (Game *)game;
    if (!g) return 2;
    *host_seconds = g->t_host;
    *device_seconds = g->t_gpu;
    return 0;
}

int pr_game_set_device_tree(void *game, int on) {
    Game *g = (Game *)game;
    if (!g) return -1;
    const int was = g->device_tree ? 1 : 0;
    g->device_tree = on != 0;
    return was;
}

int pr_game_get_regrets(void *game, float *upper, float *river) {
    Game *g = (Game *)game;
    if (!g) return 2;
    if (int st = g->dt_pull()) return st;
    if (upper) memcpy(upper, g->regrets.data(), g->regrets.size() * sizeof(float));
    if (river) return pr_get_regrets(g->builder, river);
    return 0;
}

int pr_game_set_regrets(void *game, const float *upper, const float *river) {
    Game *g = (Game *)game;
    if (!g) return 2;
    if (upper)
        for (size_t i = 0; i < g->regrets.size(); i++)
            if (!std::isfinite(upper[i])) return 2;
    if (river)
        for (size_t i = 0, n = g->river_board.size() * 26 * 256; i < n; i++)
            if (!std::isfinite(river[i])) return 2;
    if (int st = g->dt_pull()) return st;
    if (river)
        if (int st = pr_set_regrets(g->builder, river)) return st;
    if (upper) memcpy(g->regrets.data(), upper, g->regrets.size() * sizeof(float));
    g->dev_stale = true;
    return 0;
}

size_t pr_game_upper_regret_count(void *game) { return game ? ((Game *)game)->regrets.size() : 0; }

int pr_game_enable_average(void *game) {
    Game *g = (Game *)game;
    if (!g) return 2;
    if (g->avg_on) return 0;
    if (int st = g->dt_pull()) return st;
    const int st = pr_enable_average(g->builder);
    if (st) return st;
    g->avg_upper.assign(g->regrets.size(), 0.0f);
    g->avg_on = true;
    g->dev_stale = true;
    return 0;
}

// ---- checkpoints -------------------------------------------------------------------
// File layout (little endian):
//   magic "PRBCKPT1" | u32 version (1) | u32 flags (bit 0: average sums present)
//   u64 flop | u64 river roots | u64 upper regret floats
//   u64 FNV-1a 64 hash of everything after this header
//   f32 river regrets [roots][26][256] | f32 upper regrets [upper]
//   if flags & 1: f32 river average sums [roots][26][256] | f32 upper average sums [upper]
// Tables are not stored: they follow from the flop and are rebuilt on the device.
namespace {
struct CkptHeader {
    char magic[8];
    uint32_t version, flags;
    uint64_t flop, rivers, upper, hash;
};
uint64_t fnv1a(const void *p, size_t n, uint64_t h) {
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < n; i++) h = (h ^ c[i]) * 1099511628211ull;
    return h;
}
}  // namespace

int pr_game_save(void *game, const char *path) {
    Game *g = (Game *)game;
    if (!g || !path) return 2;
    if (int st = g->dt_pull()) return st;
    const size_t nr = g->river_board.size() * 26 * 256, nu = g->regrets.size();
    std::vector<float> river(nr), river_avg;
    if (pr_get_regrets(g->builder, river.data())) return 1;
    if (g->avg_on) {
        river_avg.resize(nr);
        if (pr_get_average(g->builder, river_avg.data())) return 1;
    }
    CkptHeader hd{};
    memcpy(hd.magic, "PRBCKPT1", 8);
    hd.version = 1;
    hd.flags = g->avg_on ? 1u : 0u;
    hd.flop = g->flop;
    hd.rivers = g->river_board.size();
    hd.upper = nu;
    uint64_t h = 1469598103934665603ull;
    h = fnv1a(river.data(), nr * 4, h);
    h = fnv1a(g->regrets.data(), nu * 4, h);
    if (g->avg_on) {
        h = fnv1a(river_avg.data(), nr * 4, h);
        h = fnv1a(g->avg_upper.data(), nu * 4, h);
    }
    hd.hash = h;
    FILE *f = fopen(path, "wb");
    if (!f) return 2;
    bool ok = fwrite(&hd, sizeof(hd), 1, f) == 1 && fwrite(river.data(), 4, nr, f) == nr &&
              fwrite(g->regrets.data(), 4, nu, f) == nu;
    if (ok && g->avg_on)
        ok = fwrite(river_avg.data(), 4, nr, f) == nr && fwrite(g->avg_upper.data(), 4, nu, f) == nu;
    ok = (fclose(f) == 0) && ok;
    return ok ? 0 : 1;
}

int pr_game_load(void *game, const char *path) {
    Game *g = (Game *)game;
    if (!g || !path) return 2;
    FILE *f = fopen(path, "rb");
    if (!f) return 2;
    CkptHeader hd{};
    const size_t nr = g->river_board.size() * 26 * 256, nu = g->regrets.size();
    bool ok = fread(&hd, sizeof(hd), 1, f) == 1 && memcmp(hd.magic, "PRBCKPT1", 8) == 0 && hd.version == 1 &&
              hd.flop == g->flop && hd.rivers == g->river_board.size() && hd.upper == nu;
    std::vector<float> river(nr), upper(nu), river_avg, upper_avg;
    ok = ok && fread(river.data(), 4, nr, f) == nr && fread(upper.data(), 4, nu, f) == nu;
    if (ok && (hd.flags & 1)) {
        river_avg.resize(nr);
        upper_avg.resize(nu);
        ok = fread(river_avg.data(), 4, nr, f) == nr && fread(upper_avg.data(), 4, nu, f) == nu;
    }
    fclose(f);
    if (!ok) return 3;
    uint64_t h = 1469598103934665603ull;
    h = fnv1a(river.data(), nr * 4, h);
    h = fnv1a(upper.data(), nu * 4, h);
    if (hd.flags & 1) {
        h = fnv1a(river_avg.data(), nr * 4, h);
        h = fnv1a(upper_avg.data(), nu * 4, h);
    }
    if (h != hd.hash) return 3;  // corrupted file
    if (g->dt_pull()) return 1;
    if (pr_set_regrets(g->builder, river.data())) return 1;
    g->regrets = upper;
    if (hd.flags & 1) {
        if (pr_game_enable_average(g)) return 1;
        if (pr_set_average(g->builder, river_avg.data())) return 1;
        g->avg_upper = upper_avg;
    }
    g->dev_stale = true;
    return 0;
}

int pr_game_get_average(void *game, float *upper, float *river) {
    Game *g = (Game *)game;
    if (!g || !g->avg_on) return 2;
    if (int st = g->dt_pull()) return st;
    if (upper) memcpy(upper, g->avg_upper.data(), g->avg_upper.size() * sizeof(float));
    if (river) return pr_get_average(g->builder, river);
    return 0;
}

}  // extern "C"
