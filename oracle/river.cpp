// Oracle (test infrastructure only): the river subtree and its CPU CFR traversal.
//
// The tree is the one src/cuda/builder.cu:8-138 builds (states numbered in build order,
// edges numbered when add_transition runs, i.e. after the child's subtree); it equals the
// tree of src/builder.rs:34-79 + src/state.rs:66-217 below a River node. The traversal
// restates the CPU branch of src/state.rs:377-433 (48 rivers, masking, apply_updates) and
// the recursive src/state.rs:219-296 with AbstractStrategy (src/strategy.rs:86-153),
// evaluate_fold (src/state.rs:456-492) and evaluate_showdown (src/state.rs:494-569).
#include "oracle_internal.h"

#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

namespace {

// Order in which a river pass visits the 48 river cards: ascending (0, the order of
// state.rs:377-433) or descending (1). Both give the same sum; the descending order changes
// only the f32 rounding of the sums over rivers, which lets a test measure how far the game's
// trajectory depends on summation order alone. Set by or_set_river_order.
std::atomic<int> g_river_descending{0};

enum Term { NonTerminal = 0, SBWins = 1, BBWins = 2, Showdown = 3, River = 4 };
enum Act { Fold = 0, Check = 1, Call = 2, Raise = 3, DealRiver = 4 };
enum Player { Small = 0, Big = 1 };

struct RNode {
    int terminal, action, actor, parent;
    float sb, bb;  // offsets from the root bet
    bool dealt;    // five board cards (after DealRiver)
    int nchild;
    int child[3];
    int edge[3];
};

struct RTree {
    RNode n[OR_RIVER_STATES];
    int nstates = 0, nedges = 0;

    int possible(const RNode &s, int raises, int *out) {
        switch (s.action) {
            case Fold: return 0;
            case Check: out[0] = Call; out[1] = Raise; return 2;
            case Call:
                if (!s.dealt) { out[0] = DealRiver; return 1; }
                return 0;
            case Raise:
                out[0] = Fold; out[1] = Call;
                if (raises < 4) { out[2] = Raise; return 3; }
                return 2;
            case DealRiver: out[0] = Check; out[1] = Raise; return 2;
        }
        return 0;
    }

    RNode get_action(const RNode &s, int action) {
        RNode t = s;
        t.actor = s.actor == Small ? Big : Small;
        t.action = action;
        t.nchild = 0;
        float other = s.actor == Small ? s.bb : s.sb;
        switch (action) {
            case Fold: t.terminal = s.actor == Small ? BBWins : SBWins; break;
            case Check: t.terminal = NonTerminal; break;
            case Call:
                t.terminal = s.dealt ? Showdown : River;
                t.sb = other;
                t.bb = other;
                break;
            case Raise:
                t.terminal = NonTerminal;
                if (s.actor == Small) t.sb = s.bb + 2.0f;
                else t.bb = s.sb + 2.0f;
                break;
            case DealRiver:
                t.actor = Small;
                t.terminal = NonTerminal;
                t.dealt = true;
                break;
        }
        return t;
    }

    void build(int s, int raises) {
        int acts[3];
        int na = possible(n[s], raises, acts);
        for (int i = 0; i < na; i++) {
            int nr = acts[i] == Raise ? raises + 1 : 0;
            int c = nstates++;
            n[c] = get_action(n[s], acts[i]);
            n[c].parent = s;
            build(c, nr);
            int k = n[s].nchild++;
            n[s].child[k] = c;
            n[s].edge[k] = n[s].terminal == NonTerminal ? nedges++ : -1;
        }
    }

    RTree() {
        RNode r{};
        r.terminal = River;
        r.action = Call;
        r.actor = Small;
        r.parent = -1;
        r.sb = r.bb = 0.0f;
        r.dealt = false;
        n[0] = r;
        nstates = 1;
        build(0, 0);
    }
};

const RTree &tree() {
    static RTree t;
    return t;
}

template <typename T>
using Vec = std::vector<T>;

struct Board {
    const uint16_t *eval;   // packed (inverse) eval of this board
    const uint16_t *abstr;  // bucket of each hand
    uint16_t sorted[OR_HANDS];  // vectorized_eval order: hand | 2048 flag
};

template <typename T>
struct RiverEval {
    const uint64_t *card_order;
    const RTree &tr;
    float bet;
    const float *regrets;  // [26][256]
    float *updates;        // [26][256] or null
    int upd;
    bool exploit;
    float *avg = nullptr;  // [26][256] average-strategy sums or null

    // strategy.rs:129-150 (get_strategy of AbstractStrategy)
    void strategy(const RNode &s, const Board &b, Vec<T> *out) {
        int nk = s.nchild;
        T sum[OR_BUCKETS];
        for (int i = 0; i < OR_BUCKETS; i++) {
            sum[i] = T(0);
            for (int j = 0; j < nk; j++) sum[i] += T(regrets[s.edge[j] * OR_BUCKETS + i]);
        }
        for (int k = 0; k < nk; k++) out[k].assign(OR_HANDS, T(0));
        for (int i = 0; i < OR_HANDS; i++) {
            int a = b.abstr[i];
            for (int k = 0; k < nk; k++) {
                if (sum[a] <= T(1e-4f)) out[k][i] = T(1) / T(nk);
                else out[k][i] = T(regrets[s.edge[k] * OR_BUCKETS + a]) / sum[a];
            }
        }
    }

    Vec<T> fold(const Vec<T> &opp, const RNode &s, int folding) {
        Vec<T> result(OR_HANDS, T(0));
        T range_sum = 0;
        T coll[52] = {};
        for (int i = 0; i < OR_HANDS; i++) {
            range_sum += opp[i];
            int c1, c2;
            or_separate(card_order[i], &c1, &c2);
            coll[c1] += opp[i];
            coll[c2] += opp[i];
        }
        for (int i = 0; i < OR_HANDS; i++) {
            result[i] = range_sum + opp[i];
            int c1, c2;
            or_separate(card_order[i], &c1, &c2);
            result[i] -= coll[c1];
            result[i] -= coll[c2];
        }
        T b = T(folding == Small ? bet + s.sb : bet + s.bb);
        T m = b * (upd == folding ? T(-1) : T(1));
        for (auto &x : result) x *= m;
        return result;
    }

    Vec<T> showdown(const Vec<T> &opp, const RNode &s, const Board &bd) {
        Vec<T> result(OR_HANDS, T(0));
        T b = T(bet + s.sb);
        // group boundaries from the flags
        std::vector<int> starts;
        for (int i = 0; i < OR_HANDS; i++)
            if (i == 0 || (bd.sorted[i] & 2048)) starts.push_back(i);
        starts.push_back(OR_HANDS);
        int ng = (int)starts.size() - 1;
        {
            T coll[52] = {};
            T cumulative = 0;
            for (int g = 0; g < ng; g++) {
                T cur = 0;
                T cur_coll[52] = {};
                for (int p = starts[g]; p < starts[g + 1]; p++) {
                    int idx = bd.sorted[p] & 2047;
                    int c[2];
                    or_separate(card_order[idx], &c[0], &c[1]);
                    result[idx] += cumulative;
                    cur += opp[idx];
                    for (int k = 0; k < 2; k++) {
                        result[idx] -= coll[c[k]];
                        cur_coll[c[k]] += opp[idx];
                    }
                }
                cumulative += cur;
                for (int i = 0; i < 52; i++) coll[i] += cur_coll[i];
            }
        }
        {
            T coll[52] = {};
            T cumulative = 0;
            for (int g = ng - 1; g >= 0; g--) {
                T cur = 0;
                T cur_coll[52] = {};
                for (int p = starts[g]; p < starts[g + 1]; p++) {
                    int idx = bd.sorted[p] & 2047;
                    int c[2];
                    or_separate(card_order[idx], &c[0], &c[1]);
                    result[idx] -= cumulative;
                    cur += opp[idx];
                    for (int k = 0; k < 2; k++) {
                        result[idx] += coll[c[k]];
                        cur_coll[c[k]] += opp[idx];
                    }
                }
                cumulative += cur;
                for (int i = 0; i < 52; i++) coll[i] += cur_coll[i];
            }
        }
        for (auto &x : result) x *= b;
        return result;
    }

    // state.rs:219-296 for the river part of the tree.
    Vec<T> eval(int si, const Vec<T> &sb, const Vec<T> &bbr, const Board &bd, int *err) {
        const RNode &s = tr.n[si];
        const Vec<T> &opp = upd == Small ? bbr : sb;
        switch (s.terminal) {
            case NonTerminal: {
                bool br_here = (upd == s.actor) && exploit;
                Vec<T> avg(OR_HANDS, br_here ? -std::numeric_limits<T>::infinity() : T(0));
                Vec<T> strat[3];
                strategy(s, bd, strat);
                if (this->avg && s.actor == upd && !exploit) {
                    // average-strategy sums: the updater's reach into the node times the
                    // action probability, summed into the hand's bucket (not in the reference)
                    const Vec<T> &mine = upd == Small ? sb : bbr;
                    for (int i = 0; i < OR_HANDS; i++) {
                        int a = bd.abstr[i];
                        for (int k = 0; k < s.nchild; k++)
                            this->avg[s.edge[k] * OR_BUCKETS + a] += float(mine[i] * strat[k][i]);
                    }
                }
                Vec<T> results[3];
                for (int k = 0; k < s.nchild; k++) {
                    const Vec<T> &prob = strat[k];
                    Vec<T> u;
                    if (s.actor == Small) {
                        Vec<T> r(OR_HANDS);
                        for (int i = 0; i < OR_HANDS; i++) r[i] = sb[i] * prob[i];
                        u = eval(s.child[k], r, bbr, bd, err);
                    } else {
                        Vec<T> r(OR_HANDS);
                        for (int i = 0; i < OR_HANDS; i++) r[i] = bbr[i] * prob[i];
                        u = eval(s.child[k], sb, r, bd, err);
                    }
                    if (upd == s.actor) {
                        if (!exploit) {
                            for (int i = 0; i < OR_HANDS; i++) avg[i] += u[i] * prob[i];
                            results[k] = std::move(u);
                        } else {
                            for (int i = 0; i < OR_HANDS; i++) avg[i] = std::fmax(avg[i], u[i]);
                        }
                    } else {
                        for (int i = 0; i < OR_HANDS; i++) avg[i] += u[i];
                    }
                }
                if (s.actor == upd && !exploit && updates) {
                    // update_add (strategy.rs:118-127): i outer, action inner
                    for (int i = 0; i < OR_HANDS; i++) {
                        int a = bd.abstr[i];
                        if (a >= OR_BUCKETS) { *err = 1; continue; }  // strategy.rs:122 assert
                        for (int k = 0; k < s.nchild; k++)
                            updates[s.edge[k] * OR_BUCKETS + a] += float(results[k][i] - avg[i]);
                    }
                }
                return avg;
            }
            case Showdown: return showdown(opp, s, bd);
            case SBWins: return fold(opp, s, Big);
            case BBWins: return fold(opp, s, Small);
            default: *err = 2; return Vec<T>(OR_HANDS, T(0));
        }
    }
};

// state.rs:377-433 (CPU branch of the River node) for one subgame.
template <typename T>
int river_one(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, uint64_t board4,
              float bet, const T *opp_in, float *regrets, const float *regrets_ro, int player,
              bool exploit, T *out, const T *own_in = nullptr, float *avg = nullptr) {
    static thread_local uint64_t card_order[OR_HANDS];
    static thread_local bool init = false;
    if (!init) { or_card_order(card_order); init = true; }
    const RTree &tr = tree();
    std::vector<float> updates(OR_RIVER_EDGES * OR_BUCKETS, 0.0f);
    RiverEval<T> ev{card_order, tr, bet, regrets ? regrets : regrets_ro,
                    (regrets && !exploit) ? updates.data() : nullptr, player, exploit, avg};
    Vec<T> total(OR_HANDS, T(0));
    Vec<T> own(OR_HANDS, T(1));
    int count = 0, err = 0;
    Board bd;
    const bool descending = g_river_descending.load(std::memory_order_relaxed) != 0;
    for (int j = 0; j < 52; j++) {
        const int rc = descending ? 51 - j : j;
        uint64_t rb = 1ull << rc;
        if (rb & board4) continue;
        count++;
        uint64_t cards = board4 | rb;
        int slot = (int)or_colex_index(cards ^ flop);
        bd.eval = eval + (size_t)slot * OR_EVAL_LEN;
        bd.abstr = abstr + (size_t)slot * OR_HANDS;
        for (int h = 0; h < OR_HANDS; h++) {
            int pos = bd.eval[h] & 2047;
            bd.sorted[pos] = (uint16_t)h;
        }
        for (int p = 0; p < OR_HANDS; p++) bd.sorted[p] |= (bd.eval[p] & 2048);
        Vec<T> opp(OR_HANDS), mine(OR_HANDS);
        for (int i = 0; i < OR_HANDS; i++) {
            bool blocked = (card_order[i] & cards) != 0;
            opp[i] = blocked ? T(0) : opp_in[i];
            mine[i] = blocked ? T(0) : (own_in ? own_in[i] : own[i]);
        }
        // node 1 is the DealRiver child of the River root
        Vec<T> res = player == Small ? ev.eval(1, mine, opp, bd, &err) : ev.eval(1, opp, mine, bd, &err);
        for (int i = 0; i < OR_HANDS; i++)
            if (card_order[i] & cards) res[i] = T(0);
        for (int i = 0; i < OR_HANDS; i++) total[i] += res[i];
    }
    // apply_updates (strategy.rs:152-160) on the updating player's nodes
    if (regrets && !exploit) {
        for (int s = 0; s < tr.nstates; s++) {
            const RNode &n = tr.n[s];
            if (n.terminal != NonTerminal || n.actor != player) continue;
            for (int k = 0; k < n.nchild; k++) {
                float *r = regrets + n.edge[k] * OR_BUCKETS;
                const float *u = updates.data() + n.edge[k] * OR_BUCKETS;
                for (int i = 0; i < OR_BUCKETS; i++) {
                    r[i] += u[i];
                    r[i] = std::fmax(r[i], 0.0f);
                }
            }
        }
    }
    if (count != 48) err = 3;  // state.rs:430
    T scale = T(1) / T(48);
    for (int i = 0; i < OR_HANDS; i++) out[i] = total[i] * scale;
    return err;
}

}  // namespace

int or_river_one_f32(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, uint64_t board4,
                     float bet, const float *opp, float *regrets, int player, bool exploit,
                     float *out) {
    return river_one<float>(flop, eval, abstr, board4, bet, opp, regrets, nullptr, player, exploit,
                            out);
}

int or_river_one_f32_avg(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, uint64_t board4,
                         float bet, const float *opp, const float *own, float *regrets, float *avg,
                         int player, float *out) {
    return river_one<float>(flop, eval, abstr, board4, bet, opp, regrets, nullptr, player, false, out,
                            own, avg);
}

int or_river_one_f64(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, uint64_t board4,
                     float bet, const double *opp, const float *regrets, int player, double *out) {
    return river_one<double>(flop, eval, abstr, board4, bet, opp, nullptr, regrets, player, true,
                             out);
}

extern "C" void or_set_river_order(int descending) { g_river_descending.store(descending ? 1 : 0); }

extern "C" void or_river_tree(int *terminal, int *actor, int *parent, float *sb_off,
                              float *bb_off, int *nchild, int *child, int *edge) {
    const RTree &t = tree();
    for (int s = 0; s < t.nstates; s++) {
        terminal[s] = t.n[s].terminal;
        actor[s] = t.n[s].actor;
        parent[s] = t.n[s].parent;
        sb_off[s] = t.n[s].sb;
        bb_off[s] = t.n[s].bb;
        nchild[s] = t.n[s].nchild;
        for (int k = 0; k < 3; k++) {
            child[s * 3 + k] = k < t.n[s].nchild ? t.n[s].child[k] : -1;
            edge[s * 3 + k] = k < t.n[s].nchild ? t.n[s].edge[k] : -1;
        }
    }
}

extern "C" int or_river_batch(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, int n,
                              const uint64_t *board4, const float *bet, const float *opp_range,
                              float *regrets, int player, int calc_exploit, float *result,
                              int nthreads) {
    std::atomic_int err(0);
    or_parallel_for(n, nthreads, [&](int i) {
        int e = river_one<float>(flop, eval, abstr, board4[i], bet[i], opp_range + (size_t)i * OR_HANDS,
                                 regrets + (size_t)i * OR_RIVER_EDGES * OR_BUCKETS, nullptr, player,
                                 calc_exploit != 0, result + (size_t)i * OR_HANDS);
        if (e) err = e;
    });
    return err;
}

extern "C" int or_river_batch_avg(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, int n,
                                  const uint64_t *board4, const float *bet, const float *opp_range,
                                  const float *own_range, float *regrets, float *avg, int player,
                                  float *result, int nthreads) {
    std::atomic_int err(0);
    or_parallel_for(n, nthreads, [&](int i) {
        int e = river_one<float>(flop, eval, abstr, board4[i], bet[i], opp_range + (size_t)i * OR_HANDS,
                                 regrets + (size_t)i * OR_RIVER_EDGES * OR_BUCKETS, nullptr, player, false,
                                 result + (size_t)i * OR_HANDS, own_range + (size_t)i * OR_HANDS,
                                 avg + (size_t)i * OR_RIVER_EDGES * OR_BUCKETS);
        if (e) err = e;
    });
    return err;
}

extern "C" int or_river_br_f64(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, int n,
                               const uint64_t *board4, const double *bet, const double *opp_range,
                               const float *regrets, int player, double *result, int nthreads) {
    std::atomic_int err(0);
    or_parallel_for(n, nthreads, [&](int i) {
        int e = river_one<double>(flop, eval, abstr, board4[i], (float)bet[i],
                                  opp_range + (size_t)i * OR_HANDS, nullptr,
                                  regrets + (size_t)i * OR_RIVER_EDGES * OR_BUCKETS, player, true,
                                  result + (size_t)i * OR_HANDS);
        if (e) err = e;
    });
    return err;
}
