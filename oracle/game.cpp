// Oracle (test infrastructure only): the full fixed-flop limit game on the CPU.
//
// Restates src/builder.rs:13-79 (tree construction), src/state.rs:66-217 (get_action,
// including the suit-permutation bookkeeping of the flop, :143-182), src/state.rs:219-376
// (recursive CFR / best response over preflop, flop and turn, rayon over turn cards),
// src/strategy.rs:37-82 (RegularStrategy), src/permutation_handler.rs:7-34 (permute) and
// src/game.rs:30-143 (perform_iter and the exploitability figure). River nodes delegate to
// the river oracle (river.cpp), exactly where the reference's CPU build recurses into its
// River branch (state.rs:377-433).
#include "oracle_internal.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <set>
#include <vector>

namespace {

enum Term { NonTerminal = 0, SBWins = 1, BBWins = 2, Showdown = 3, FlopT = 4, TurnT = 5, RiverT = 6 };
enum Act { Fold, Check, Call, Raise, DealHole, DealFlop, DealTurn, DealRiver };
enum Player { Small = 0, Big = 1 };

struct GNode {
    int terminal = NonTerminal, action = DealHole;
    uint64_t cards = 0;
    float sbbet = 0, bbbet = 0;
    int actor = Small;
    std::vector<std::unique_ptr<GNode>> next;
    std::vector<std::array<int, 4>> perms;
    std::vector<std::vector<float>> regrets;  // RegularStrategy, one 1326 vector per action
    std::vector<std::vector<float>> avg;      // average-strategy sums, same shape (not in the reference)
    int river = -1;                            // index of the river root (River nodes)
};

struct Game {
    uint64_t flop;
    int nthreads;
    uint64_t card_order[OR_HANDS];
    std::vector<uint16_t> eval, coll, abstr;
    std::unique_ptr<GNode> root;
    std::vector<uint64_t> river_board;
    std::vector<float> river_bet;
    std::vector<float> river_regrets;  // [rivers][26][256]
    // Average-strategy sums (not in the reference, which keeps none): at the updater's
    // decision nodes, its reach into the node times the action probability, per hand above
    // the river and per bucket in the river subgames ([rivers][26][256]), both in f32.
    bool avg_on = false;
    std::vector<float> river_avg;
    std::vector<float> root_values[2];  // the root's values of the last CFR pass per updater

    static int popc(uint64_t x) { return __builtin_popcountll(x); }

    // builder.rs:55-79
    std::vector<int> possible(const GNode &s, int raises) {
        switch (s.action) {
            case Fold: return {};
            case Check: return {Call, Raise};
            case Call:
                switch (popc(s.cards)) {
                    case 0: return {DealFlop};
                    case 3: return {DealTurn};
                    case 4: return {};  // River: the river subtree lives in river.cpp
                    default: return {};
                }
            case Raise:
                if (raises < 4) return {Fold, Call, Raise};
                return {Fold, Call};
            case DealHole: return {Fold, Check, Raise};
            default: return {Check, Raise};  // DealFlop, DealTurn
        }
    }

    static uint64_t permute_cards(uint64_t cards, const std::array<int, 4> &p) {
        uint64_t out = 0;
        while (cards) {
            int c = __builtin_ctzll(cards);
            cards &= cards - 1;
            out |= 1ull << (13 * p[or_suit(c)] + or_rank(c));
        }
        return out;
    }

    // state.rs:66-217
    std::vector<std::unique_ptr<GNode>> get_action(const GNode &s, int action) {
        int opponent = s.actor == Small ? Big : Small;
        int fold_winner = s.actor == Small ? BBWins : SBWins;
        float other = s.actor == Small ? s.bbbet : s.sbbet;
        auto st = std::make_unique<GNode>();
        st->terminal = s.terminal;
        st->action = action;
        st->cards = s.cards;
        st->sbbet = s.sbbet;
        st->bbbet = s.bbbet;
        st->actor = opponent;
        std::vector<std::unique_ptr<GNode>> out;
        switch (action) {
            case Fold: st->terminal = fold_winner; break;
            case Check:
                st->terminal = NonTerminal;
                st->sbbet = s.bbbet;
                break;
            case Call:
                st->sbbet = other;
                st->bbbet = other;
                switch (popc(s.cards)) {
                    case 0: st->terminal = FlopT; break;
                    case 3: st->terminal = TurnT; break;
                    case 4:
                        st->terminal = RiverT;
                        st->river = (int)river_board.size();
                        river_board.push_back(s.cards);
                        river_bet.push_back(other);
                        break;
                    default: st->terminal = Showdown; break;
                }
                break;
            case Raise: {
                float amount = popc(s.cards) < 4 ? 1.0f : 2.0f;
                st->terminal = NonTerminal;
                if (s.actor == Small) st->sbbet = s.bbbet + amount;
                else st->bbbet = s.sbbet + amount;
                break;
            }
            case DealFlop: {
                // one fixed flop; permutations of [C,H,S,D] in itertools order that map it to
                // a flop not seen yet (state.rs:146-172)
                std::set<uint64_t> seen;
                std::array<int, 4> p = {0, 1, 2, 3};
                do {
                    uint64_t img = permute_cards(flop, p);
                    if (seen.insert(img).second) st->perms.push_back(p);
                } while (std::next_permutation(p.begin(), p.end()));
                st->terminal = NonTerminal;
                st->cards = flop;
                st->actor = Small;
                out.push_back(std::move(st));
                return out;
            }
            case DealTurn:
                for (int c = 0; c < 52; c++) {
                    uint64_t t = 1ull << c;
                    if (t & s.cards) continue;
                    auto n = std::make_unique<GNode>();
                    n->terminal = NonTerminal;
                    n->action = DealTurn;
                    n->cards = s.cards | t;
                    n->sbbet = s.sbbet;
                    n->bbbet = s.bbbet;
                    n->actor = Small;
                    out.push_back(std::move(n));
                }
                return out;
        }
        out.push_back(std::move(st));
        return out;
    }

    // builder.rs:34-53
    void build(GNode &s, int raises) {
        for (int action : possible(s, raises)) {
            int nr = action == Raise ? raises + 1
                     : (action == DealHole || action == DealFlop || action == DealTurn ||
                        action == DealRiver)
                         ? 0
                         : raises;
            for (auto &n : get_action(s, action)) {
                build(*n, nr);
                s.next.push_back(std::move(n));
                if (s.terminal == NonTerminal) s.regrets.emplace_back(OR_HANDS, 0.0f);
            }
        }
    }

    Game(uint64_t f, int nt) : flop(f), nthreads(nt) {
        or_card_order(card_order);
        eval.resize((size_t)OR_HANDS * OR_EVAL_LEN);
        coll.resize((size_t)OR_HANDS * OR_COLL_LEN);
        abstr.resize((size_t)OR_HANDS * OR_HANDS);
        or_pack_flop_tables(flop, eval.data(), coll.data(), abstr.data(), nthreads);
        root = std::make_unique<GNode>();
        root->terminal = NonTerminal;
        root->action = DealHole;
        root->sbbet = 0.5f;
        root->bbbet = 1.0f;
        root->actor = Small;
        build(*root, 1);
        river_regrets.assign(river_board.size() * OR_RIVER_EDGES * OR_BUCKETS, 0.0f);
    }

    // permutation_handler.rs:7-34
    template <typename T>
    std::vector<T> permute(const std::array<int, 4> &p, const std::vector<T> &v) {
        std::vector<T> r(OR_HANDS, T(0));
        for (int i = 0; i < OR_HANDS; i++) {
            uint64_t n = permute_cards(card_order[i], p);
            r[or_colex_index(n)] = v[i];
        }
        return r;
    }

    // strategy.rs:68-81
    template <typename T>
    std::vector<std::vector<T>> strategy(const GNode &s) {
        size_t n = s.regrets.size();
        std::vector<T> sum(OR_HANDS, T(0));
        for (size_t k = 0; k < n; k++)
            for (int i = 0; i < OR_HANDS; i++) sum[i] += T(s.regrets[k][i]);
        std::vector<std::vector<T>> out(n, std::vector<T>(OR_HANDS));
        for (size_t k = 0; k < n; k++)
            for (int i = 0; i < OR_HANDS; i++)
                out[k][i] = sum[i] <= T(1e-4f) ? T(1) / T(n) : T(s.regrets[k][i]) / sum[i];
        return out;
    }

    template <typename T>
    std::vector<T> fold(const GNode &s, const std::vector<T> &opp, int upd, int folding) {
        std::vector<T> result(OR_HANDS);
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
            int c1, c2;
            or_separate(card_order[i], &c1, &c2);
            result[i] = range_sum + opp[i];
            result[i] -= coll[c1];
            result[i] -= coll[c2];
        }
        T b = T(folding == Small ? s.sbbet : s.bbbet);
        T m = b * (upd == folding ? T(-1) : T(1));
        for (auto &x : result) x *= m;
        return result;
    }

    template <typename T>
    std::vector<T> river(GNode &s, const std::vector<T> &opp, const std::vector<T> &own, int upd,
                         bool exploit);

    void enable_average(GNode &s) {
        if (s.terminal == NonTerminal) s.avg.assign(s.regrets.size(), std::vector<float>(OR_HANDS, 0.0f));
        for (auto &n : s.next) enable_average(*n);
    }

    // sum of all upper-tree average sums (regrets with which = 0)
    double upper_total(const GNode &s, int which) const {
        double t = 0;
        for (const auto &v : which ? s.avg : s.regrets)
            for (float x : v) t += x;
        for (const auto &n : s.next) t += upper_total(*n, which);
        return t;
    }

    // state.rs:219-376
    template <typename T>
    std::vector<T> eval_state(GNode &s, const std::vector<T> &sb, const std::vector<T> &bb,
                              int upd, bool exploit) {
        const std::vector<T> &opp = upd == Small ? bb : sb;
        switch (s.terminal) {
            case NonTerminal: {
                std::vector<T> avg(OR_HANDS, (upd == s.actor && exploit)
                                                 ? -std::numeric_limits<T>::infinity()
                                                 : T(0));
                auto strat = strategy<T>(s);
                std::vector<std::vector<T>> results;
                for (size_t k = 0; k < s.next.size(); k++) {
                    const auto &prob = strat[k];
                    std::vector<T> r(OR_HANDS);
                    std::vector<T> u;
                    if (s.actor == Small) {
                        for (int i = 0; i < OR_HANDS; i++) r[i] = sb[i] * prob[i];
                        u = eval_state<T>(*s.next[k], r, bb, upd, exploit);
                    } else {
                        for (int i = 0; i < OR_HANDS; i++) r[i] = bb[i] * prob[i];
                        u = eval_state<T>(*s.next[k], sb, r, upd, exploit);
                    }
                    if (upd == s.actor) {
                        if (!exploit) {
                            for (int i = 0; i < OR_HANDS; i++) avg[i] += u[i] * prob[i];
                            results.push_back(std::move(u));
                        } else {
                            for (int i = 0; i < OR_HANDS; i++) avg[i] = std::fmax(avg[i], u[i]);
                        }
                    } else {
                        for (int i = 0; i < OR_HANDS; i++) avg[i] += u[i];
                    }
                }
                if (s.actor == upd && !exploit && avg_on) {
                    const std::vector<T> &own = s.actor == Small ? sb : bb;
                    for (size_t k = 0; k < s.next.size(); k++)
                        for (int i = 0; i < OR_HANDS; i++) s.avg[k][i] += float(own[i] * strat[k][i]);
                }
                if (s.actor == upd && !exploit) {
                    // RegularStrategy::update_add (strategy.rs:57-66)
                    for (size_t k = 0; k < results.size(); k++)
                        for (int i = 0; i < OR_HANDS; i++) {
                            float r = s.regrets[k][i] + float(results[k][i] - avg[i]);
                            s.regrets[k][i] = std::fmax(r, 0.0f);
                        }
                }
                return avg;
            }
            case SBWins: return fold<T>(s, opp, upd, Big);
            case BBWins: return fold<T>(s, opp, upd, Small);
            case FlopT: {
                std::vector<T> total(OR_HANDS, T(0));
                T count = 0;
                for (auto &n : s.next) {
                    std::vector<T> nsb = sb, nbb = bb;
                    for (int i = 0; i < OR_HANDS; i++)
                        if (card_order[i] & n->cards) nsb[i] = nbb[i] = T(0);
                    auto res = eval_state<T>(*n, nsb, nbb, upd, exploit);
                    for (int i = 0; i < OR_HANDS; i++)
                        if (card_order[i] & n->cards) res[i] = T(0);
                    for (auto &p : n->perms) {
                        count += T(1);
                        auto pr = permute<T>(p, res);
                        for (int i = 0; i < OR_HANDS; i++) total[i] += pr[i];
                    }
                }
                T scale = T(1) / count;
                for (auto &x : total) x *= scale;
                return total;
            }
            case TurnT: {
                std::vector<std::vector<T>> res(s.next.size());
                or_parallel_for((int)s.next.size(), nthreads, [&](int j) {
                    GNode &n = *s.next[j];
                    std::vector<T> nsb = sb, nbb = bb;
                    for (int i = 0; i < OR_HANDS; i++)
                        if (card_order[i] & n.cards) nsb[i] = nbb[i] = T(0);
                    auto r = eval_state<T>(n, nsb, nbb, upd, exploit);
                    for (int i = 0; i < OR_HANDS; i++)
                        if (card_order[i] & n.cards) r[i] = T(0);
                    res[j] = std::move(r);
                });
                std::vector<T> total(OR_HANDS, T(0));
                for (auto &v : res)
                    for (int i = 0; i < OR_HANDS; i++) total[i] += v[i];
                T scale = T(1) / T(s.next.size());
                for (auto &x : total) x *= scale;
                return total;
            }
            case RiverT: return river<T>(s, opp, upd == Small ? sb : bb, upd, exploit);
            default: return std::vector<T>(OR_HANDS, T(0));
        }
    }
};

template <>
std::vector<float> Game::river<float>(GNode &s, const std::vector<float> &opp,
                                      const std::vector<float> &own, int upd, bool exploit) {
    std::vector<float> out(OR_HANDS);
    const size_t off = (size_t)s.river * OR_RIVER_EDGES * OR_BUCKETS;
    if (avg_on && !exploit)
        or_river_one_f32_avg(flop, eval.data(), abstr.data(), s.cards, s.sbbet, opp.data(), own.data(),
                             river_regrets.data() + off, river_avg.data() + off, upd, out.data());
    else
        or_river_one_f32(flop, eval.data(), abstr.data(), s.cards, s.sbbet, opp.data(),
                         river_regrets.data() + off, upd, exploit, out.data());
    return out;
}

template <>
std::vector<double> Game::river<double>(GNode &s, const std::vector<double> &opp,
                                        const std::vector<double> &, int upd, bool exploit) {
    std::vector<double> out(OR_HANDS);
    or_river_one_f64(flop, eval.data(), abstr.data(), s.cards, s.sbbet, opp.data(),
                     river_regrets.data() + (size_t)s.river * OR_RIVER_EDGES * OR_BUCKETS, upd,
                     out.data());
    return out;
}

}  // namespace

extern "C" void *or_game_new(uint64_t flop, int nthreads) { return new Game(flop, nthreads); }
extern "C" void or_game_free(void *g) { delete (Game *)g; }
extern "C" int or_game_num_rivers(void *g) { return (int)((Game *)g)->river_board.size(); }

extern "C" void or_game_river_roots(void *g, uint64_t *board4, float *bet) {
    Game *G = (Game *)g;
    for (size_t i = 0; i < G->river_board.size(); i++) {
        board4[i] = G->river_board[i];
        bet[i] = G->river_bet[i];
    }
}

extern "C" void or_game_iterate(void *g) {
    Game *G = (Game *)g;
    std::vector<float> ones(OR_HANDS, 1.0f);
    G->root_values[0] = G->eval_state<float>(*G->root, ones, ones, Small, false);
    G->root_values[1] = G->eval_state<float>(*G->root, ones, ones, Big, false);
}

extern "C" void or_game_enable_average(void *g) {
    Game *G = (Game *)g;
    if (G->avg_on) return;
    G->enable_average(*G->root);
    G->river_avg.assign(G->river_regrets.size(), 0.0f);
    G->avg_on = true;
}

extern "C" int or_game_root_values(void *g, float *sb, float *bb) {
    Game *G = (Game *)g;
    if (G->root_values[0].size() != OR_HANDS) return 2;
    std::memcpy(sb, G->root_values[0].data(), sizeof(float) * OR_HANDS);
    std::memcpy(bb, G->root_values[1].data(), sizeof(float) * OR_HANDS);
    return 0;
}

extern "C" void or_game_totals(void *g, double *upper_regrets, double *upper_avg, double *river_regrets,
                               double *river_avg) {
    Game *G = (Game *)g;
    *upper_regrets = G->upper_total(*G->root, 0);
    *upper_avg = G->avg_on ? G->upper_total(*G->root, 1) : 0.0;
    double r = 0, a = 0;
    for (float x : G->river_regrets) r += x;
    for (float x : G->river_avg) a += x;
    *river_regrets = r;
    *river_avg = a;
}

extern "C" int or_game_river_average(void *g, float *out) {
    Game *G = (Game *)g;
    if (!G->avg_on) return 2;
    std::memcpy(out, G->river_avg.data(), G->river_avg.size() * sizeof(float));
    return 0;
}

extern "C" void or_game_exploitability(void *g, int use_f64, double *sum_sb, double *sum_bb,
                                       double *mbh) {
    Game *G = (Game *)g;
    if (use_f64) {
        std::vector<double> ones(OR_HANDS, 1.0);
        auto sb = G->eval_state<double>(*G->root, ones, ones, Small, true);
        auto bb = G->eval_state<double>(*G->root, ones, ones, Big, true);
        double s1 = 0, s2 = 0;
        for (int i = 0; i < OR_HANDS; i++) { s1 += sb[i]; s2 += bb[i]; }
        *sum_sb = s1;
        *sum_bb = s2;
        *mbh = (s1 + s2) * 1000.0 / 1326.0 / 1255.0 / 2.0;
    } else {
        std::vector<float> ones(OR_HANDS, 1.0f);
        auto sb = G->eval_state<float>(*G->root, ones, ones, Small, true);
        auto bb = G->eval_state<float>(*G->root, ones, ones, Big, true);
        float s1 = 0, s2 = 0;
        for (int i = 0; i < OR_HANDS; i++) { s1 += sb[i]; s2 += bb[i]; }
        *sum_sb = s1;
        *sum_bb = s2;
        // game.rs:175
        *mbh = (double)((s1 + s2) * 1000.0f / 1326.0f / 1255.0f / 2.0f);
    }
}

extern "C" void or_game_river_regrets(void *g, float *out) {
    Game *G = (Game *)g;
    std::memcpy(out, G->river_regrets.data(), G->river_regrets.size() * sizeof(float));
}
