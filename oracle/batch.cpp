// Oracle (test infrastructure only): general river subgames, restated on the CPU for the
// batched solver's parity tests. The reference has no general trees (its river tree is the
// fixed limit tree of src/cuda/builder.cu:8-138); the rules restated here are the batch
// solver's own, and the CFR arithmetic is the reference's (strategy.rs:138-156: regret
// matching with the sum <= 1e-4 cutoff, regrets clipped at zero after each update;
// state.rs:436-569: showdown and fold values with card removal), per hand instead of per
// bucket.
//
// Tree rules: player 0 acts first; both players have pot/2 in and `stack` behind. Not facing
// a bet: check, or bet 0.5 pot / 1 pot / all-in (the enabled sizes, capped at the stack,
// repeated amounts dropped); player 0's check passes the action, player 1's check ends in a
// showdown. Facing a bet: fold, call (showdown), or raise to-call + fraction x (pot after the
// call) / all-in while raises remain and the player has more than the call behind. At most
// max_raises bets + raises. A fold loses pot/2 + the folder's river chips; a showdown moves
// pot/2 + the river chips from the worse hand to the better one.
//
// Leaf values are computed pairwise over all opponent hands (O(n^2)), in double precision,
// then rounded to the pass's precision.
#include <math.h>
#include <string.h>

#include <memory>
#include <vector>

#include "oracle_internal.h"

namespace {

struct Node {
    int kind = 0;    // 0 decision, 1 fold, 2 showdown
    int actor = 0;   // decision: to act; fold: folder
    float stake = 0;
    std::vector<std::unique_ptr<Node>> kids;
};

struct Spec {
    float pot, stack;
    uint32_t sizes;
    int max_raises;
};

// The subtree of a betting state, children in action order. Chip amounts are single
// precision, added in the order the rules state them.
std::unique_ptr<Node> grow(const Spec &sp, float c0, float c1, int actor, int raises) {
    auto n = std::make_unique<Node>();
    n->kind = 0;
    n->actor = actor;
    const float mine = actor == 0 ? c0 : c1, theirs = actor == 0 ? c1 : c0;
    const float left = sp.stack - mine;
    const float owe = theirs - mine;
    const float pot_now = sp.pot + c0 + c1;
    const float frac[2] = {0.5f, 1.0f};
    std::vector<float> amounts;  // chips this action puts in, for bets and raises
    auto push_amount = [&](float a, float floor_amt) {
        for (float b : amounts)
            if (b == a) return;
        if (a > floor_amt) amounts.push_back(a);
    };
    if (owe <= 0.0f) {
        if (actor == 0) {
            n->kids.push_back(grow(sp, c0, c1, 1, raises));  // check: player 1 to act
        } else {
            auto sd = std::make_unique<Node>();  // check behind: showdown
            sd->kind = 2;
            sd->stake = 0.5f * sp.pot + c0;
            n->kids.push_back(std::move(sd));
        }
        if (raises < sp.max_raises && left > 0.0f) {
            for (int k = 0; k < 3; k++) {
                if (!((sp.sizes >> k) & 1)) continue;
                float a = k == 2 ? left : frac[k] * pot_now;
                if (a > left) a = left;
                push_amount(a, 0.0f);
            }
        }
    } else {
        auto fold = std::make_unique<Node>();
        fold->kind = 1;
        fold->actor = actor;
        fold->stake = 0.5f * sp.pot + mine;
        n->kids.push_back(std::move(fold));
        auto call = std::make_unique<Node>();
        call->kind = 2;
        call->stake = 0.5f * sp.pot + theirs;
        n->kids.push_back(std::move(call));
        if (raises < sp.max_raises && left > owe) {
            for (int k = 0; k < 3; k++) {
                if (!((sp.sizes >> k) & 1)) continue;
                float a = k == 2 ? left : owe + frac[k] * (pot_now + owe);
                if (a > left) a = left;
                push_amount(a, owe);
            }
        }
    }
    for (float a : amounts) {
        const float n0 = actor == 0 ? c0 + a : c0;
        const float n1 = actor == 1 ? c1 + a : c1;
        n->kids.push_back(grow(sp, n0, n1, 1 - actor, raises + 1));
    }
    return n;
}

// Flattened tree in pre-order, edges numbered by parent in pre-order, leaves in pre-order.
struct Flat {
    std::vector<int> kind, actor, parent, in_edge, nchild, first_edge, leaf, depth;
    std::vector<double> stake;
    std::vector<std::vector<int>> child;  // node ids of the children
    int edges = 0, leaves = 0;
};

int flatten(const Node *n, int parent, int in_edge, int depth, Flat &f) {
    const int id = (int)f.kind.size();
    f.kind.push_back(n->kind);
    f.actor.push_back(n->actor);
    f.parent.push_back(parent);
    f.in_edge.push_back(in_edge);
    f.nchild.push_back((int)n->kids.size());
    f.first_edge.push_back(-1);
    f.leaf.push_back(-1);
    f.depth.push_back(depth);
    f.stake.push_back(n->stake);
    f.child.emplace_back();
    if (n->kind != 0) {
        f.leaf[id] = f.leaves++;
        return id;
    }
    const int e0 = f.edges;
    f.first_edge[id] = e0;
    f.edges += (int)n->kids.size();
    for (size_t k = 0; k < n->kids.size(); k++) {
        const int c = flatten(n->kids[k].get(), id, e0 + (int)k, depth + 1, f);
        f.child[id].push_back(c);
    }
    return id;
}

bool make_tree(float pot, float stack, uint32_t sizes, int max_raises, Flat &f) {
    if (!(pot > 0) || !(stack >= 0) || !(sizes & 7) || max_raises < 1) return false;
    Spec sp{pot, stack, sizes & 7u, max_raises};
    auto root = grow(sp, 0.0f, 0.0f, 0, 0);
    flatten(root.get(), -1, -1, 0, f);
    return true;
}

struct Sub {
    uint64_t board;
    Flat t;
    float pot;
    std::vector<int> live;                 // colex hands that miss the board
    std::vector<int> ca, cb;               // the two cards of each colex hand
    std::vector<uint32_t> value;           // hand value on the board, per colex hand
    std::vector<float> range[2];           // per colex hand
    std::vector<float> regret, avg;        // [edge][1326]
};

inline void cards_of(int h, int *a, int *b) { or_separate(or_pair_from_index(h), a, b); }

// Opponent weights x[o] at a leaf -> values of the updater's hands (double).
void leaf_values(const Sub &s, int node, int player, const std::vector<double> &x, std::vector<double> &out) {
    out.assign(OR_HANDS, 0.0);
    const int kind = s.t.kind[node];
    const double stake = s.t.stake[node];
    for (int h : s.live) {
        const int a = s.ca[h], b = s.cb[h];
        double acc = 0;
        for (int o : s.live) {
            const int c = s.ca[o], d = s.cb[o];
            if (a == c || a == d || b == c || b == d) continue;
            if (kind == 2) {
                if (s.value[h] > s.value[o]) acc += x[o];
                else if (s.value[h] < s.value[o]) acc -= x[o];
            } else {
                acc += x[o];
            }
        }
        if (kind == 2) out[h] = stake * acc;
        else out[h] = (s.t.actor[node] == player ? -stake : stake) * acc;
    }
}

template <typename T>
T sigma_of(const float *src, int first, int n, int k, int h, bool average) {
    T sum = T(0);
    for (int e = 0; e < n; e++) {
        const T v = T(src[(size_t)(first + e) * OR_HANDS + h]);
        sum += v > T(0) ? v : T(0);
    }
    const T cut = average ? T(0) : T(1e-4f);
    const T v = T(src[(size_t)(first + k) * OR_HANDS + h]);
    return sum <= cut ? T(1) / T(n) : (v > T(0) ? v : T(0)) / sum;
}

// One CFR half-iteration for `player` in single precision (per-hand form of
// state.rs:219-296 / strategy.rs:138-156).
void cfr_half(Sub &s, int player, bool accumulate) {
    const Flat &t = s.t;
    const int N = (int)t.kind.size();
    std::vector<std::vector<float>> po(N, std::vector<float>(OR_HANDS)), pp(N, std::vector<float>(OR_HANDS));
    // top-down reach, pre-order
    for (int i = 0; i < N; i++) {
        for (int h = 0; h < OR_HANDS; h++) {
            if (i == 0) {
                po[0][h] = s.range[1 - player][h];
                pp[0][h] = 1.0f;
                continue;
            }
            const int m = t.parent[i];
            const int k = t.in_edge[i] - t.first_edge[m];
            const float sg = sigma_of<float>(s.regret.data(), t.first_edge[m], t.nchild[m], k, h, false);
            if (t.actor[m] == player) {
                po[i][h] = po[m][h];
                pp[i][h] = pp[m][h] * sg;
                if (accumulate) s.avg[(size_t)t.in_edge[i] * OR_HANDS + h] += pp[m][h] * sg;
            } else {
                po[i][h] = po[m][h] * sg;
                pp[i][h] = pp[m][h];
            }
        }
    }
    // values, reverse pre-order (children before parents)
    std::vector<std::vector<float>> v(N, std::vector<float>(OR_HANDS, 0.0f));
    std::vector<double> x(OR_HANDS), lv;
    for (int i = N - 1; i >= 0; i--) {
        if (t.kind[i] != 0) {
            for (int h = 0; h < OR_HANDS; h++) x[h] = po[i][h];
            leaf_values(s, i, player, x, lv);
            for (int h = 0; h < OR_HANDS; h++) v[i][h] = (float)lv[h];
            continue;
        }
        const int n = t.nchild[i];
        for (int h = 0; h < OR_HANDS; h++) {
            float acc = 0.0f;
            for (int k = 0; k < n; k++) {
                const float u = v[t.child[i][k]][h];
                if (t.actor[i] == player)
                    acc += sigma_of<float>(s.regret.data(), t.first_edge[i], n, k, h, false) * u;
                else
                    acc += u;
            }
            v[i][h] = acc;
        }
        if (t.actor[i] == player) {
            for (int h = 0; h < OR_HANDS; h++)
                for (int k = 0; k < n; k++) {
                    float &r = s.regret[(size_t)(t.first_edge[i] + k) * OR_HANDS + h];
                    r = fmaxf((r + v[t.child[i][k]][h]) - v[i][h], 0.0f);
                }
        }
    }
}

// Best response (max at the player's nodes) or evaluation (strategy-weighted), double.
double br_eval(const Sub &s, int player, bool use_average, bool best, double *root) {
    const Flat &t = s.t;
    const int N = (int)t.kind.size();
    const float *src = use_average ? s.avg.data() : s.regret.data();
    std::vector<std::vector<double>> po(N, std::vector<double>(OR_HANDS));
    for (int i = 0; i < N; i++) {
        for (int h = 0; h < OR_HANDS; h++) {
            if (i == 0) {
                po[0][h] = s.range[1 - player][h];
                continue;
            }
            const int m = t.parent[i];
            const int k = t.in_edge[i] - t.first_edge[m];
            if (t.actor[m] == player) po[i][h] = po[m][h];
            else po[i][h] = po[m][h] * sigma_of<double>(src, t.first_edge[m], t.nchild[m], k, h, use_average);
        }
    }
    std::vector<std::vector<double>> v(N, std::vector<double>(OR_HANDS, 0.0));
    std::vector<double> lv;
    for (int i = N - 1; i >= 0; i--) {
        if (t.kind[i] != 0) {
            leaf_values(s, i, player, po[i], lv);
            v[i] = lv;
            continue;
        }
        const int n = t.nchild[i];
        for (int h = 0; h < OR_HANDS; h++) {
            double acc = (t.actor[i] == player && best) ? -INFINITY : 0.0;
            for (int k = 0; k < n; k++) {
                const double u = v[t.child[i][k]][h];
                if (t.actor[i] != player) acc += u;
                else if (best) acc = acc > u ? acc : u;
                else acc += sigma_of<double>(src, t.first_edge[i], n, k, h, use_average) * u;
            }
            v[i][h] = acc;
        }
    }
    double sum = 0;
    for (int h : s.live) sum += (double)s.range[player][h] * v[0][h];
    if (root)
        for (int h = 0; h < OR_HANDS; h++) root[h] = v[0][h];
    return sum;
}

}  // namespace

extern "C" {

int or_bet_tree(float pot, float stack, uint32_t sizes, int max_raises, int *kind, int *actor, int *parent,
                int *in_edge, int *nchild, float *stake, int *depth, int max_nodes, int *num_nodes, int *num_edges,
                int *num_leaves) {
    Flat f;
    if (!make_tree(pot, stack, sizes, max_raises, f)) return 2;
    const int n = (int)f.kind.size();
    *num_nodes = n;
    *num_edges = f.edges;
    *num_leaves = f.leaves;
    if (n > max_nodes) return 3;
    for (int i = 0; i < n; i++) {
        kind[i] = f.kind[i];
        actor[i] = f.actor[i];
        parent[i] = f.parent[i];
        in_edge[i] = f.in_edge[i];
        nchild[i] = f.nchild[i];
        stake[i] = (float)f.stake[i];
        depth[i] = f.depth[i];
    }
    return 0;
}

void *or_sub_new(uint64_t board, float pot, float stack, uint32_t sizes, int max_raises, const float *r0,
                 const float *r1) {
    Sub *s = new Sub();
    s->board = board;
    s->pot = pot;
    if (!make_tree(pot, stack, sizes, max_raises, s->t)) {
        delete s;
        return nullptr;
    }
    s->value.assign(OR_HANDS, 0);
    s->ca.resize(OR_HANDS);
    s->cb.resize(OR_HANDS);
    for (int h = 0; h < OR_HANDS; h++) cards_of(h, &s->ca[h], &s->cb[h]);
    s->range[0].assign(r0, r0 + OR_HANDS);
    s->range[1].assign(r1, r1 + OR_HANDS);
    for (int h = 0; h < OR_HANDS; h++) {
        const uint64_t hm = or_pair_from_index(h);
        if (hm & board) {
            s->range[0][h] = s->range[1][h] = 0.0f;
            continue;
        }
        s->live.push_back(h);
        s->value[h] = or_hand_value(hm | board);
    }
    s->regret.assign((size_t)s->t.edges * OR_HANDS, 0.0f);
    s->avg.assign((size_t)s->t.edges * OR_HANDS, 0.0f);
    return s;
}

void or_sub_free(void *s) { delete (Sub *)s; }
int or_sub_edges(void *s) { return ((Sub *)s)->t.edges; }

void or_sub_get(void *sp, int which, float *out) {
    Sub *s = (Sub *)sp;
    const std::vector<float> &v = which ? s->avg : s->regret;
    memcpy(out, v.data(), v.size() * sizeof(float));
}

void or_sub_set(void *sp, int which, const float *in) {
    Sub *s = (Sub *)sp;
    std::vector<float> &v = which ? s->avg : s->regret;
    memcpy(v.data(), in, v.size() * sizeof(float));
}

void or_sub_cfr_half(void *s, int player, int accumulate) { cfr_half(*(Sub *)s, player, accumulate != 0); }

double or_sub_best_response(void *s, int player, int use_average, double *root) {
    return br_eval(*(Sub *)s, player, use_average != 0, true, root);
}

double or_sub_value(void *s, int player, int use_average, double *root) {
    return br_eval(*(Sub *)s, player, use_average != 0, false, root);
}

// Sum over clash-free hand pairs of r0(h) r1(o).
double or_sub_joint(void *sp) {
    Sub *s = (Sub *)sp;
    double j = 0;
    for (int h : s->live) {
        const int a = s->ca[h], b = s->cb[h];
        for (int o : s->live) {
            const int c = s->ca[o], d = s->cb[o];
            if (a == c || a == d || b == c || b == d) continue;
            j += (double)s->range[0][h] * s->range[1][o];
        }
    }
    return j;
}

}  // extern "C"
