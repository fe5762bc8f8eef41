// The flop and turn streets of a fixed-flop no-limit game with general bet sizes (no
// reference counterpart: the reference's game is the limit tree of src/state.rs and
// src/builder.rs). Host code, shared by the full-game solver and its C ABI.
//
// Rules. Both players have put pot/2 into the pot before the flop and have `stack` chips
// behind. On each street player 0 acts first.
//  * Not facing a bet: check, or bet frac x (pot + both players' chips of the street) for
//    each fraction, capped at the chips behind, or all-in (the chips behind). Amounts that
//    coincide with an earlier option, and zero amounts, are dropped. A check by player 0
//    passes the action; a check by player 1 ends the street.
//  * Facing a bet of `to_call`: fold, call (ends the street), or raise while raises remain
//    and the player has more than `to_call` behind: to_call + frac x (pot after the call),
//    capped at the chips behind, or all-in. At most `max_raises` bets and raises per street.
//  * A fold loses pot/2 + the folder's chips of the street, where pot is the pot at the
//    start of the street (so pot/2 holds each player's chips of earlier streets).
//  * The end of the flop is a chance node that deals the turn: one child per card off the
//    flop, in card order, each the root of a turn street with the grown pot and the chips
//    left behind. The end of the turn is a leaf: the river (dealt by chance, 48 cards) and
//    its betting, solved as river subgames with the leaf's pot and stack.
// Nodes are stored in pre-order, chance children in card order. Edges (one per child of a
// decision node) are numbered in the pre-order of their nodes, children in action order;
// leaves in pre-order.
#pragma once
#include <stdint.h>

#include <cmath>
#include <vector>

namespace prb {

enum : uint8_t { kFDecision = 0, kFFold = 1, kFDeal = 2, kFLeaf = 3 };

constexpr int kFMaxKids = 8;      // decision children: fold, call, up to 6 bets
constexpr int kFMaxFracs = 4;

struct FNode {
    uint8_t kind;     // kFDecision, kFFold, kFDeal, kFLeaf
    uint8_t actor;    // decision: player to act; fold: the player who folded
    uint8_t nchild;   // decision: actions; deal: cards dealt (49)
    uint8_t street;   // 0 flop, 1 turn
    int32_t parent;   // -1 at the root
    int32_t in_edge;  // edge from a decision parent, -1 below a deal node and at the root
    int32_t edge;     // decision: first out-edge; leaf: leaf index; otherwise -1
    int32_t kids;     // decision and deal: offset of the children in the child list
    int32_t level;    // distance from the root
    float stake;      // fold: pot/2 + folder's chips of the street; leaf: pot at the river
    float stack;      // leaf: chips behind at the river
    uint32_t pad;
    uint64_t board;   // cards dealt so far (flop, plus the turn card below a deal node)
};
static_assert(sizeof(FNode) == 48, "FNode is 48 bytes");

struct StreetRules {
    float fracs[kFMaxFracs];
    int nfrac = 0;
    bool allin = false;
    int max_raises = 0;
};

struct FullTree {
    std::vector<FNode> nodes;
    std::vector<int32_t> kids;     // child node ids of decision and deal nodes
    std::vector<int32_t> leaves;   // node id of each leaf
    int num_edges = 0, levels = 0;
};

namespace fulltree_detail {

struct Builder {
    FullTree *t;
    uint64_t flop;
    StreetRules rules[2];
    int max_nodes;
    bool ok = true;

    int add(uint8_t kind, uint8_t actor, int parent, int level, int street, uint64_t board) {
        if ((int)t->nodes.size() >= max_nodes) {
            ok = false;
            return -1;
        }
        FNode n{};
        n.kind = kind;
        n.actor = actor;
        n.street = (uint8_t)street;
        n.parent = parent;
        n.in_edge = -1;
        n.edge = -1;
        n.kids = -1;
        n.level = level;
        n.board = board;
        t->nodes.push_back(n);
        if (level + 1 > t->levels) t->levels = level + 1;
        return (int)t->nodes.size() - 1;
    }

    // the end of a street: a deal node after the flop, a leaf after the turn
    void street_end(int self, int street, float pot, float behind, uint64_t board) {
        FNode &n = t->nodes[self];
        if (street == 1) {
            n.kind = kFLeaf;
            n.edge = (int32_t)t->leaves.size();
            n.stake = pot;
            n.stack = behind;
            t->leaves.push_back(self);
            return;
        }
        n.kind = kFDeal;
        std::vector<int> cards;
        for (int c = 0; c < 52; c++)
            if (!((flop >> c) & 1)) cards.push_back(c);
        n.nchild = (uint8_t)cards.size();
        const int off = (int)t->kids.size();
        t->nodes[self].kids = off;
        t->kids.resize(off + cards.size(), -1);
        const int level = t->nodes[self].level;
        for (size_t i = 0; i < cards.size() && ok; i++) {
            const uint64_t b = board | (1ull << cards[i]);
            const int child = add(kFDecision, 0, self, level + 1, 1, b);
            if (child < 0) return;
            t->kids[off + i] = child;
            visit(child, 1, pot, behind, 0.0f, 0.0f, 0, 0);
        }
    }

    // a decision node of `street`: pot at the street's start, chips behind at its start,
    // street chips c0 / c1, player to act, bets and raises so far
    void visit(int self, int street, float pot, float stack, float c0, float c1, int actor, int raises) {
        const StreetRules &R = rules[street];
        const uint64_t board = t->nodes[self].board;
        const float mine = actor == 0 ? c0 : c1, theirs = actor == 0 ? c1 : c0;
        const float behind = stack - mine;
        const float to_call = theirs - mine;
        const float pot_now = pot + c0 + c1;
        // actions: 0 check, 1 bet/raise putting in `put`, 2 fold, 3 call
        int kind[kFMaxKids];
        float put[kFMaxKids];
        int na = 0;
        auto add_bet = [&](float amt, float floor_amt) {
            for (int j = 0; j < na; j++)
                if (kind[j] == 1 && put[j] == amt) return;
            if (amt > floor_amt && na < kFMaxKids) {
                kind[na] = 1;
                put[na++] = amt;
            }
        };
        if (to_call <= 0.0f) {
            kind[na] = 0;
            put[na++] = 0.0f;
            if (raises < R.max_raises && behind > 0.0f) {
                for (int k = 0; k < R.nfrac; k++) add_bet(fminf(R.fracs[k] * pot_now, behind), 0.0f);
                if (R.allin) add_bet(behind, 0.0f);
            }
        } else {
            kind[na] = 2;
            put[na++] = 0.0f;
            kind[na] = 3;
            put[na++] = to_call;
            if (raises < R.max_raises && behind > to_call) {
                for (int k = 0; k < R.nfrac; k++)
                    add_bet(fminf(to_call + R.fracs[k] * (pot_now + to_call), behind), to_call);
                if (R.allin) add_bet(behind, to_call);
            }
        }
        const int first_edge = t->num_edges;
        t->num_edges += na;
        const int off = (int)t->kids.size();
        t->kids.resize(off + na, -1);
        {
            FNode &n = t->nodes[self];
            n.nchild = (uint8_t)na;
            n.edge = first_edge;
            n.kids = off;
        }
        const int level = t->nodes[self].level;
        for (int a = 0; a < na && ok; a++) {
            int child = -1;
            switch (kind[a]) {
                case 0:  // check
                    if (actor == 0) {
                        child = add(kFDecision, 1, self, level + 1, street, board);
                        if (child < 0) return;
                        t->nodes[child].in_edge = first_edge + a;
                        t->kids[off + a] = child;
                        visit(child, street, pot, stack, c0, c1, 1, raises);
                    } else {
                        child = add(kFLeaf, 0, self, level + 1, street, board);
                        if (child < 0) return;
                        t->nodes[child].in_edge = first_edge + a;
                        t->kids[off + a] = child;
                        street_end(child, street, pot + c0 + c1, stack - c0, board);
                    }
                    break;
                case 1: {  // bet or raise
                    const float n0 = actor == 0 ? c0 + put[a] : c0;
                    const float n1 = actor == 1 ? c1 + put[a] : c1;
                    child = add(kFDecision, (uint8_t)(1 - actor), self, level + 1, street, board);
                    if (child < 0) return;
                    t->nodes[child].in_edge = first_edge + a;
                    t->kids[off + a] = child;
                    visit(child, street, pot, stack, n0, n1, 1 - actor, raises + 1);
                    break;
                }
                case 2:  // fold
                    child = add(kFFold, (uint8_t)actor, self, level + 1, street, board);
                    if (child < 0) return;
                    t->nodes[child].in_edge = first_edge + a;
                    t->nodes[child].stake = 0.5f * pot + mine;
                    t->kids[off + a] = child;
                    break;
                case 3: {  // call: both have `theirs` in
                    child = add(kFLeaf, 0, self, level + 1, street, board);
                    if (child < 0) return;
                    t->nodes[child].in_edge = first_edge + a;
                    t->kids[off + a] = child;
                    street_end(child, street, pot + 2.0f * theirs, stack - theirs, board);
                    break;
                }
            }
        }
    }
};

}  // namespace fulltree_detail

// Builds the flop and turn streets; false if the spec is bad or the tree has more than
// max_nodes nodes.
inline bool build_full_tree(uint64_t flop, float pot, float stack, const StreetRules &flop_rules,
                            const StreetRules &turn_rules, int max_nodes, FullTree *t) {
    t->nodes.clear();
    t->kids.clear();
    t->leaves.clear();
    t->num_edges = t->levels = 0;
    if (__builtin_popcountll(flop) != 3 || (flop >> 52) || !(pot > 0.0f) || !(stack >= 0.0f) ||
        !std::isfinite(pot) || !std::isfinite(stack))
        return false;
    for (const StreetRules *r : {&flop_rules, &turn_rules}) {
        if (r->nfrac < 0 || r->nfrac > kFMaxFracs || r->max_raises < 0 || r->max_raises > 4) return false;
        for (int k = 0; k < r->nfrac; k++)
            if (!(r->fracs[k] > 0.0f) || !std::isfinite(r->fracs[k])) return false;
    }
    fulltree_detail::Builder b{t, flop, {flop_rules, turn_rules}, max_nodes};
    const int root = b.add(kFDecision, 0, -1, 0, 0, flop);
    b.visit(root, 0, pot, stack, 0.0f, 0.0f, 0, 0);
    return b.ok;
}

}  // namespace prb
