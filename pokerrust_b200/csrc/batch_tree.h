// Bet trees of general river subgames (no reference counterpart: the reference solves only
// the fixed limit tree of src/cuda/builder.cu). Host code, shared by the batch solver and
// its C ABI.
//
// Rules. Player 0 acts first. Both players have put pot/2 into the pot before the river
// and have `stack` chips behind (0 after an all-in: both check to the showdown). `sizes`
// enables bets of 0.5 pot (bit 0), 1 pot (bit 1) and all-in (bit 2); at most `max_raises`
// bets and raises happen on the river.
//  * Not facing a bet: check, or bet each enabled size. A fractional bet is
//    frac x (pot + both players' river chips), capped at the player's remaining stack;
//    all-in is the remaining stack. Amounts that coincide with an earlier option are dropped.
//    Check by player 0 gives the turn to player 1; check behind (player 1) is a showdown.
//  * Facing a bet of `to_call`: fold, call (a showdown), or raise while raises remain and
//    the player has more than `to_call` behind. A fractional raise puts in
//    to_call + frac x (pot after calling), capped at the remaining stack.
//  * Payoffs are chips won from the opponent: a fold loses pot/2 + the folder's river chips;
//    a showdown moves pot/2 + the (equal) river chips from loser to winner, ties move nothing.
// Nodes are stored in pre-order. Edges (one per child of a decision node) are numbered in
// the order of their parents, children in action order.
#pragma once
#include <stdint.h>

#include <cmath>
#include <vector>

namespace prb {

enum : uint8_t { kBDecision = 0, kBFold = 1, kBShowdown = 2 };

constexpr int kBMaxDepth = 8;     // root = depth 0
constexpr int kBMaxNodes = 128;
constexpr int kBMaxLeaves = 64;

struct BNode {
    uint8_t kind;      // kBDecision, kBFold, kBShowdown
    uint8_t actor;     // decision: player to act; fold: the player who folded
    uint8_t nchild;    // decision nodes
    uint8_t depth;
    uint16_t parent;   // 0xFFFF at the root
    uint16_t in_edge;  // edge from the parent (0xFFFF at the root)
    uint16_t edge;     // decision: first out-edge; leaf: leaf index
    uint16_t pad;
    float stake;       // fold: pot/2 + folder's river chips; showdown: pot/2 + river chips
};
static_assert(sizeof(BNode) == 16, "BNode is 16 bytes");

struct BTree {
    std::vector<BNode> nodes;
    std::vector<uint8_t> edge_owner;  // acting player of each edge's parent
    int num_edges = 0, num_leaves = 0, depth = 0;
};

// Builds the tree of one subgame; false if it exceeds the limits above or the spec is bad.
inline bool build_bet_tree(float pot, float stack, uint32_t sizes, int max_raises, BTree *t) {
    t->nodes.clear();
    t->edge_owner.clear();
    t->num_edges = t->num_leaves = t->depth = 0;
    if (!(pot > 0.0f) || !(stack >= 0.0f) || !std::isfinite(pot) || !std::isfinite(stack) || (sizes & 7u) == 0 ||
        (sizes & ~7u) || max_raises < 1)
        return false;
    struct St {
        float c[2];    // river chips of each player
        int actor, raises;
    };
    const float fracs[3] = {0.5f, 1.0f, 0.0f};
    bool ok = true;
    // recursive pre-order construction
    struct Rec {
        BTree *t;
        float pot, stack;
        uint32_t sizes;
        int max_raises;
        const float *fracs;
        bool *ok;
        int add(uint8_t kind, uint8_t actor, int parent, int depth, float stake) {
            if ((int)t->nodes.size() >= kBMaxNodes || depth >= kBMaxDepth) {
                *ok = false;
                return -1;
            }
            BNode n{};
            n.kind = kind;
            n.actor = actor;
            n.depth = (uint8_t)depth;
            n.parent = parent < 0 ? 0xFFFF : (uint16_t)parent;
            n.in_edge = 0xFFFF;
            n.stake = stake;
            t->nodes.push_back(n);
            if (depth > t->depth) t->depth = depth;
            return (int)t->nodes.size() - 1;
        }
        void visit(int self, const St &s, int depth) {
            const int p = s.actor, o = 1 - p;
            const float behind = stack - s.c[p];
            const float to_call = s.c[o] - s.c[p];
            const float in_pot = pot + s.c[0] + s.c[1];
            struct Act {
                int kind;  // 0 check, 1 bet/raise (to amount), 2 fold, 3 call
                float put;
            };
            Act acts[8];
            int na = 0;
            if (to_call <= 0.0f) {
                acts[na++] = {0, 0.0f};
                if (s.raises < max_raises && behind > 0.0f) {
                    for (int k = 0; k < 3; k++) {
                        if (!((sizes >> k) & 1u)) continue;
                        float amt = k == 2 ? behind : fracs[k] * in_pot;
                        if (amt > behind) amt = behind;
                        bool dup = false;
                        for (int j = 0; j < na; j++) dup |= acts[j].kind == 1 && acts[j].put == amt;
                        if (!dup && amt > 0.0f) acts[na++] = {1, amt};
                    }
                }
            } else {
                acts[na++] = {2, 0.0f};
                acts[na++] = {3, to_call};
                if (s.raises < max_raises && behind > to_call) {
                    for (int k = 0; k < 3; k++) {
                        if (!((sizes >> k) & 1u)) continue;
                        float amt = k == 2 ? behind : to_call + fracs[k] * (in_pot + to_call);
                        if (amt > behind) amt = behind;
                        bool dup = false;
                        for (int j = 0; j < na; j++) dup |= acts[j].kind == 1 && acts[j].put == amt;
                        if (!dup && amt > to_call) acts[na++] = {1, amt};
                    }
                }
            }
            BTree *tr = t;
            tr->nodes[self].nchild = (uint8_t)na;
            tr->nodes[self].edge = (uint16_t)tr->num_edges;
            const int first_edge = tr->num_edges;
            tr->num_edges += na;
            for (int a = 0; a < na; a++) tr->edge_owner.push_back((uint8_t)p);
            for (int a = 0; a < na && *ok; a++) {
                int child = -1;
                St n = s;
                switch (acts[a].kind) {
                    case 0:  // check
                        if (p == 0) {
                            n.actor = 1;
                            child = add(kBDecision, 1, self, depth + 1, 0.0f);
                            if (child >= 0) {
                                tr->nodes[child].in_edge = (uint16_t)(first_edge + a);
                                visit(child, n, depth + 1);
                            }
                        } else {
                            child = add(kBShowdown, 0, self, depth + 1, 0.5f * pot + s.c[0]);
                            if (child >= 0) {
                                tr->nodes[child].in_edge = (uint16_t)(first_edge + a);
                                tr->nodes[child].edge = (uint16_t)tr->num_leaves++;
                            }
                        }
                        break;
                    case 1:  // bet or raise
                        n.c[p] += acts[a].put;
                        n.actor = o;
                        n.raises = s.raises + 1;
                        child = add(kBDecision, (uint8_t)o, self, depth + 1, 0.0f);
                        if (child >= 0) {
                            tr->nodes[child].in_edge = (uint16_t)(first_edge + a);
                            visit(child, n, depth + 1);
                        }
                        break;
                    case 2:  // fold
                        child = add(kBFold, (uint8_t)p, self, depth + 1, 0.5f * pot + s.c[p]);
                        if (child >= 0) {
                            tr->nodes[child].in_edge = (uint16_t)(first_edge + a);
                            tr->nodes[child].edge = (uint16_t)tr->num_leaves++;
                        }
                        break;
                    case 3:  // call
                        child = add(kBShowdown, 0, self, depth + 1, 0.5f * pot + s.c[o]);
                        if (child >= 0) {
                            tr->nodes[child].in_edge = (uint16_t)(first_edge + a);
                            tr->nodes[child].edge = (uint16_t)tr->num_leaves++;
                        }
                        break;
                }
            }
        }
    };
    Rec r{t, pot, stack, sizes & 7u, max_raises, fracs, &ok};
    const int root = r.add(kBDecision, 0, -1, 0, 0.0f);
    St s0{{0.0f, 0.0f}, 0, 0};
    r.visit(root, s0, 0);
    if (t->num_leaves > kBMaxLeaves) ok = false;
    return ok;
}

}  // namespace prb
