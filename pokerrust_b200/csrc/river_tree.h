// The limit river subtree every river subgame of the fixed-flop game uses.
//
// It is the tree src/cuda/builder.cu:8-138 of the reference builds for one river root
// (equal to the tree of src/builder.rs:34-79 and src/state.rs:66-217 below a River node):
// River -> DealRiver -> {Check -> {Call = showdown, Raise}, Raise}, raises of +2.0 and at
// most four raises. States are numbered in build order; an edge gets its number when the
// builder's add_transition runs, i.e. after the child's whole subtree is built. The host
// builder in builder.cpp rebuilds this tree from those rules and checks it against these
// tables at start-up, so the constants below are a compiled form of the reference rules.
#pragma once

namespace prb {

constexpr int kStates = 28;
constexpr int kEdges = 26;
constexpr int kBuckets = 256;

enum : int { kNonTerminal = 0, kSBWins = 1, kBBWins = 2, kShowdown = 3, kRiver = 4 };

#define PRB_TABLE(name, type, ...)                                  \
    __host__ __device__ constexpr type name(int i) {                \
        constexpr type t[] = {__VA_ARGS__};                         \
        return t[i];                                                \
    }

// state -> terminal kind
PRB_TABLE(kTerm, int, 4, 0, 0, 3, 0, 2, 3, 0, 1, 3, 0, 2, 3, 0, 1, 3, 0, 1, 3, 0, 2, 3, 0, 1, 3, 0,
          2, 3)
// player to act at a decision state (0 small blind, 1 big blind)
PRB_TABLE(kActor, int, 0, 0, 1, 0, 0, 1, 1, 1, 0, 0, 0, 1, 1, 1, 0, 0, 1, 0, 0, 0, 1, 1, 1, 0, 0, 0,
          1, 1)
PRB_TABLE(kParent, int, -1, 0, 1, 2, 2, 4, 4, 4, 7, 7, 7, 10, 10, 10, 13, 13, 1, 16, 16, 16, 19, 19,
          19, 22, 22, 22, 25, 25)
// small / big blind bet minus the river root bet
PRB_TABLE(kSbOff, float, 0, 0, 0, 0, 0, 0, 2, 4, 4, 4, 4, 4, 6, 8, 8, 8, 2, 2, 2, 2, 2, 4, 6, 6, 6,
          6, 6, 8)
PRB_TABLE(kBbOff, float, 0, 0, 0, 0, 2, 2, 2, 2, 2, 4, 6, 6, 6, 6, 6, 8, 0, 0, 2, 4, 4, 4, 4, 4, 6,
          8, 8, 8)
PRB_TABLE(kNChild, int, 1, 2, 2, 0, 3, 0, 0, 3, 0, 0, 3, 0, 0, 2, 0, 0, 3, 0, 0, 3, 0, 0, 3, 0, 0,
          2, 0, 0)
// children and edge ids, three per state (state * 3 + action)
PRB_TABLE(kChild3, int, 1, -1, -1, 2, 16, -1, 3, 4, -1, -1, -1, -1, 5, 6, 7, -1, -1, -1, -1, -1,
          -1, 8, 9, 10, -1, -1, -1, -1, -1, -1, 11, 12, 13, -1, -1, -1, -1, -1, -1, 14, 15, -1,
          -1, -1, -1, -1, -1, -1, 17, 18, 19, -1, -1, -1, -1, -1, -1, 20, 21, 22, -1, -1, -1, -1,
          -1, -1, 23, 24, 25, -1, -1, -1, -1, -1, -1, 26, 27, -1, -1, -1, -1, -1, -1, -1)
PRB_TABLE(kEdge3, int, -1, -1, -1, 13, 25, -1, 0, 12, -1, -1, -1, -1, 1, 2, 11, -1, -1, -1, -1,
          -1, -1, 3, 4, 10, -1, -1, -1, -1, -1, -1, 5, 6, 9, -1, -1, -1, -1, -1, -1, 7, 8, -1,
          -1, -1, -1, -1, -1, -1, 14, 15, 24, -1, -1, -1, -1, -1, -1, 16, 17, 23, -1, -1, -1, -1,
          -1, -1, 18, 19, 22, -1, -1, -1, -1, -1, -1, 20, 21, -1, -1, -1, -1, -1, -1, -1)
__host__ __device__ constexpr int kChild(int s, int k) { return kChild3(s * 3 + k); }
__host__ __device__ constexpr int kEdge(int s, int k) { return kEdge3(s * 3 + k); }

// Leaves: the 9 showdowns first, then the 8 folds. A leaf's "channel" is its index here.
constexpr int kNumSD = 9;
constexpr int kNumFold = 8;
constexpr int kNumLeaves = kNumSD + kNumFold;
PRB_TABLE(kLeaf, int, 3, 6, 9, 12, 15, 18, 21, 24, 27, 5, 8, 11, 14, 17, 20, 23, 26)
// Decision states, parents before children (the DealRiver state first).
constexpr int kNumDecision = 10;
PRB_TABLE(kDecision, int, 1, 2, 4, 7, 10, 13, 16, 19, 22, 25)

// Value multiplier of a leaf for the updating player: the showdown bet, or the folding
// player's bet with a minus sign when the updater folded (state.rs:456-492,
// poker.cu:415-431).
__host__ __device__ constexpr float leaf_scale(int leaf_state, int updater, float root_bet) {
    return kTerm(leaf_state) == kShowdown ? root_bet + kSbOff(leaf_state)
           : kTerm(leaf_state) == kSBWins
               ? (updater == 1 ? -(root_bet + kBbOff(leaf_state)) : (root_bet + kBbOff(leaf_state)))
               : (updater == 0 ? -(root_bet + kSbOff(leaf_state)) : (root_bet + kSbOff(leaf_state)));
}

}  // namespace prb
