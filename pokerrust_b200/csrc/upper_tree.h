// Device traversal of the preflop, flop and turn tree (upper_tree.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace prb {

// Node kinds; the values are those of the host tree in game.cu.
enum : int8_t { kUDecide = 0, kUSBWins = 1, kUBBWins = 2, kUFlop = 4, kUTurn = 5, kURiver = 6 };

struct DevNode {
    int8_t kind, actor, nchild, pad0;
    int32_t first;          // first child in UpperView::kids
    unsigned long long cards;
    float sb, bb;
    long long regret;       // offset of nchild * 1326 regrets (decision nodes)
    int32_t river;          // river root index (kURiver)
    int32_t perm_first;     // flop children: suit permutations [perm_first, perm_first + nperm)
    int32_t nperm;
    int32_t pad1;
};

struct UpperView {
    const DevNode *nodes;
    const int32_t *kids;
    const int32_t *perm_maps;  // [perm][1326]: hand index -> permuted hand index
    const float *regrets;      // read by the top-down sweep
};

// Ranges of the root: every hand 1 for both players (rows of kRangeStride, padding 0).
cudaError_t upper_set_root(float *Rf, double *Rd, cudaStream_t s);

// Top-down sweep of one tree level: the children's reach vectors of every node in
// level_nodes[0, count); river roots write the updater's opponent range to river_opp (and the
// updater's own range to river_own when it is not null), row = river index.
template <typename T>
cudaError_t upper_down(const UpperView &v, const int *level_nodes, int count, int upd, T *R, T *river_opp,
                       float *river_own, cudaStream_t s);

// Bottom-up sweep of one tree level: the updater's values at every node in level_nodes; in a
// CFR pass (best_response 0) decision nodes of the updater also update regrets and, when avg
// is not null, the average-strategy sums.
template <typename T>
cudaError_t upper_up(const UpperView &v, const int *level_nodes, int count, int upd, int best_response,
                     const T *R, T *V, const T *river_val, float *regrets, float *avg, cudaStream_t s);

}  // namespace prb
