// Batched solver of general river subgames (batch_solver.cu): many independent river
// subgames, each with its own 5-card board, pot, stack and bet tree (batch_tree.h), solved
// with per-hand regrets by one persistent kernel fed from a device work queue.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "batch_tree.h"

namespace prb {

constexpr int kBLive = 1081;   // hands that share no card with a 5-card board
constexpr int kBRow = 1088;    // per-hand rows, padded to a multiple of 32
constexpr int kBLists = 47;    // off-board cards
constexpr int kBListLen = 46;  // live hands holding one off-board card
constexpr int kBChunks = kBRow / 32;
constexpr int kBChunks64 = kBRow / 64;  // 64-hand chunks of the rank-order scan

// One subgame as the kernels see it.
struct BSub {
    unsigned long long board;
    int node_off, num_nodes;
    int edge_off;  // first regret row: rows of kBRow values, one per edge
    int num_edges, num_leaves;
    float pot;
};

// Per-subgame hand layout, built on the device from the board. Hands are held in rank
// order ("positions"), weakest first, positions kBLive.. kBRow-1 are padding.
struct BPack {
    uint32_t grp[kBRow];             // first | last position of the tie group << 16
    uint32_t lists[kBRow];           // list of the low card | list of the high card << 8 |
                                     //   first << 16 | last << 24 index of the tie group in the low card's list
    uint32_t lists2[kBRow];          // first | last << 8: the same in the high card's list
    uint16_t hand[kBRow];            // colex hand index of each position (0xFFFF: padding)
    uint16_t clpos[kBLists][48];     // positions holding each off-board card, in rank order
    uint8_t list_card[48];
    uint16_t pos_of[1328];           // position of each colex hand (0xFFFF: blocked)
};

static_assert(offsetof(BPack, clpos) % 4 == 0 && sizeof(BPack) % 4 == 0, "card lists move as 4-byte words");

enum { kBModeCFR = 0, kBModeBR = 1, kBModeEval = 2 };

struct BLaunch {
    const BSub *subs;
    const BNode *nodes;
    const BPack *packs;
    const float *ranges;  // [subgame][2][kBRow], position order
    float *regrets;       // [edge row][kBRow]
    float *avg;           // [edge row][kBRow] (average-strategy sums) or null
    const int *order;     // work queue: subgame ids in schedule order
    int *head;            // queue head, zero before the launch
    int count;            // subgames in the queue
    int player;           // updating / best-responding player
    int use_average;      // BR / Eval: strategies from the average sums instead of regrets
    void *root_out;       // [subgame][kBRow] root values of `player` (V), or null
    void *sum_out;        // [subgame] sum over hands of range x root value (V), or null
    void *child_out;      // [subgame][8][kBRow] values of the root's children (V), or null
    const double *ranges64;  // double passes: [subgame][2][kBRow] opponent weights, or null (use ranges)
    int own_reach;        // CFR: average sums weighted by the updater's range (subgames inside a larger
                          // game, whose ranges change between iterations), not by 1
    const float *avg_weight;  // CFR: device scalar multiplying this pass's average-sum terms, or null (1)
};

// Builds the packs and position-order ranges of `count` subgames: ranges_in holds
// [subgame][2][1326] colex-order ranges.
cudaError_t launch_batch_setup(const BSub *subs, int count, BPack *packs, const float *ranges_in,
                               float *ranges_pos, int *err, cudaStream_t stream);

// One pass over the queue. K = hands per thread (2, 3 or 4); fp64 selects double
// arithmetic (best response and evaluation only). ctas = grid size (persistent CTAs).
// dense (K = 4 CFR passes in single precision only): the configuration with registers capped
// for 3 CTAs per SM; it expects groups of batch_dense_group() leaves.
cudaError_t launch_batch_pass(int mode, int K, int fp64, int avg, const BLaunch &a, int ctas, int max_leaves,
                              cudaStream_t stream, int dense = 0);

// Adds 1 to the device scalar *w (the next iteration's average weight), on `stream`.
cudaError_t launch_weight_step(float *w, cudaStream_t stream);

// Threads per CTA and shared memory of a configuration.
int batch_threads(int K);
size_t batch_smem_bytes(int K, int fp64, int group_leaves);
int batch_group_leaves(int fp64);
// Leaf group of the dense K = 4 configuration (3 CTAs per SM fit in shared memory).
int batch_dense_group();
// Resident CTAs per SM the configuration allows (0 if it cannot launch).
int batch_ctas_per_sm(int mode, int K, int fp64, int avg);
// The same for the dense K = 4 CFR configuration.
int batch_dense_ctas_per_sm(int avg);

}  // namespace prb
