// Library-internal hooks of the batched river solver for a larger game that owns river
// subgames (the full-game solver): device views of the batch's packs and range rows, passes
// launched on the caller's stream, and range-weighted average sums.
#pragma once
#include <cuda_runtime.h>

#include "batch_solver.h"

namespace prb {

struct BatchView {
    const BPack *packs;   // [count] position tables of each subgame
    float *ranges;        // [count][2][kBRow] position-order ranges
    double *ranges64;     // [count][2][kBRow] double ranges for best responses (null until asked for)
    int count;
    cudaStream_t stream;  // the batch's own stream
};

// Device views of a batch; need64 allocates the double range rows on first use.
int batch_view(void *batch, BatchView *v, bool need64);
// CFR passes weight the average sums by the updater's range (reach into the subgame) instead
// of 1.
int batch_set_own_weight(void *batch, bool on);
// CFR average-sum terms multiplied by the device scalar *weight (null: 1), e.g. the iteration
// number for linearly weighted averages.
int batch_set_avg_weight(void *batch, const float *weight);
// One pass of `mode` (kBModeCFR / kBModeBR / kBModeEval) for `player` over every subgame,
// queued on stream `on`; root values ([count][kBRow], position order, float or double as
// fp64) go to root_out. Double passes read ranges64.
int batch_run_pass(void *batch, int mode, int player, int fp64, int use_average, void *root_out,
                   cudaStream_t on);
// Zeroes the regrets and average sums, queued on stream `on`.
int batch_clear(void *batch, cudaStream_t on);
// The batch's regret and average-sum rows (avg null when averages are off) and the bytes of
// each array.
int batch_rows(void *batch, float **regrets, float **avg, size_t *bytes);

}  // namespace prb
