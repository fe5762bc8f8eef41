// Launchers of the river CFR kernel (river_cfr.cu).
#pragma once
#include <cuda_runtime.h>

#include "layout.h"

namespace prb {

enum { kModeCFR = 0, kModeBR = 1 };

// Shared memory per CTA for a pass; max_groups / max_card_groups are the largest tie-group
// counts over the flop's boards.
size_t river_smem_bytes(int mode, int fp64, int max_groups, int max_card_groups);

// One pass over n river subgames: CFR (regret update of `updater`'s edges, results are
// counterfactual values) or best response (results are best-response values, regrets
// read only). ranges / results: n rows of kRangeStride values; regrets: n * 26 * 256.
// In CFR mode with own_ranges (the updater's ranges, same rows) and avg_sums (n * 26 * 256)
// the pass also accumulates average-strategy sums.
cudaError_t launch_river(int mode, const SubgameDesc *desc, int n, const float *ranges, float *results,
                         float *regrets, const BoardPack *packs, unsigned long long flop, int updater,
                         int max_groups, int max_card_groups, const float *own_ranges, float *avg_sums,
                         cudaStream_t stream);

// Best response in double precision.
cudaError_t launch_river_br64(const SubgameDesc *desc, int n, const double *ranges, double *results,
                              float *regrets, const BoardPack *packs, unsigned long long flop, int updater,
                              int max_groups, int max_card_groups, cudaStream_t stream);

}  // namespace prb
