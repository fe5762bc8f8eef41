// Launchers of the river CFR kernel (river_cfr.cu).
#pragma once
#include <cuda_runtime.h>

#include "layout.h"

namespace prb {

enum { kModeCFR = 0, kModeBR = 1 };

size_t river_smem_bytes();

// One pass over n river subgames: CFR (regret update of `updater`'s edges, results are
// counterfactual values) or best response (results are best-response values, regrets
// read only). ranges / results: n rows of kRangeStride floats; regrets: n * 26 * 256.
cudaError_t launch_river(int mode, const SubgameDesc *desc, int n, const float *ranges,
                         float *results, float *regrets, const BoardPack *packs,
                         unsigned long long flop, int updater, cudaStream_t stream);

}  // namespace prb
