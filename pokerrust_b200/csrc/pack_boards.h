// Launcher of the device-side table re-pack (pack_boards.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "layout.h"

namespace prb {

// err[0] gets error bits: 1 sort position out of range, 2 not a permutation, 4 a blocked
// hand outside the bottom group, 8 bucket >= 256, 16 card list length. err[1] / err[2] get
// the largest tie-group counts over the boards (rank list / all card lists).
void launch_pack_boards(unsigned long long flop, const uint16_t *eval, const uint16_t *abstr,
                        BoardPack *packs, int *err, cudaStream_t stream);

}  // namespace prb
