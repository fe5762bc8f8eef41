// Launcher of the device-side table generation (gen_tables.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace prb {

// Fills, for all 1326 {turn, river} slots of `flop`, the packed tables in the reference's
// layout: eval (1326 * 1838), coll (1326 * 2652) and buckets (1326 * 1326), u16.
cudaError_t launch_gen_tables(unsigned long long flop, uint16_t *eval, uint16_t *coll, uint16_t *abstr,
                              cudaStream_t stream);

}  // namespace prb
