// NVTX ranges around the host entry points (river passes, batch iterations, game iterations,
// exploitability, value-network steps), so that a timeline tool (nsys, ncu --nvtx) shows
// which call a kernel belongs to. NVTX 3 is header-only; with no tool attached a range costs
// a call through a no-op pointer.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace prb {

class TraceRange {
  public:
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

}  // namespace prb
