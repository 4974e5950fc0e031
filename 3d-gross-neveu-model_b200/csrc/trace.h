// trace.h -- NVTX ranges on the host timeline around the library's phases
// (a trajectory, a solve, a force, the condensate, a batched or served step),
// for profilers that record NVTX (ncu --nvtx filters on them).  NVTX v3 is
// header-only: without a tool attached a range costs a pointer test.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace gn {

struct TraceRange {
  explicit TraceRange(const char *name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange &) = delete;
  TraceRange &operator=(const TraceRange &) = delete;
};

}  // namespace gn
