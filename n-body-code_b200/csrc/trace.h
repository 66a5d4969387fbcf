// NVTX ranges around the engine's public calls, so an Nsight timeline shows
// set_state / acc_jerk / step / energy / force_calculation by name.  NVTX 3 is
// header-only: without a profiler attached each range costs a branch.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace nbody {

struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace nbody
