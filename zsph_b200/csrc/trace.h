// NVTX ranges for profilers (nsys timelines, ncu --nvtx filters).  NVTX 3 is
// header-only: with no tool attached a range costs a few nanoseconds; with
// one (NVTX_INJECTION64_PATH, or a profiler that sets it) the tool receives
// each range's name.  The library names a range after each entry point and,
// inside a step, after each kernel group (search, boundary, governing).
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace zsph {

class TraceRange {
 public:
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace zsph
