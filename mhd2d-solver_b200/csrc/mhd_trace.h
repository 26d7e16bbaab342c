// NVTX ranges on the host side of the library (header-only NVTX 3): each
// entry point and each stage it enqueues opens a named range, so a timeline
// tool (Nsight Systems) shows which call and which RK3 stage launched every
// kernel.  Without a tool attached the calls do nothing measurable.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace mhd {

class TraceRange {
 public:
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace mhd

#define MHD_TRACE_CAT2(a, b) a##b
#define MHD_TRACE_CAT(a, b) MHD_TRACE_CAT2(a, b)
// Opens a range that closes at the end of the enclosing scope.
#define MHD_TRACE(name) ::mhd::TraceRange MHD_TRACE_CAT(mhd_trace_, __LINE__)(name)
