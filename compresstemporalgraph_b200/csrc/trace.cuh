// Named ranges for profiler timelines (NVTX v3, header-only): every public workload call, the
// loader included, shows up by name under nsys or `ncu --nvtx`.  Without a tool attached the calls
// return at once.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace tga {
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};
}  // namespace tga

#define TGA_TRACE(name) ::tga::TraceRange tga_trace_range_(name)
