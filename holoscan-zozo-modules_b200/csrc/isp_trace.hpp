// isp_trace.hpp - NVTX ranges around the host-side phases of the pipeline:
// frame submission, the statistics and tile pass launches, host staging,
// batch build and replay, the serving loop's admission, launch and reaping,
// the colour converter and the side-by-side view. The ranges live in the
// domain "holoscan.isp" and mark where the host enqueues each phase, so a
// timeline tool (Nsight Systems, or any NVTX injection library named by
// NVTX_INJECTION64_PATH) shows them above the kernels they queue. The
// reference module has no tracing; its benchmark times with CUDA events
// (modules/isp/tests/benchmark.cpp:137-142), which this build keeps.
//
// NVTX3 is header-only: with no tool attached, a range is a test of a
// function pointer, so the ranges stay on in every build.
#pragma once

#include <nvtx3/nvToolsExt.h>

#include <cstdint>

namespace isp_b200 {

// Colours per kind of phase, for a timeline's legend.
constexpr uint32_t kTraceFrame = 0xFF76B900U;   // a frame's submission
constexpr uint32_t kTraceKernel = 0xFF1F77B4U;  // one kernel launch
constexpr uint32_t kTraceCopy = 0xFFFF7F0EU;    // host <-> device staging
constexpr uint32_t kTraceServe = 0xFF9467BDU;   // serving loop steps

// The library's NVTX domain, created once per process (null, and every
// range a no-op, when no tool is attached).
inline nvtxDomainHandle_t trace_domain() {
  static const nvtxDomainHandle_t domain = nvtxDomainCreateA("holoscan.isp");
  return domain;
}

// One NVTX range for the lifetime of the object (push on construction, pop on
// destruction), named by a string literal.
class TraceRange {
 public:
  explicit TraceRange(const char* name, uint32_t argb = kTraceFrame) {
    nvtxEventAttributes_t a{};
    a.version = NVTX_VERSION;
    a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
    a.colorType = NVTX_COLOR_ARGB;
    a.color = argb;
    a.messageType = NVTX_MESSAGE_TYPE_ASCII;
    a.message.ascii = name;
    nvtxDomainRangePushEx(trace_domain(), &a);
  }
  ~TraceRange() { nvtxDomainRangePop(trace_domain()); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace isp_b200
