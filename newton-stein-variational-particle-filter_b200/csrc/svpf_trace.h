// svpf_trace.h -- NVTX ranges around the host entry points that launch or
// wait for device work.  A profiler that reads NVTX (nsys, ncu --nvtx) then
// files every kernel under the C function that issued it, named as in the
// C ABI (svpf_step_graph, svpf_batch_graph_launch, svpf_grad_backward, ...);
// nested calls nest (svpf_step -> svpf_step_graph).  The NVTX v3 headers are
// header-only: with no tool attached a push or pop is a call through a
// function pointer to an empty stub.  Building with -DSVPF_NO_NVTX removes
// the ranges altogether.
#pragma once

#ifndef SVPF_NO_NVTX
#include <nvtx3/nvToolsExt.h>
#endif

namespace svpf {

class TraceRange {
public:
    explicit TraceRange(const char* name) {
#ifndef SVPF_NO_NVTX
        nvtxRangePushA(name);
#else
        (void)name;
#endif
    }
    ~TraceRange() {
#ifndef SVPF_NO_NVTX
        nvtxRangePop();
#endif
    }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace svpf

// One range for the rest of the enclosing scope, named after the function.
#define SVPF_TRACE() ::svpf::TraceRange svpf_trace_range_(__func__)
