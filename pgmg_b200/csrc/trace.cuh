// NVTX ranges around the library's host-side phases: set-up (stencil upload
// or assembly, Galerkin hierarchy, coarse LU), solves, residual checks,
// mixed-precision refinement steps, V-cycles, autotuning and batch steps.  A
// profiler that records NVTX (Nsight Compute with --nvtx and its
// --nvtx-include filters, Nsight Systems) attributes each kernel launch to
// the ranges open on the launching thread.  NVTX v3 is header-only: with no
// tool attached (NVTX_INJECTION64_PATH unset) a range is two calls through
// no-op function pointers.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace pgmg {

// Pushes `name` on this thread's NVTX range stack (when `on`) until end()
// or the end of the scope, whichever comes first: every return path pops it.
class TraceRange {
public:
    explicit TraceRange(const char* name, bool on = true) : on_(on) {
        if (on_) nvtxRangePushA(name);
    }
    ~TraceRange() { end(); }
    void end() {
        if (on_) nvtxRangePop();
        on_ = false;
    }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;

private:
    bool on_;
};

}  // namespace pgmg
