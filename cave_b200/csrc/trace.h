// trace.h -- NVTX ranges around the library's phases, the counterpart of the reference's named
// timestamp spans (queryManager.h:13-97; searchSimulation / searchManager / searchCopy,
// searchSystem.cpp:542-618). Nsight Systems shows them on the host timeline with the kernels
// each one launched, and `ncu --nvtx --nvtx-include <range>/` filters launches by them. NVTX is
// header-only (nvtx3): without a tool attached a range costs one call into an empty stub.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace cave {

struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace cave
