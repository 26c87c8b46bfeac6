// es_nvtx.h - NVTX ranges (domain "es_b200") around the stages of the C ABI
// and the runner: grid upload, sector set-up, lifetimes, temperatures, batch
// recording and replay, GPU grid builds, and each sample of a .config sweep.
// A profiler that reads NVTX (Nsight Systems; ncu --nvtx --nvtx-include
// "es_b200@<range>/") shows them on its timeline or filters kernels by them.
// Header-only NVTX v3: without a tool attached a range costs one branch. The
// reference times its stages with host counters only
// (src/sim/SimulationCPU.cpp:37-40,62-68; src/SimulationRunner.cpp:45-62).
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace es {

inline nvtxDomainHandle_t nvtx_domain()
{
    static const nvtxDomainHandle_t d = nvtxDomainCreateA("es_b200");
    return d;
}

class Range {
public:
    explicit Range(const char* name)
    {
        nvtxEventAttributes_t a = {};
        a.version = NVTX_VERSION;
        a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
        a.messageType = NVTX_MESSAGE_TYPE_ASCII;
        a.message.ascii = name;
        nvtxDomainRangePushEx(nvtx_domain(), &a);
    }
    ~Range() { nvtxDomainRangePop(nvtx_domain()); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

}  // namespace es
