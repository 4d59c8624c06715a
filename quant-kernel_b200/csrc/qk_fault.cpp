// qk_fault.cpp -- see qk_fault.h.
#include "qk_fault.h"

#include <cstdlib>
#include <cstring>

#include <nvtx3/nvToolsExt.h>

namespace qkb {

namespace {

thread_local bool tl_injected = false;

int armed_sites() {
    const char* v = std::getenv("QK_B200_FAULT");
    if (!v || !*v) return 0;
    int sites = 0;
    if (std::strstr(v, "alloc")) sites |= kFaultAlloc;
    if (std::strstr(v, "launch")) sites |= kFaultLaunch;
    if (std::strstr(v, "copy")) sites |= kFaultCopy;
    if (std::strstr(v, "collective")) sites |= kFaultCollective;
    return sites;
}

}  // namespace

cudaError_t injected_fault(FaultSite site) {
    if (!(armed_sites() & site)) return cudaSuccess;
    tl_injected = true;
    switch (site) {
        case kFaultAlloc: return cudaErrorMemoryAllocation;
        case kFaultLaunch: return cudaErrorLaunchFailure;
        default: return cudaErrorUnknown;
    }
}

bool take_injected_flag() {
    const bool f = tl_injected;
    tl_injected = false;
    return f;
}

NvtxRange::NvtxRange(const char* name) { nvtxRangePushA(name); }
NvtxRange::~NvtxRange() { nvtxRangePop(); }

}  // namespace qkb
