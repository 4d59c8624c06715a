// qk_fault.h -- host-side fault injection and NVTX ranges.
//
// Fault injection exercises the library's error paths without faulting a GPU:
// QK_B200_FAULT names the sites that fail, comma-separated --
//   alloc   device / pinned allocations report cudaErrorMemoryAllocation
//   launch  kernel launches report cudaErrorLaunchFailure before launching
//   copy    host<->device copies report cudaErrorUnknown before copying
//   collective  the sharded execute reports cudaErrorUnknown instead of
//               issuing its NCCL exchange (after its own simulate kernels)
// The variable is read at every site, so a process can arm and disarm it.
// An injected failure is reported like a real one (QK_ERR_RUNTIME_INIT and a
// "cuda error: ..." message) with "[injected]" appended to the message.
//
// NVTX ranges ("qk.build", "qk.execute", ...) mark the host phases for
// profilers; without an attached tool they cost one branch.
#pragma once

#include <cuda_runtime.h>

namespace qkb {

enum FaultSite : int { kFaultAlloc = 1, kFaultLaunch = 2, kFaultCopy = 4, kFaultCollective = 8 };

// cudaSuccess, or the injected error for `site` when QK_B200_FAULT arms it.
cudaError_t injected_fault(FaultSite site);
// True once on this thread after an injected failure (then cleared).
bool take_injected_flag();

class NvtxRange {
public:
    explicit NvtxRange(const char* name);
    ~NvtxRange();
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace qkb
