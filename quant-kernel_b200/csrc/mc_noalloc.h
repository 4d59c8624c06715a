// mc_noalloc.h -- limits and interface of the allocation-free Heston batch.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace qkb {

struct BatchInput;

// Capacity of the fixed device array (one per GPU, held until exit).
constexpr int32_t kNoAllocMaxOptions = 4096;
constexpr int64_t kNoAllocMaxTiles = 262144;  // an option takes min(4096, ceil(pairs/512))
constexpr size_t kNoAllocScratchBytes = 17400064;  // 16.6 MiB

enum class NoAllocStatus { kOk, kTooManyOptions, kTooManyTiles, kCudaError };

// Prices a Heston batch (host arrays in, host arrays out) with every device
// buffer inside the fixed array; out_stderr may be null.
NoAllocStatus noalloc_heston_batch(const BatchInput& in, double* out_prices, double* out_stderr,
                                   cudaError_t* cuda_err, int64_t* tiles_needed);

}  // namespace qkb
