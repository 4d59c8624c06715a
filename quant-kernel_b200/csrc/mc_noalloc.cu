// mc_noalloc.cu -- Heston batch pricing that allocates no memory.
//
// Some callers cannot call cudaMalloc: pricing services that run inside a
// host framework owning every device allocation (a caching allocator, a
// memory pool with a hard cap), processes that must not grow their GPU
// footprint after start-up, or code paths with latency budgets that an
// allocation (and the device synchronisation a cudaFree implies) would
// break.  For them, qk_mcm_heston_monte_carlo_price_batch_noalloc runs the
// same simulate and finalize kernels as the regular Heston batch, with every
// buffer those kernels need -- option records, tile offsets, per-tile partial
// sums, prices and standard errors -- carved out of one file-scope device
// array of fixed size.  The array exists once per GPU that loads the library
// and is held until the process exits.
//
// Limits: at most kMaxOptions options and kMaxTiles tiles per call.  An
// option of P paths has ceil(P/2) antithetic pairs and takes
// min(4096, ceil(pairs / 512)) tiles: a tile holds 512 pairs until an option
// would need more than 4096 tiles (over 2^22 paths), after which each tile
// holds 512 * ceil(pairs / 2^21) pairs.  1024 options of 262144 paths fill the
// array.  Larger calls are rejected before any GPU work.
//
// Every call shares the array and it keeps the last call's contents.  Nothing
// in it has to start at zero: each call overwrites every record, tile slot and
// result before reading it.  Calls are serialised by a host lock and return
// only after their results are copied back, so calls through this entry point
// never overlap on the GPU; any other work that touched the same array while a
// call runs would race with it.
//
// The copies and launches go to a non-blocking stream of the library's own,
// created once per device at set-up: the legacy default stream would join
// (and so break) a global-mode stream capture that another thread of the
// process has in progress.
#include "mc_noalloc.h"

#include <cstring>
#include <mutex>

#include "mc_launch.h"
#include "mc_plan.h"
#include "qk_fault.h"

namespace qkb {

namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

constexpr size_t kOffRecords = 0;
constexpr size_t kOffTileBegin = align256(kOffRecords + sizeof(McOption) * kNoAllocMaxOptions);
constexpr size_t kOffPartials = align256(kOffTileBegin + sizeof(int64_t) * (kNoAllocMaxOptions + 1));
constexpr size_t kOffPrices = align256(kOffPartials + sizeof(TilePartial) * kNoAllocMaxTiles);
constexpr size_t kOffStderr = align256(kOffPrices + sizeof(double) * kNoAllocMaxOptions);
constexpr size_t kScratchBytes = align256(kOffStderr + sizeof(double) * kNoAllocMaxOptions);
static_assert(kScratchBytes == kNoAllocScratchBytes, "scratch size stated in mc_noalloc.h");

// The scratch array.  In host code this name is only a stand-in for the
// device symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;                               // serialises calls (and set-up)
unsigned char* g_scratch_dev[kMaxDevices] = {};  // per-device address, set once
cudaStream_t g_stream_dev[kMaxDevices] = {};     // per-device stream, set once

// Fixed launch shape: 256 threads x 2 pairs = 512 antithetic pairs per tile
// pass.  The regular entry uses 128-thread CTAs; the same paths summed in
// other tile groups agree to ~1e-15 relative (double-double sums), not always
// bit for bit.
constexpr int kBlock = 256;
constexpr int kUpt = 2;

// Set-up on `dev` (the current device), once: the scratch array's device
// address and the library's stream for this entry point.
cudaError_t device_setup(int dev, unsigned char** base, cudaStream_t* stream) {
    if (g_scratch_dev[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_dev[dev] = static_cast<unsigned char*>(p);
    }
    if (g_stream_dev[dev] == nullptr) {
        cudaStream_t s = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
        g_stream_dev[dev] = s;
    }
    *base = g_scratch_dev[dev];
    *stream = g_stream_dev[dev];
    return cudaSuccess;
}

}  // namespace

NoAllocStatus noalloc_heston_batch(const BatchInput& in, double* out_prices, double* out_stderr,
                                   cudaError_t* cuda_err, int64_t* tiles_needed) {
    *cuda_err = cudaSuccess;
    *tiles_needed = 0;
    if (in.n > kNoAllocMaxOptions) return NoAllocStatus::kTooManyOptions;

    // Pass 1: tile count, host only, nothing stored.
    int64_t total = 0;
    for (int32_t i = 0; i < in.n; ++i) {
        McOption o = pack_option(in, i, true);
        total += tile_option(o, kBlock, kUpt);
    }
    *tiles_needed = total;
    if (total > kNoAllocMaxTiles) return NoAllocStatus::kTooManyTiles;

    std::lock_guard<std::mutex> lock(g_mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess && (dev < 0 || dev >= kMaxDevices)) e = cudaErrorInvalidDevice;
    unsigned char* base = nullptr;
    cudaStream_t st = nullptr;
    if (e == cudaSuccess) e = device_setup(dev, &base, &st);
    if (e != cudaSuccess) {
        *cuda_err = e;
        return NoAllocStatus::kCudaError;
    }
    McOption* d_rec = reinterpret_cast<McOption*>(base + kOffRecords);
    int64_t* d_tb = reinterpret_cast<int64_t*>(base + kOffTileBegin);
    TilePartial* d_part = reinterpret_cast<TilePartial*>(base + kOffPartials);
    double* d_price = reinterpret_cast<double*>(base + kOffPrices);
    double* d_se = reinterpret_cast<double*>(base + kOffStderr);

    // Pass 2: pack in fixed stack chunks and copy each (copies from pageable
    // memory, which return once the source has been read: no staging buffer
    // of ours).
    constexpr int kChunk = 64;
    McOption rec[kChunk];
    int64_t tb[kChunk];
    int64_t running = 0;
    for (int32_t i0 = 0; i0 < in.n && e == cudaSuccess; i0 += kChunk) {
        const int32_t m = (in.n - i0) < kChunk ? (in.n - i0) : kChunk;
        for (int32_t j = 0; j < m; ++j) {
            rec[j] = pack_option(in, i0 + j, true);
            rec[j].tile_begin = running;
            running += tile_option(rec[j], kBlock, kUpt);
            tb[j] = rec[j].tile_begin;
        }
        e = cudaMemcpyAsync(d_rec + i0, rec, sizeof(McOption) * m, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_tb + i0, tb, sizeof(int64_t) * m, cudaMemcpyHostToDevice, st);
        // the stack chunk is rewritten next: wait until this one is consumed
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_tb + in.n, &running, sizeof(int64_t), cudaMemcpyHostToDevice, st);

    if (e == cudaSuccess && running > 0) {
        SimArgs a;
        a.opts = d_rec;
        a.tile_begin = d_tb;
        a.n = in.n;
        a.n_tiles = running;
        a.partials = d_part;
        a.max_ctas = 0x7fffffff;
        e = injected_fault(kFaultLaunch);
        if (e == cudaSuccess) e = launch_simulate(kFamHeston, true, kBlock, kUpt, 1, a, st);
    }
    if (e == cudaSuccess) e = launch_finalize(d_rec, in.n, d_part, d_price, d_se, nullptr, nullptr, st);
    if (e == cudaSuccess) e = injected_fault(kFaultCopy);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out_prices, d_price, sizeof(double) * in.n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && out_stderr)
        e = cudaMemcpyAsync(out_stderr, d_se, sizeof(double) * in.n, cudaMemcpyDeviceToHost, st);
    // the results are in the caller's arrays only once the stream is done; on
    // an error, drain what was queued before returning so that the next call
    // never overlaps it
    const cudaError_t es = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = es;
    if (e != cudaSuccess) {
        *cuda_err = e;
        return NoAllocStatus::kCudaError;
    }
    return NoAllocStatus::kOk;
}

}  // namespace qkb
