// mc_plan.h -- host runtime of the Monte Carlo path: batch validation and
// packing, device buffers, launches, CUDA graphs and the autotuner.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "mc_types.h"

namespace qkb {

// SoA view of one batch in host memory (any field a model does not use may be
// null when no option of that model is present).
struct BatchInput {
    const int32_t* model = nullptr;  // null: every option uses `uniform_model`
    int32_t uniform_model = 0;
    const double *spot = nullptr, *strike = nullptr, *t = nullptr, *vol = nullptr, *r = nullptr,
                 *q = nullptr;
    const double *v0 = nullptr, *kappa = nullptr, *theta = nullptr, *sigma = nullptr,
                 *rho = nullptr;
    const double* weight_clip = nullptr;  // Heston LR delta; null: taken from `vol`
    const double* shift = nullptr;        // importance sampling; null: taken from `v0`
    const int32_t *option_type = nullptr, *paths = nullptr, *steps = nullptr;
    const uint64_t* seed = nullptr;
    int32_t n = 0;
};

enum : int32_t {
    kFlagPersistent = 0x1,
    kFlagGraph = 0x2,
    kFlagNoAntithetic = 0x4,
    kFlagTiming = 0x8,
    kFlagAutotune = 0x10,
    kFlagFamilyGrids = 0x20,
    kFlagStepUnroll2 = 0x40,
};

// Grow-only device / pinned host allocations.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};
struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

// upt > 0: one single-family grid with `upt` units per thread.  For plans
// over several families: upt == kUptPersistent runs one persistent
// work-stealing kernel, upt == kUptFamilyGrids one grid per family group
// (the autotuner picks between them).
constexpr int kUptPersistent = 0;
constexpr int kUptFamilyGrids = -1;

struct LaunchConfig {
    int block = 256;
    int upt = 2;
    int su = 1;  // step blocks per loop iteration (stepwise single-family grids)
};

class Plan {
public:
    Plan() = default;
    ~Plan();
    Plan(const Plan&) = delete;
    Plan& operator=(const Plan&) = delete;

    // Validates and packs `in`, uploads it.  Returns a CUDA error (or
    // cudaErrorInvalidValue with `err` set for a bad input set).
    cudaError_t build(const BatchInput& in, int32_t flags, std::string* err);
    cudaError_t execute(cudaStream_t stream);
    cudaError_t results(double* out_price, double* out_se);
    cudaError_t release();
    // Waits for the last execute and refreshes last_simulate_ms().
    cudaError_t sync_stats();

    int32_t n() const { return n_; }
    int64_t n_tiles() const { return n_tiles_; }
    int64_t path_steps() const { return path_steps_; }
    double last_simulate_ms() const { return last_ms_; }
    int launches() const {
        if (n_tiles_ <= 0) return 1;
        return (cfg_.upt == kUptFamilyGrids ? (int)groups_.size() : 1) + 1;
    }
    int block() const { return cfg_.block; }
    int upt() const { return cfg_.upt; }
    int step_unroll() const { return cfg_.upt > 0 ? cfg_.su : 1; }
    int ctas() const { return max_ctas_; }
    bool persistent() const { return persistent_; }
    double* d_price() const { return static_cast<double*>(d_price_.p); }
    double* d_se() const { return static_cast<double*>(d_se_.p); }
    int device() const { return device_; }
    TilePartial* d_partials() const { return static_cast<TilePartial*>(d_partials_.p); }
    cudaStream_t stream() const { return stream_; }

    // ---- one rank's share of a batch priced on several GPUs ----
    // Tile bounds b[0..world] of a contiguous partition of the plan's tiles
    // (work order) balanced by path-steps: rank k simulates [b[k], b[k+1]).
    // The same plan on every rank gives the same bounds.
    const std::vector<int64_t>& shard_bounds(int world);
    // Orders work on `st` after the plan's own uploads (no-op on its stream).
    cudaError_t order_after_upload(cudaStream_t st);
    // The simulate kernels over tiles [lo, hi) only (per-family grids).
    cudaError_t launch_tiles(cudaStream_t st, int64_t lo, int64_t hi, bool timing);
    // The finalize kernel over every option (results in the caller's order).
    cudaError_t launch_finalize_all(cudaStream_t st);
    // The stream results() waits on.
    void note_stream(cudaStream_t st) { last_stream_ = st; }

private:
    cudaError_t ensure_stream();
    cudaError_t layout_tiles(const LaunchConfig& cfg);  // tile geometry + upload
    cudaError_t launch_all(cudaStream_t st, bool timing);
    cudaError_t autotune();
    cudaError_t capture_graph();
    void drop_graph();

    int device_ = -1;
    cudaStream_t stream_ = nullptr;
    cudaStream_t last_stream_ = nullptr;
    int32_t flags_ = 0;
    int32_t n_ = 0;
    int64_t n_tiles_ = 0;
    int64_t path_steps_ = 0;
    int family_ = -1;  // single family of all simulated options, or -1 (mixed / none)
    bool anti_ = true;
    bool persistent_ = false;
    LaunchConfig cfg_;
    int max_ctas_ = 0;
    double last_ms_ = 0.0;
    bool counter_ready_ = false;

    std::vector<McOption> opts_;       // host copy (units/tiles filled per layout)
    std::vector<int32_t> order_;       // device record k is option order_[k]
    struct Group {                     // options of one (family, antithetic) pair
        int family;
        bool anti;
        int32_t opt_lo, opt_hi;        // record range in work order
        int64_t tile_lo, tile_hi;
    };
    std::vector<Group> groups_;        // filled for multi-family plans
    std::vector<int64_t> shard_bounds_;  // cached partition (shard_world_ ranks)
    int shard_world_ = 0;
    DevBuf d_opts_, d_tile_begin_, d_partials_, d_price_, d_se_, d_counter_, d_out_index_,
        d_groups_;
    PinnedBuf h_opts_, h_tile_begin_, h_price_, h_se_, h_out_index_, h_groups_;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
};

// Packs option i of `in` (entry checks, special cases, model constants).
McOption pack_option(const BatchInput& in, int32_t i, bool anti_stepwise);
// Fills o.tiles / o.unit_iters for a launch of `block` threads with `upt`
// units each; returns o.tiles.
int32_t tile_option(McOption& o, int block, int upt);

// Contiguous partition of n items with the given costs into `world` ranges
// of near-equal total cost: bounds[0] = 0, bounds[world] = n, and bounds[r]
// is the item boundary whose cumulative cost is nearest r/world of the total
// (ties: the earlier boundary; never below bounds[r - 1]).  Host only.
void partition_by_cost(const double* cost, int64_t n, int world, int64_t* bounds);

// Per-thread, per-device scratch plan used by the one-shot batch calls.
Plan* thread_scratch_plan(int device);

// Default launch shape per family, and the autotuner's cached choice.
LaunchConfig default_config(int family);
bool tuned_config(const std::string& key, LaunchConfig* out);
void store_tuned_config(const std::string& key, const LaunchConfig& cfg);

}  // namespace qkb
