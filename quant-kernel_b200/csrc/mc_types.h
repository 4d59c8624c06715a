// mc_types.h -- plain data shared by the host runtime and the kernels.
#pragma once

#include <cstdint>

namespace qkb {

// Largest step count a stepwise option may have: the kernels count steps in
// int32 blocks of up to 12, so the last block's index must not wrap.  Larger
// counts (over 2.1e9 steps per path) are rejected as invalid input (NaN).
constexpr int32_t kMaxSteps = 0x7FFFFFFF - 64;

// ---------------------------------------------------------------------------
// Model codes (same values as QK_MC_* in include/qk_api.h).
// ---------------------------------------------------------------------------
enum : int32_t {
    kStandard = 0,
    kAntithetic = 1,
    kEuler = 2,
    kMilstein = 3,
    kLocalVol = 4,
    kTerminalPlain = 5,
    kHeston = 6,
    kHestonLrDelta = 7,  // likelihood-ratio delta under the Heston model
    // terminal GBM with a variance-reduction estimator
    kControlVariates = 8,     // control_variates.cpp:10-52
    kImportanceSampling = 9,  // importance_sampling.cpp:11-36
    kStratified = 10,         // stratified_sampling.cpp:11-35
    kQmcSobol = 11,           // quasi_monte_carlo.cpp:10-32
    kQmcHalton = 12,          // quasi_monte_carlo.cpp:34-56
    kNumModels = 13
};

enum : int32_t { kModeSimulate = 0, kModeConstant = 1 };

// ---------------------------------------------------------------------------
// Option record: 128 bytes, packed on the host, read once per tile.
//
// Model constants of the stepwise models (FP32, rounded from FP64 host values):
//   Euler/LV (2,4):    p0 = (r - q) dt               p1 = vol sqrt(dt)
//                      p2 = 1e-12 / spot (floor of S/spot)
//   Milstein (3):      p0 = (r - q) dt - c           p1 = vol sqrt(dt)
//                      p2 = 1e-12 / spot             p3 = c = vol^2 dt / 2
//   Heston (6):        p0 = (r - q) dt   p1 = dt/2   p2 = sqrt(dt)
//                      p3 = kappa dt     p4 = kappa theta dt
//                      p5 = sigma sqrt(dt)           p6 = rho
//                      p7 = sqrt(max(1 - rho^2, 0))  p8 = v0
//                      p9 = log(1e-12 / spot) (floor of log(S/spot))
//   Heston LR delta (7): the Heston constants; the record's weight_clip
//                      bounds the first-step score z1 / (sqrt(v0) sqrt(dt) S0)
// The terminal models (0, 1, 5) and the variance-reduction models (8-12) keep
// FP64 constants in d[] (the same bytes):
//   d0 = (r - q - vol^2/2) t      d1 = vol sqrt(t)
//   d2 = importance-sampling shift
//   d3 = spot exp((r - q) t), the mean of S_T (control-variate centre)
// ---------------------------------------------------------------------------
struct alignas(16) McOption {
    double spot;
    double strike;
    double disc;         // exp(-r t)
    union {
        double const_price;  // result when mode == kModeConstant
        double weight_clip;  // Heston LR delta (simulated): |score| bound
    };
    uint64_t seed;
    int64_t tile_begin;  // first tile of this option in the plan
    int32_t tiles;       // tiles of this option (0 when constant)
    int32_t model;
    int32_t option_type;
    int32_t paths;
    int32_t steps;
    int32_t units;       // antithetic: ceil(paths/2) pairs; plain: paths
    int32_t samples;     // standard-error samples: full pairs or paths
    int32_t unit_iters;  // per-thread passes over the tile
    int32_t mode;
    int32_t antithetic;
    union {
        float p[10];
        double d[5];
    };
};
static_assert(sizeof(McOption) == 128, "McOption layout");

// Per-tile partial sums: y = pair mean (antithetic) or payoff (plain).  The
// unpaired last path of an odd antithetic count is kept apart in `lone`: it
// belongs in the price but not in the pair-mean variance.  Stratified
// sampling puts the sum of squared differences of paired strata in q; the
// control-variate model adds plain FP64 sums of the centred control
// c = S_T - E[S_T]: sum c, sum c^2 and sum c * payoff.
struct alignas(16) TilePartial {
    double sy_hi, sy_lo;  // sum of y over full samples
    double q_hi, q_lo;    // sum of y^2 over full samples
    double lone;          // payoff of the unpaired path (0 elsewhere)
    double cx, cxx, cxy;  // control variates only (0 elsewhere)
};
static_assert(sizeof(TilePartial) == 64, "TilePartial layout");

}  // namespace qkb
