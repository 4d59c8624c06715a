// mc_launch.h -- host-side launch interface of the Monte Carlo kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace qkb {

struct McOption;
struct TilePartial;

// Kernel families: the models that share one simulation loop.
enum : int {
    kFamTerminal = 0,
    kFamEuler = 1,
    kFamMilstein = 2,
    kFamHeston = 3,
    kFamHestonLr = 4,
    kFamVr = 5,  // terminal GBM with a variance-reduction estimator (models 8-12)
    kNumFamilies = 6
};

// Units per thread compiled into the persistent mixed-model kernel (and used
// by the per-family grids of a mixed plan).  The stepwise families take four:
// the mixed benchmark batch ran 52.9 ms with four (persistent kernel, seven
// CTAs per SM) against 56.1 ms with two stepwise units per thread; Heston
// keeps two, whose four-unit body needs 79-93 registers.
// Results do not depend on these (tile sums are exact double-double sums
// merged in a fixed order).
constexpr int kUptTerminal = 1;
constexpr int kUptStepwise = 4;
constexpr int kUptHeston = 2;
constexpr int kUptVr = 1;

// The one family -> units-per-thread map: the persistent kernel's family
// bodies, the tiling of every mixed plan and the default single-family
// tiling all take it, so a mixed launch and the per-method calls tile each
// option alike and give the same bits.
constexpr int family_upt(int family) {
    return family == kFamTerminal ? kUptTerminal
         : family == kFamVr ? kUptVr
         : (family == kFamHeston || family == kFamHestonLr) ? kUptHeston
         : kUptStepwise;
}
template <int FAMILY>
constexpr int kFamilyUpt = family_upt(FAMILY);  // the same, as a compile-time constant for kernels

inline bool family_is_stepwise(int family) {
    return family == kFamEuler || family == kFamMilstein || family == kFamHeston ||
           family == kFamHestonLr;
}

// Two Philox step blocks per loop iteration (step unrolling 2) are compiled
// for the stepwise families at 1 and 2 units per thread, and for the
// one-factor families also at 4 (their default tiling); Heston's four-unit
// body has no registers to spare for a second block of Philox words.
constexpr bool step_unroll2_compiled(int family, int upt) {
    return (family == kFamEuler || family == kFamMilstein) ? (upt == 1 || upt == 2 || upt == 4)
         : (family == kFamHeston || family == kFamHestonLr) ? (upt == 1 || upt == 2)
         : false;
}

struct SimArgs {
    const McOption* opts;      // device, n records
    const int64_t* tile_begin; // device, n + 1 entries
    int32_t n;
    int64_t n_tiles;
    TilePartial* partials;     // device, indexed by absolute tile
    int32_t max_ctas;          // grid cap (grid-stride beyond it)
    int64_t tile0 = 0;         // absolute index of this launch's first tile
};

// The persistent kernel's view of a plan's work order: runs of consecutive
// records of one (family, antithetic) pair.  Group g holds records
// [opt_lo, opt_hi) and tiles [tile_hi of g - 1 (0 for g = 0), tile_hi); every
// record of a group has at least one tile, and the groups cover all tiles.
constexpr int kMaxGroups = 16;
struct GroupTable {
    int32_t count;
    int32_t code[kMaxGroups];  // family * 2 + antithetic
    int32_t opt_lo[kMaxGroups];
    int32_t opt_hi[kMaxGroups];
    int64_t tile_hi[kMaxGroups];
};

int family_of(int32_t model);

// su: step blocks per loop iteration of the stepwise families (1 or 2; 2 only
// with upt 1 or 2); other families take 1.
cudaError_t launch_simulate(int family, bool anti, int block, int upt, int su, const SimArgs& a,
                            cudaStream_t st);
// groups: device copy of the plan's GroupTable.
cudaError_t launch_persistent(int block, const SimArgs& a, const GroupTable* groups,
                              unsigned long long* work_counter, cudaStream_t st);
// out_index (nullable): record k's results go to slot out_index[k].
cudaError_t launch_finalize(const McOption* opts, int32_t n, const TilePartial* partials,
                            double* out_price, double* out_se, const int32_t* out_index,
                            unsigned long long* work_counter, cudaStream_t st);
// Resident CTAs on `device` for a family kernel (family >= 0) or the
// persistent kernel (family < 0); 0 on error.
int max_resident_ctas(int family_or_persistent, int block, int upt, int device);

}  // namespace qkb
