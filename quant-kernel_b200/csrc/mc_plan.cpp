// mc_plan.cpp -- host runtime of the Monte Carlo path.
//
// Validation and special cases follow the reference pricers one to one
// (yluoc/Quant-Kernel):
//   standard_monte_carlo.cpp:14-23   antithetic_variates.cpp:14-19
//   euler_maruyama.cpp:14-19         milstein.cpp:14-19
//   local_vol_monte_carlo.cpp:61-66  heston_monte_carlo.cpp:17-26
//   control_variates.cpp:13-18       importance_sampling.cpp:14-20
//   stratified_sampling.cpp:14-19    quasi_monte_carlo.cpp:13-18, 36-41
//   option_util.h:27-50, monte_carlo_methods/common/internal_util.h:13-26
// An invalid option gets NaN and the batch still returns QK_OK
// (qk_api.cpp:1152-1159 writes per-element results), t <= 1e-12 gives the
// undiscounted intrinsic value, and only standard MC has the zero-vol
// discounted-forward branch.  Everything else is simulated on the GPU.
#include "mc_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>

#include "mc_launch.h"
#include "qk_fault.h"

namespace qkb {

namespace {

constexpr double kEps = 1e-12;
constexpr int64_t kMaxTilesPerOption = 4096;
constexpr int64_t kTerminalItersPerThread = 4;
constexpr int64_t kMinTerminalTiles = 32;

double nan_value() { return std::numeric_limits<double>::quiet_NaN(); }

bool finite_bits(double x) {
    uint64_t bits;
    std::memcpy(&bits, &x, sizeof bits);
    return (bits & 0x7FF0000000000000ull) != 0x7FF0000000000000ull;
}

// std::max(a, b) == (a < b) ? b : a; the reference's NaN results follow it.
double smax(double a, double b) { return (a < b) ? b : a; }

double intrinsic(double x, double y, int32_t ot) {
    if (ot == 0) return smax(0.0, x - y);
    if (ot == 1) return smax(0.0, y - x);
    return nan_value();
}

bool valid_option_type(int32_t ot) { return ot == 0 || ot == 1; }

bool valid_common_inputs(double spot, double strike, double t, double vol, double r, double q,
                         int32_t ot) {
    if (!valid_option_type(ot)) return false;
    if (!finite_bits(spot) || !finite_bits(strike) || !finite_bits(t) || !finite_bits(vol) ||
        !finite_bits(r) || !finite_bits(q))
        return false;
    return spot > 0.0 && strike > 0.0 && t >= 0.0 && vol >= 0.0;
}

void set_const(McOption& o, double price) {
    o.mode = kModeConstant;
    o.const_price = price;
    o.tiles = 0;
    o.units = 0;
}

int32_t geti(const int32_t* a, int32_t i, int32_t dflt) { return a ? a[i] : dflt; }

int upt_for(int family, bool persistent, const LaunchConfig& cfg) {
    return persistent ? family_upt(family) : cfg.upt;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Device name (the autotuner's cache key), looked up once per device:
// cudaGetDeviceProperties costs milliseconds.
std::string device_name(int dev) {
    static std::mutex mu;
    static std::map<int, std::string> names;
    std::lock_guard<std::mutex> lk(mu);
    auto it = names.find(dev);
    if (it != names.end()) return it->second;
    cudaDeviceProp prop;
    std::string s = cudaGetDeviceProperties(&prop, dev) == cudaSuccess ? prop.name : "unknown";
    for (char& c : s)
        if (c == ' ' || c == '|') c = '_';
    names[dev] = s;
    return s;
}

}  // namespace

// Packs option i: validation, special cases and model constants; the tile
// geometry is filled by tile_option().
McOption pack_option(const BatchInput& in, int32_t i, bool anti_stepwise) {
    McOption o;
    std::memset(&o, 0, sizeof o);
    const int32_t m = in.model ? in.model[i] : in.uniform_model;
    o.model = m;
    o.option_type = in.option_type[i];
    o.paths = in.paths[i];
    o.seed = in.seed ? in.seed[i] : 0;  // the quasi-Monte Carlo calls take no seed
    o.spot = in.spot[i];
    o.strike = in.strike[i];
    o.mode = kModeSimulate;
    const double spot = in.spot[i], strike = in.strike[i], t = in.t[i];
    const int32_t ot = o.option_type, paths = o.paths;

    if (m == kStandard || m == kAntithetic || m == kTerminalPlain) {
        const double vol = in.vol[i], r = in.r[i], q = in.q[i];
        o.steps = 1;
        if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths <= 1) {
            set_const(o, nan_value());
            return o;
        }
        if (t <= kEps) {
            set_const(o, intrinsic(spot, strike, ot));
            return o;
        }
        if (m == kStandard && vol <= kEps) {
            const double fwd = spot * std::exp((r - q) * t);
            set_const(o, std::exp(-r * t) * intrinsic(fwd, strike, ot));
            return o;
        }
        o.disc = std::exp(-r * t);
        o.antithetic = (m != kTerminalPlain) ? 1 : 0;
        const int32_t n_norm = o.antithetic ? paths - paths / 2 : paths;
        o.units = (int32_t)(((int64_t)n_norm + 3) / 4);
        o.samples = o.antithetic ? paths / 2 : paths;
        // model_concepts.h:93-102, evaluated in the same order, kept in FP64
        o.d[0] = (r - q - 0.5 * vol * vol) * t;
        o.d[1] = vol * std::sqrt(smax(t, 0.0));
        return o;
    }
    if (m == kEuler || m == kMilstein || m == kLocalVol) {
        const double vol = in.vol[i], r = in.r[i], q = in.q[i];
        const int32_t steps = geti(in.steps, i, 0);
        o.steps = steps;
        if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) ||
            !(paths > 1 && steps > 0 && steps <= kMaxSteps)) {
            set_const(o, nan_value());
            return o;
        }
        if (t <= kEps) {
            set_const(o, intrinsic(spot, strike, ot));
            return o;
        }
        o.disc = std::exp(-r * t);
        o.antithetic = anti_stepwise ? 1 : 0;
        o.units = o.antithetic ? paths - paths / 2 : paths;
        o.samples = o.antithetic ? paths / 2 : paths;
        const double dt = t / (double)steps;
        const double sq = std::sqrt(dt);
        const double c = (m == kMilstein) ? 0.5 * vol * vol * dt : 0.0;
        o.p[0] = (float)((r - q) * dt - c);
        o.p[1] = (float)(vol * sq);
        o.p[2] = (float)(1e-12 / spot);
        o.p[3] = (float)c;
        return o;
    }
    if (m == kHeston || m == kHestonLrDelta) {
        const double r = in.r[i], q = in.q[i];
        const double v0 = in.v0[i], kappa = in.kappa[i], theta = in.theta[i];
        const double sigma = in.sigma[i], rho = in.rho[i];
        const int32_t steps = geti(in.steps, i, 0);
        o.steps = steps;
        // heston_monte_carlo.cpp:18-24 -- no finiteness test: a NaN passes the
        // comparisons and flows through the simulation as in the reference.
        // heston_lr_delta.cpp:46-53 adds weight_clip <= 0 -> NaN; a NaN clip
        // propagates to a NaN delta there, so it is rejected here.
        const double clip = (m == kHestonLrDelta) ? (in.weight_clip ? in.weight_clip[i] : in.vol[i]) : 1.0;
        if (!valid_option_type(ot) || spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0 ||
            kappa < 0.0 || theta < 0.0 || sigma < 0.0 || rho < -1.0 || rho > 1.0 ||
            !(paths > 1 && steps > 0 && steps <= kMaxSteps) || !(clip > 0.0)) {
            set_const(o, nan_value());
            return o;
        }
        if (t <= kEps) {
            if (m == kHestonLrDelta)  // heston_lr_delta.cpp:56-60: intrinsic delta
                set_const(o, ot == 0 ? (spot > strike ? 1.0 : 0.0) : (spot < strike ? -1.0 : 0.0));
            else
                set_const(o, intrinsic(spot, strike, ot));
            return o;
        }
        if (m == kHestonLrDelta && !(std::sqrt(smax(v0, 0.0)) > 1e-15)) {
            set_const(o, 0.0);  // every score is 0 (heston_lr_delta.cpp:91-93)
            return o;
        }
        if (m == kHestonLrDelta) o.weight_clip = clip;
        o.disc = std::exp(-r * t);
        o.antithetic = anti_stepwise ? 1 : 0;
        o.units = o.antithetic ? paths - paths / 2 : paths;
        o.samples = o.antithetic ? paths / 2 : paths;
        const double dt = t / (double)steps;
        const double sq = std::sqrt(dt);
        o.p[0] = (float)((r - q) * dt);
        o.p[1] = (float)(0.5 * dt);
        o.p[2] = (float)sq;
        o.p[3] = (float)(kappa * dt);
        o.p[4] = (float)(kappa * theta * dt);
        o.p[5] = (float)(sigma * sq);
        o.p[6] = (float)rho;
        o.p[7] = (float)std::sqrt(smax(1.0 - rho * rho, 0.0));
        o.p[8] = (float)v0;
        o.p[9] = (float)std::log(1e-12 / spot);
        return o;
    }
    if (m >= kControlVariates && m <= kQmcHalton) {
        const double vol = in.vol[i], r = in.r[i], q = in.q[i];
        const double shift = (m == kImportanceSampling) ? (in.shift ? in.shift[i] : in.v0[i]) : 0.0;
        o.steps = 1;
        // control variates need three paths (control_variates.cpp:14-15); a
        // non-finite shift is rejected (importance_sampling.cpp:15-16)
        const int32_t min_paths = (m == kControlVariates) ? 3 : 2;
        if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths < min_paths ||
            !finite_bits(shift)) {
            set_const(o, nan_value());
            return o;
        }
        if (t <= kEps) {
            set_const(o, intrinsic(spot, strike, ot));
            return o;
        }
        o.disc = std::exp(-r * t);
        o.antithetic = 0;
        o.units = (int32_t)(((int64_t)paths + 3) / 4);
        o.samples = paths;
        // model_concepts.h:93-102, evaluated in the same order
        o.d[0] = (r - q - 0.5 * vol * vol) * t;
        o.d[1] = vol * std::sqrt(smax(t, 0.0));
        o.d[2] = shift;
        o.d[3] = spot * std::exp((r - q) * t);
        return o;
    }
    set_const(o, nan_value());  // unknown model code
    return o;
}

int32_t tile_option(McOption& o, int block, int upt) {
    if (o.mode != kModeSimulate || o.units <= 0) {
        o.tiles = 0;
        o.unit_iters = 0;
        return 0;
    }
    const int64_t per_iter = (int64_t)block * upt;
    const int64_t units = o.units;
    int64_t iters = (units + per_iter * kMaxTilesPerOption - 1) / (per_iter * kMaxTilesPerOption);
    if (iters < 1) iters = 1;
    // Terminal units (one quad of paths, no time steps) are cheap next to a
    // tile's fixed cost -- record load, option search and the double-double
    // CTA reduction -- so large terminal options give each thread several
    // units, while keeping at least kMinTerminalTiles tiles to spread over
    // the SMs.  A function of the option alone, like the rest of the
    // geometry: a batch and a scalar call tile an option the same way.
    const int fam = family_of(o.model);
    if (fam == kFamTerminal || fam == kFamVr) {
        const int64_t cap = units / (per_iter * kMinTerminalTiles);
        const int64_t want = std::min<int64_t>(kTerminalItersPerThread, cap);
        if (want > iters) iters = want;
    }
    const int64_t tile_units = per_iter * iters;
    o.unit_iters = (int32_t)iters;
    o.tiles = (int32_t)((units + tile_units - 1) / tile_units);
    return o.tiles;
}

// ----------------------------------------------------------------------------
cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    release();
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = injected_fault(kFaultAlloc);
    if (e == cudaSuccess) e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        return e;
    }
    cap = want;
    return cudaSuccess;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}
cudaError_t PinnedBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    release();
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = injected_fault(kFaultAlloc);
    if (e == cudaSuccess) e = cudaMallocHost(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        return e;
    }
    cap = want;
    return cudaSuccess;
}
void PinnedBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

// ----------------------------------------------------------------------------
// Default launch shapes (measured on B200; the autotuner may override them).
// 128-thread CTAs: at the Heston benchmark (1024 options x 262144 paths x 200
// steps) block 128 ran 2.4% faster than 256 with the same registers (six CTAs
// of 128 per SM instead of three of 256: finer tiles, a shorter tail), and the
// autotuner picked it for the mixed-model batch too.  One block size for every
// family, and each family's units per thread from family_upt(), keep the
// persistent and single-family tilings identical, so both give the same bits.
LaunchConfig default_config(int family) {
    LaunchConfig c;
    c.block = 128;
    c.upt = family_upt(family);
    return c;
}

namespace {
std::mutex g_tune_mu;
std::map<std::string, LaunchConfig>& tune_map() {
    static std::map<std::string, LaunchConfig> m;
    return m;
}
bool g_tune_loaded = false;

const char* tune_path() {
    const char* p = std::getenv("QK_B200_TUNE_CACHE");
    return (p && *p) ? p : nullptr;
}

void load_tune_file_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = tune_path();
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char line[600], key[512];
    // one entry per line: <key> <block> <upt> [<step unroll>]
    while (std::fgets(line, sizeof line, f)) {
        int block = 0, upt = 0, su = 1;
        if (std::sscanf(line, "%511s %d %d %d", key, &block, &upt, &su) < 3) continue;
        if ((block == 128 || block == 256) &&
            (upt == 1 || upt == 2 || upt == 4 || upt == kUptPersistent || upt == kUptFamilyGrids) &&
            (su == 1 || (su == 2 && (upt == 1 || upt == 2 || upt == 4))))
            tune_map()[key] = LaunchConfig{block, upt, su};
    }
    std::fclose(f);
}
}  // namespace

bool tuned_config(const std::string& key, LaunchConfig* out) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    load_tune_file_locked();
    auto it = tune_map().find(key);
    if (it == tune_map().end()) return false;
    *out = it->second;
    return true;
}

void store_tuned_config(const std::string& key, const LaunchConfig& cfg) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    load_tune_file_locked();
    tune_map()[key] = cfg;
    const char* path = tune_path();
    if (!path) return;
    FILE* f = std::fopen(path, "w");
    if (!f) return;
    for (const auto& kv : tune_map())
        std::fprintf(f, "%s %d %d %d\n", kv.first.c_str(), kv.second.block, kv.second.upt,
                     kv.second.su);
    std::fclose(f);
}

// ----------------------------------------------------------------------------
Plan::~Plan() { release(); }

cudaError_t Plan::release() {
    drop_graph();
    if (device_ >= 0) {
        DeviceGuard g(device_);
        d_opts_.release();
        d_tile_begin_.release();
        d_partials_.release();
        d_price_.release();
        d_se_.release();
        d_counter_.release();
        d_out_index_.release();
        h_out_index_.release();
        d_groups_.release();
        h_groups_.release();
        h_opts_.release();
        h_tile_begin_.release();
        h_price_.release();
        h_se_.release();
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (stream_) cudaStreamDestroy(stream_);
    }
    ev0_ = ev1_ = nullptr;
    stream_ = nullptr;
    device_ = -1;
    return cudaSuccess;
}

void Plan::drop_graph() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    graph_exec_ = nullptr;
    graph_ = nullptr;
}

cudaError_t Plan::ensure_stream() {
    if (stream_) return cudaSuccess;
    cudaError_t e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    e = cudaEventCreate(&ev0_);
    if (e != cudaSuccess) return e;
    return cudaEventCreate(&ev1_);
}

cudaError_t Plan::build(const BatchInput& in, int32_t flags, std::string* err) {
    NvtxRange range("qk.build");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (device_ >= 0 && device_ != dev) release();
    device_ = dev;
    drop_graph();
    e = ensure_stream();
    if (e != cudaSuccess) return e;

    flags_ = flags;
    n_ = in.n;
    opts_.resize((size_t)in.n);
    const bool anti_stepwise = (flags & kFlagNoAntithetic) == 0;
    int fam = -2;  // -2: none yet, -1: mixed
    bool anti = true;
    path_steps_ = 0;
    for (int32_t i = 0; i < in.n; ++i) {
        McOption o = pack_option(in, i, anti_stepwise);
        if (o.mode == kModeSimulate) {
            const int f = family_of(o.model);
            const bool a = o.antithetic != 0;
            if (fam == -2) {
                fam = f;
                anti = a;
            } else if (fam != f || anti != a) {
                fam = -1;
            }
            path_steps_ += (int64_t)o.paths * (int64_t)std::max(o.steps, 1);
        }
        opts_[(size_t)i] = o;
    }
    family_ = (fam == -2) ? kFamTerminal : fam;
    anti_ = anti;
    persistent_ = (fam == -1) || (flags & kFlagPersistent);
    if (persistent_) {
        const bool grids = (flags & kFlagFamilyGrids) && !(flags & kFlagPersistent);
        cfg_ = LaunchConfig{default_config(kFamHeston).block,
                            grids ? kUptFamilyGrids : kUptPersistent};
    } else {
        cfg_ = default_config(family_);
    }
    const std::string key = device_name(device_) + "|" + (persistent_ ? "persistent" : std::to_string(family_)) +
                            "|" + (anti_ ? "anti" : "plain");
    LaunchConfig tuned;
    if (tuned_config(key, &tuned)) {
        cfg_.block = tuned.block;
        // a multi-family plan takes the tuned mode unless the caller asked
        // for the persistent kernel explicitly
        if (!persistent_ || (tuned.upt <= 0 && !(flags & (kFlagPersistent | kFlagFamilyGrids))))
            cfg_.upt = tuned.upt;
        if (persistent_ && cfg_.upt > 0) cfg_.upt = kUptPersistent;
        cfg_.su = (!persistent_ && step_unroll2_compiled(family_, cfg_.upt)) ? tuned.su : 1;
    }
    // QK_PLAN_STEP_UNROLL2: two step blocks per loop iteration where compiled
    if ((flags & kFlagStepUnroll2) && !persistent_ && step_unroll2_compiled(family_, cfg_.upt))
        cfg_.su = 2;
    e = layout_tiles(cfg_);
    if (e != cudaSuccess) return e;
    if ((flags & kFlagAutotune) && n_tiles_ > 0) {
        e = autotune();
        if (e != cudaSuccess) return e;
        store_tuned_config(key, cfg_);
    }
    (void)err;
    return cudaSuccess;
}

// Work order of the persistent kernel: heavy families first, and within a
// family the costliest tiles first, so that the last tiles handed out are
// short ones (a small tail) and co-resident CTAs mostly run the same code.
static int family_rank(int fam) {
    switch (fam) {
        case kFamHeston:
        case kFamHestonLr: return 0;
        case kFamMilstein: return 1;
        case kFamEuler: return 2;
        case kFamVr: return 3;
        default: return 4;  // terminal
    }
}

cudaError_t Plan::layout_tiles(const LaunchConfig& cfg) {
    const int32_t n = n_;
    shard_world_ = 0;  // the tile geometry may change: partitions are stale
    shard_bounds_.clear();
    // tile geometry per option (independent of the order)
    for (int32_t i = 0; i < n; ++i) {
        McOption& o = opts_[(size_t)i];
        tile_option(o, cfg.block, upt_for(family_of(o.model), persistent_, cfg));
    }
    order_.resize((size_t)n);
    for (int32_t i = 0; i < n; ++i) order_[(size_t)i] = i;
    if (persistent_) {
        auto tile_cost = [&](const McOption& o) {
            return (double)o.unit_iters * (double)std::max(o.steps, 1);
        };
        std::stable_sort(order_.begin(), order_.end(), [&](int32_t a, int32_t b) {
            const McOption& oa = opts_[(size_t)a];
            const McOption& ob = opts_[(size_t)b];
            const int ra = family_rank(family_of(oa.model)), rb = family_rank(family_of(ob.model));
            if (ra != rb) return ra < rb;
            const int fa = family_of(oa.model), fb = family_of(ob.model);
            if (fa != fb) return fa < fb;  // Heston before its LR-delta variant
            if (oa.antithetic != ob.antithetic) return oa.antithetic > ob.antithetic;
            return tile_cost(oa) > tile_cost(ob);
        });
    }
    int64_t total = 0;
    std::vector<int64_t> begin((size_t)n + 1);
    for (int32_t k = 0; k < n; ++k) {
        McOption& o = opts_[(size_t)order_[(size_t)k]];
        begin[(size_t)k] = total;
        o.tile_begin = total;
        total += o.tiles;
    }
    begin[(size_t)n] = total;
    n_tiles_ = total;
    groups_.clear();
    if (persistent_) {
        for (int32_t k = 0; k < n; ++k) {
            const McOption& o = opts_[(size_t)order_[(size_t)k]];
            if (o.tiles <= 0) continue;  // constant results: finalize only
            const int fam = family_of(o.model);
            const bool anti = o.antithetic != 0;
            if (groups_.empty() || groups_.back().family != fam || groups_.back().anti != anti ||
                groups_.back().opt_hi != k)
                groups_.push_back(Group{fam, anti, k, k, o.tile_begin, o.tile_begin});
            groups_.back().opt_hi = k + 1;
            groups_.back().tile_hi = o.tile_begin + o.tiles;
        }
    }

    cudaError_t e;
    const size_t opt_bytes = sizeof(McOption) * (size_t)std::max(n, 1);
    const size_t tb_bytes = sizeof(int64_t) * ((size_t)n + 1);
    if ((e = d_opts_.ensure(opt_bytes)) != cudaSuccess) return e;
    if ((e = d_tile_begin_.ensure(tb_bytes)) != cudaSuccess) return e;
    if ((e = d_partials_.ensure(sizeof(TilePartial) * (size_t)std::max<int64_t>(total, 1))) != cudaSuccess) return e;
    if ((e = d_price_.ensure(sizeof(double) * (size_t)std::max(n, 1))) != cudaSuccess) return e;
    if ((e = d_se_.ensure(sizeof(double) * (size_t)std::max(n, 1))) != cudaSuccess) return e;
    if ((e = d_counter_.ensure(sizeof(unsigned long long))) != cudaSuccess) return e;
    if ((e = h_opts_.ensure(opt_bytes)) != cudaSuccess) return e;
    if ((e = h_tile_begin_.ensure(tb_bytes)) != cudaSuccess) return e;
    const size_t ix_bytes = sizeof(int32_t) * (size_t)std::max(n, 1);
    if (persistent_) {
        if ((e = d_out_index_.ensure(ix_bytes)) != cudaSuccess) return e;
        if ((e = h_out_index_.ensure(ix_bytes)) != cudaSuccess) return e;
        if ((e = d_groups_.ensure(sizeof(GroupTable))) != cudaSuccess) return e;
        if ((e = h_groups_.ensure(sizeof(GroupTable))) != cudaSuccess) return e;
    }
    // The previous upload from these staging buffers may still be in flight.
    if ((e = cudaStreamSynchronize(stream_)) != cudaSuccess) return e;
    McOption* h_rec = static_cast<McOption*>(h_opts_.p);
    for (int32_t k = 0; k < n; ++k) h_rec[k] = opts_[(size_t)order_[(size_t)k]];
    std::memcpy(h_tile_begin_.p, begin.data(), tb_bytes);
    if (persistent_) {
        std::memcpy(h_out_index_.p, order_.data(), sizeof(int32_t) * (size_t)n);
        if ((e = cudaMemcpyAsync(d_out_index_.p, h_out_index_.p, sizeof(int32_t) * (size_t)n,
                                 cudaMemcpyHostToDevice, stream_)) != cudaSuccess)
            return e;
        // the persistent kernel's group table (at most 2 groups per family:
        // antithetic and plain; constant records carry no tiles)
        GroupTable* gt = static_cast<GroupTable*>(h_groups_.p);
        std::memset(gt, 0, sizeof(GroupTable));
        if (groups_.size() > (size_t)kMaxGroups) return cudaErrorInvalidConfiguration;
        gt->count = (int32_t)groups_.size();
        for (size_t k = 0; k < groups_.size(); ++k) {
            gt->code[k] = groups_[k].family * 2 + (groups_[k].anti ? 1 : 0);
            gt->opt_lo[k] = groups_[k].opt_lo;
            gt->opt_hi[k] = groups_[k].opt_hi;
            gt->tile_hi[k] = groups_[k].tile_hi;
        }
        if ((e = cudaMemcpyAsync(d_groups_.p, h_groups_.p, sizeof(GroupTable),
                                 cudaMemcpyHostToDevice, stream_)) != cudaSuccess)
            return e;
    }
    if ((e = cudaMemcpyAsync(d_opts_.p, h_opts_.p, sizeof(McOption) * (size_t)n, cudaMemcpyHostToDevice, stream_)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(d_tile_begin_.p, h_tile_begin_.p, tb_bytes, cudaMemcpyHostToDevice, stream_)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d_counter_.p, 0, sizeof(unsigned long long), stream_)) != cudaSuccess) return e;
    counter_ready_ = true;
    if (persistent_ && cfg.upt == kUptPersistent) {
        max_ctas_ = max_resident_ctas(-1, cfg.block, 0, device_);
        if (max_ctas_ <= 0) return cudaErrorInvalidConfiguration;
    } else {
        max_ctas_ = std::numeric_limits<int32_t>::max();
    }
    cfg_ = cfg;
    return cudaSuccess;
}

cudaError_t Plan::launch_all(cudaStream_t st, bool timing) {
    if (cudaError_t fe = injected_fault(kFaultLaunch)) return fe;
    SimArgs a;
    a.opts = static_cast<const McOption*>(d_opts_.p);
    a.tile_begin = static_cast<const int64_t*>(d_tile_begin_.p);
    a.n = n_;
    a.n_tiles = n_tiles_;
    a.partials = static_cast<TilePartial*>(d_partials_.p);
    a.max_ctas = max_ctas_;
    unsigned long long* counter = static_cast<unsigned long long*>(d_counter_.p);
    cudaError_t e = cudaSuccess;
    if (timing && (e = cudaEventRecord(ev0_, st)) != cudaSuccess) return e;
    const bool use_counter = persistent_ && cfg_.upt == kUptPersistent;
    if (n_tiles_ > 0) {
        if (use_counter) {
            e = launch_persistent(cfg_.block, a, static_cast<const GroupTable*>(d_groups_.p),
                                  counter, st);
        } else if (persistent_) {
            // one grid per (family, antithetic) group, back to back
            for (const Group& g : groups_) {
                SimArgs ga = a;
                ga.opts = a.opts + g.opt_lo;
                ga.tile_begin = a.tile_begin + g.opt_lo;
                ga.n = g.opt_hi - g.opt_lo;
                ga.tile0 = g.tile_lo;
                ga.n_tiles = g.tile_hi - g.tile_lo;
                e = launch_simulate(g.family, g.anti, cfg_.block,
                                    upt_for(g.family, true, cfg_), 1, ga, st);
                if (e != cudaSuccess) return e;
            }
        } else {
            e = launch_simulate(family_, anti_, cfg_.block, cfg_.upt, cfg_.su, a, st);
        }
        if (e != cudaSuccess) return e;
    }
    if (timing && (e = cudaEventRecord(ev1_, st)) != cudaSuccess) return e;
    // persistent plans hold the records in work order; the finalize kernel
    // scatters results back to the caller's order
    const int32_t* out_index = persistent_ ? static_cast<const int32_t*>(d_out_index_.p) : nullptr;
    return launch_finalize(a.opts, n_, a.partials, d_price(), d_se(), out_index,
                           use_counter ? counter : nullptr, st);
}

void partition_by_cost(const double* cost, int64_t n, int world, int64_t* bounds) {
    bounds[0] = 0;
    if (world <= 1 || n <= 0) {
        for (int r = 1; r <= world; ++r) bounds[r] = n > 0 ? n : 0;
        return;
    }
    double total = 0.0;
    for (int64_t i = 0; i < n; ++i) total += cost[i];
    int r = 1;
    double before = 0.0;  // cost of items [0, i)
    for (int64_t i = 0; i < n && r < world; ++i) {
        const double after = before + cost[i];
        // every target that item i reaches: cut before or after it, whichever
        // cumulative cost is nearer the target
        while (r < world && after >= total * (double)r / (double)world) {
            const double target = total * (double)r / (double)world;
            const int64_t cut = (target - before <= after - target) ? i : i + 1;
            bounds[r] = std::max(cut, bounds[r - 1]);
            ++r;
        }
        before = after;
    }
    for (; r < world; ++r) bounds[r] = n;
    bounds[world] = n;
}

const std::vector<int64_t>& Plan::shard_bounds(int world) {
    if (shard_world_ == world && (int)shard_bounds_.size() == world + 1) return shard_bounds_;
    // path-steps of every tile, in work order (the last tile of an option
    // holds the remainder of its units)
    std::vector<double> cost((size_t)std::max<int64_t>(n_tiles_, 0));
    for (int32_t k = 0; k < n_; ++k) {
        const McOption& o = opts_[(size_t)order_[(size_t)k]];
        if (o.tiles <= 0) continue;
        const int64_t per_tile = (int64_t)cfg_.block *
                                 upt_for(family_of(o.model), persistent_, cfg_) * o.unit_iters;
        const double steps = (double)std::max(o.steps, 1);
        for (int32_t t = 0; t < o.tiles; ++t) {
            const int64_t left = (int64_t)o.units - (int64_t)t * per_tile;
            cost[(size_t)(o.tile_begin + t)] = (double)std::min(per_tile, left) * steps;
        }
    }
    shard_bounds_.assign((size_t)world + 1, 0);
    partition_by_cost(cost.data(), n_tiles_, world, shard_bounds_.data());
    shard_world_ = world;
    return shard_bounds_;
}

cudaError_t Plan::order_after_upload(cudaStream_t st) {
    if (!st || st == stream_) return cudaSuccess;
    cudaEvent_t ready;
    cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(ready, stream_);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ready, 0);
    cudaEventDestroy(ready);
    return e;
}

cudaError_t Plan::launch_tiles(cudaStream_t st, int64_t lo, int64_t hi, bool timing) {
    if (cudaError_t fe = injected_fault(kFaultLaunch)) return fe;
    SimArgs a;
    a.opts = static_cast<const McOption*>(d_opts_.p);
    a.tile_begin = static_cast<const int64_t*>(d_tile_begin_.p);
    a.n = n_;
    a.partials = static_cast<TilePartial*>(d_partials_.p);
    a.max_ctas = std::numeric_limits<int32_t>::max();
    cudaError_t e = cudaSuccess;
    if (timing && (e = cudaEventRecord(ev0_, st)) != cudaSuccess) return e;
    if (!persistent_) {
        a.tile0 = lo;
        a.n_tiles = hi - lo;
        if (a.n_tiles > 0) e = launch_simulate(family_, anti_, cfg_.block, cfg_.upt, cfg_.su, a, st);
    } else {
        for (const Group& g : groups_) {
            const int64_t t0 = std::max(lo, g.tile_lo), t1 = std::min(hi, g.tile_hi);
            if (t1 <= t0) continue;
            SimArgs ga = a;
            ga.opts = a.opts + g.opt_lo;
            ga.tile_begin = a.tile_begin + g.opt_lo;
            ga.n = g.opt_hi - g.opt_lo;
            ga.tile0 = t0;
            ga.n_tiles = t1 - t0;
            e = launch_simulate(g.family, g.anti, cfg_.block, upt_for(g.family, true, cfg_), 1, ga,
                                st);
            if (e != cudaSuccess) return e;
        }
    }
    if (e != cudaSuccess) return e;
    if (timing && (e = cudaEventRecord(ev1_, st)) != cudaSuccess) return e;
    return cudaSuccess;
}

cudaError_t Plan::launch_finalize_all(cudaStream_t st) {
    const int32_t* out_index = persistent_ ? static_cast<const int32_t*>(d_out_index_.p) : nullptr;
    return launch_finalize(static_cast<const McOption*>(d_opts_.p), n_,
                           static_cast<const TilePartial*>(d_partials_.p), d_price(), d_se(),
                           out_index, nullptr, st);
}

cudaError_t Plan::capture_graph() {
    drop_graph();
    cudaError_t e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t le = launch_all(stream_, false);
    e = cudaStreamEndCapture(stream_, &graph_);
    if (le != cudaSuccess) return le;
    if (e != cudaSuccess) return e;
    return cudaGraphInstantiate(&graph_exec_, graph_, 0);
}

cudaError_t Plan::execute(cudaStream_t stream) {
    NvtxRange range("qk.execute");
    if (device_ < 0) return cudaErrorInvalidResourceHandle;
    DeviceGuard g(device_);
    cudaStream_t st = stream ? stream : stream_;
    // order this execute after the plan's own uploads
    if (cudaError_t oe = order_after_upload(st)) return oe;
    const bool timing = (flags_ & kFlagTiming) != 0;
    cudaError_t e;
    if (flags_ & kFlagGraph) {
        if (!graph_exec_) {
            if ((e = cudaStreamSynchronize(stream_)) != cudaSuccess) return e;
            if ((e = capture_graph()) != cudaSuccess) return e;
        }
        if (timing) cudaEventRecord(ev0_, st);
        e = cudaGraphLaunch(graph_exec_, st);
        if (timing) cudaEventRecord(ev1_, st);
    } else {
        e = launch_all(st, timing);
    }
    if (e != cudaSuccess) return e;
    last_stream_ = st;
    return cudaSuccess;
}

cudaError_t Plan::results(double* out_price, double* out_se) {
    NvtxRange range("qk.results");
    if (device_ < 0) return cudaErrorInvalidResourceHandle;
    if (cudaError_t fe = injected_fault(kFaultCopy)) return fe;
    DeviceGuard g(device_);
    cudaStream_t st = last_stream_ ? last_stream_ : stream_;
    const size_t bytes = sizeof(double) * (size_t)n_;
    cudaError_t e;
    if ((e = h_price_.ensure(bytes)) != cudaSuccess) return e;
    if (out_se && (e = h_se_.ensure(bytes)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(h_price_.p, d_price_.p, bytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if (out_se && (e = cudaMemcpyAsync(h_se_.p, d_se_.p, bytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    std::memcpy(out_price, h_price_.p, bytes);
    if (out_se) std::memcpy(out_se, h_se_.p, bytes);
    if (flags_ & kFlagTiming) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess) last_ms_ = ms;
    }
    return cudaSuccess;
}

cudaError_t Plan::sync_stats() {
    if (device_ < 0) return cudaErrorInvalidResourceHandle;
    DeviceGuard g(device_);
    if (!(flags_ & kFlagTiming)) return cudaSuccess;
    cudaError_t e = cudaEventSynchronize(ev1_);
    if (e != cudaSuccess) return e;
    float ms = 0.0f;
    e = cudaEventElapsedTime(&ms, ev0_, ev1_);
    if (e == cudaSuccess) last_ms_ = ms;
    return e;
}

// Times every candidate launch shape on this plan (one warm-up and the best
// of three timed runs each) and keeps the fastest.  Tile geometry follows the shape, so the
// plan is re-laid-out per candidate; per-path results do not change.
cudaError_t Plan::autotune() {
    std::vector<LaunchConfig> cands;
    if (persistent_) {
        cands = {LaunchConfig{128, kUptPersistent}, LaunchConfig{256, kUptPersistent}};
        if (!(flags_ & kFlagPersistent)) {
            cands.push_back(LaunchConfig{128, kUptFamilyGrids});
            cands.push_back(LaunchConfig{256, kUptFamilyGrids});
        }
    } else {
        // block size x units per thread, and for the stepwise families the
        // step unrolling (one or two Philox step blocks per loop iteration)
        for (int b : {128, 256})
            for (int u : {1, 2, 4}) {
                cands.push_back(LaunchConfig{b, u, 1});
                if (step_unroll2_compiled(family_, u)) cands.push_back(LaunchConfig{b, u, 2});
            }
    }
    LaunchConfig best = cfg_;
    float best_ms = std::numeric_limits<float>::max();
    cudaError_t e;
    for (const LaunchConfig& c : cands) {
        if ((e = layout_tiles(c)) != cudaSuccess) return e;
        if ((e = launch_all(stream_, false)) != cudaSuccess) return e;  // warm-up
        float ms = std::numeric_limits<float>::max();
        for (int rep = 0; rep < 3; ++rep) {  // best of three: shapes differ by ~1%
            if ((e = launch_all(stream_, true)) != cudaSuccess) return e;
            if ((e = cudaEventSynchronize(ev1_)) != cudaSuccess) return e;
            float t = 0.0f;
            if ((e = cudaEventElapsedTime(&t, ev0_, ev1_)) != cudaSuccess) return e;
            ms = std::min(ms, t);
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    return layout_tiles(best);
}

// ----------------------------------------------------------------------------
Plan* thread_scratch_plan(int device) {
    thread_local std::map<int, std::unique_ptr<Plan>> plans;
    auto& p = plans[device];
    if (!p) p.reset(new Plan());
    return p.get();
}

}  // namespace qkb
