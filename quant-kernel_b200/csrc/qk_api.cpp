// qk_api.cpp -- extern "C" boundary of libqk_b200.so.
//
// Error machinery restates yluoc/Quant-Kernel cpp/src/qk_api.cpp:19-117: a
// thread-local 256-byte message, "null pointer: <param>" for the first null
// argument in declaration order (QK_ERR_NULL_PTR), checked before the size,
// then "bad batch size: <n>" for n <= 0 (QK_ERR_BAD_SIZE).  Invalid elements
// get NaN and the call still returns QK_OK.  CUDA failures, which have no
// reference counterpart, return QK_ERR_RUNTIME_INIT with "cuda error: ...".
#include "../../include/qk_api.h"

#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "cf_kernels.h"
#include "mc_noalloc.h"
#include "qk_dist.h"
#include "qk_error.h"
#include "qk_handles.h"

namespace {

using qkb::fail_cuda;
using qkb::fail_null;
using qkb::fail_size;
using qkb::set_error_fmt;

struct NamedPtr {
    const void* p;
    const char* name;
};

// First null pointer in declaration order, as QK_BATCH_NULL_CHECK does.
template <size_t N>
int32_t check_nulls(const NamedPtr (&ptrs)[N]) {
    for (size_t i = 0; i < N; ++i)
        if (!ptrs[i].p) return fail_null(ptrs[i].name);
    return QK_OK;
}

const QKPluginAPI k_plugin_api = {QK_ABI_MAJOR, QK_ABI_MINOR, "quantkernel.b200.mcm.v1"};

double nan_value() { return std::numeric_limits<double>::quiet_NaN(); }

// Runs one batch through the calling thread's scratch plan.
int32_t run_batch(const qkb::BatchInput& in, int32_t flags, double* out_prices, double* out_se,
                  const char* where) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_cuda(e, where);
    qkb::Plan* plan = qkb::thread_scratch_plan(dev);
    std::string err;
    if ((e = plan->build(in, flags, &err)) != cudaSuccess) return fail_cuda(e, where);
    if ((e = plan->execute(nullptr)) != cudaSuccess) return fail_cuda(e, where);
    if ((e = plan->results(out_prices, out_se)) != cudaSuccess) return fail_cuda(e, where);
    return QK_OK;
}

qkb::BatchInput bsm_input(int32_t model, const double* spot, const double* strike, const double* t,
                          const double* vol, const double* r, const double* q,
                          const int32_t* option_type, const int32_t* paths, const int32_t* steps,
                          const uint64_t* seed, int32_t n) {
    qkb::BatchInput in;
    in.uniform_model = model;
    in.spot = spot;
    in.strike = strike;
    in.t = t;
    in.vol = vol;
    in.r = r;
    in.q = q;
    in.option_type = option_type;
    in.paths = paths;
    in.steps = steps;
    in.seed = seed;
    in.n = n;
    return in;
}

qkb::BatchInput heston_input(const double* spot, const double* strike, const double* t,
                             const double* r, const double* q, const double* v0,
                             const double* kappa, const double* theta, const double* sigma,
                             const double* rho, const int32_t* option_type, const int32_t* paths,
                             const int32_t* steps, const uint64_t* seed, int32_t n) {
    qkb::BatchInput in;
    in.uniform_model = qkb::kHeston;
    in.spot = spot;
    in.strike = strike;
    in.t = t;
    in.r = r;
    in.q = q;
    in.v0 = v0;
    in.kappa = kappa;
    in.theta = theta;
    in.sigma = sigma;
    in.rho = rho;
    in.option_type = option_type;
    in.paths = paths;
    in.steps = steps;
    in.seed = seed;
    in.n = n;
    return in;
}

// Terminal models: (spot, strike, t, vol, r, q, option_type, paths, seed).
int32_t terminal_batch(int32_t model, const double* spot, const double* strike, const double* t,
                       const double* vol, const double* r, const double* q,
                       const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
                       int32_t n, double* out_prices, double* out_se, bool want_se,
                       const char* where) {
    if (want_se) {
        const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {vol, "vol"},
                                 {r, "r"}, {q, "q"}, {option_type, "option_type"},
                                 {paths, "paths"}, {seed, "seed"}, {out_prices, "out_prices"},
                                 {out_se, "out_stderr"}};
        if (int32_t rc = check_nulls(ptrs)) return rc;
    } else {
        const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {vol, "vol"},
                                 {r, "r"}, {q, "q"}, {option_type, "option_type"},
                                 {paths, "paths"}, {seed, "seed"}, {out_prices, "out_prices"}};
        if (int32_t rc = check_nulls(ptrs)) return rc;
    }
    if (n <= 0) return fail_size(n);
    return run_batch(bsm_input(model, spot, strike, t, vol, r, q, option_type, paths, nullptr, seed, n),
                     0, out_prices, out_se, where);
}

// One-factor stepwise models: (..., option_type, paths, steps, seed).
int32_t stepwise_batch(int32_t model, const double* spot, const double* strike, const double* t,
                       const double* vol, const double* r, const double* q,
                       const int32_t* option_type, const int32_t* paths, const int32_t* steps,
                       const uint64_t* seed, int32_t n, double* out_prices, double* out_se,
                       bool want_se, const char* where) {
    if (want_se) {
        const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {vol, "vol"},
                                 {r, "r"}, {q, "q"}, {option_type, "option_type"},
                                 {paths, "paths"}, {steps, "steps"}, {seed, "seed"},
                                 {out_prices, "out_prices"}, {out_se, "out_stderr"}};
        if (int32_t rc = check_nulls(ptrs)) return rc;
    } else {
        const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {vol, "vol"},
                                 {r, "r"}, {q, "q"}, {option_type, "option_type"},
                                 {paths, "paths"}, {steps, "steps"}, {seed, "seed"},
                                 {out_prices, "out_prices"}};
        if (int32_t rc = check_nulls(ptrs)) return rc;
    }
    if (n <= 0) return fail_size(n);
    return run_batch(bsm_input(model, spot, strike, t, vol, r, q, option_type, paths, steps, seed, n),
                     0, out_prices, out_se, where);
}

int32_t heston_batch(const double* spot, const double* strike, const double* t, const double* r,
                     const double* q, const double* v0, const double* kappa, const double* theta,
                     const double* sigma, const double* rho, const int32_t* option_type,
                     const int32_t* paths, const int32_t* steps, const uint64_t* seed, int32_t n,
                     double* out_prices, double* out_se, bool want_se, const char* where) {
    if (want_se) {
        const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {r, "r"},
                                 {q, "q"}, {v0, "v0"}, {kappa, "kappa"}, {theta, "theta"},
                                 {sigma, "sigma"}, {rho, "rho"}, {option_type, "option_type"},
                                 {paths, "paths"}, {steps, "steps"}, {seed, "seed"},
                                 {out_prices, "out_prices"}, {out_se, "out_stderr"}};
        if (int32_t rc = check_nulls(ptrs)) return rc;
    } else {
        const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {r, "r"},
                                 {q, "q"}, {v0, "v0"}, {kappa, "kappa"}, {theta, "theta"},
                                 {sigma, "sigma"}, {rho, "rho"}, {option_type, "option_type"},
                                 {paths, "paths"}, {steps, "steps"}, {seed, "seed"},
                                 {out_prices, "out_prices"}};
        if (int32_t rc = check_nulls(ptrs)) return rc;
    }
    if (n <= 0) return fail_size(n);
    return run_batch(heston_input(spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                                  paths, steps, seed, n),
                     0, out_prices, out_se, where);
}

// Terminal variance-reduction models.  Null checks in each reference batch's
// declaration order: (spot, strike, t, vol, r, q, option_type, paths,
// [shift,] [seed,] out_prices); the quasi-Monte Carlo calls take no seed.
int32_t vr_batch(int32_t model, const double* spot, const double* strike, const double* t,
                 const double* vol, const double* r, const double* q, const int32_t* option_type,
                 const int32_t* paths, const double* shift, const uint64_t* seed, int32_t n,
                 double* out_prices, double* out_se, bool want_se, const char* where) {
    const bool has_seed = model != qkb::kQmcSobol && model != qkb::kQmcHalton;
    const bool has_shift = model == qkb::kImportanceSampling;
    NamedPtr ptrs[12];
    int k = 0;
    for (const NamedPtr& np : {NamedPtr{spot, "spot"}, NamedPtr{strike, "strike"}, NamedPtr{t, "t"},
                               NamedPtr{vol, "vol"}, NamedPtr{r, "r"}, NamedPtr{q, "q"},
                               NamedPtr{option_type, "option_type"}, NamedPtr{paths, "paths"}})
        ptrs[k++] = np;
    if (has_shift) ptrs[k++] = NamedPtr{shift, "shift"};
    if (has_seed) ptrs[k++] = NamedPtr{seed, "seed"};
    ptrs[k++] = NamedPtr{out_prices, "out_prices"};
    if (want_se) ptrs[k++] = NamedPtr{out_se, "out_stderr"};
    for (int i = 0; i < k; ++i)
        if (!ptrs[i].p) return fail_null(ptrs[i].name);
    if (n <= 0) return fail_size(n);
    qkb::BatchInput in = bsm_input(model, spot, strike, t, vol, r, q, option_type, paths, nullptr,
                                   has_seed ? seed : nullptr, n);
    in.shift = shift;
    return run_batch(in, 0, out_prices, out_se, where);
}

// Mixed-model input: checks the arrays that the present models need.
int32_t mixed_input(const int32_t* model, const double* spot, const double* strike,
                    const double* t, const double* vol, const double* r, const double* q,
                    const double* v0, const double* kappa, const double* theta,
                    const double* sigma, const double* rho, const int32_t* option_type,
                    const int32_t* paths, const int32_t* steps, const uint64_t* seed, int32_t n,
                    qkb::BatchInput* in) {
    const NamedPtr base[] = {{model, "model"}, {spot, "spot"}, {strike, "strike"}, {t, "t"},
                             {r, "r"}, {q, "q"}, {option_type, "option_type"}, {paths, "paths"},
                             {seed, "seed"}};
    if (int32_t rc = check_nulls(base)) return rc;
    if (n <= 0) return fail_size(n);
    bool need_vol = false, need_heston = false, need_steps = false, need_shift = false;
    for (int32_t i = 0; i < n; ++i) {
        const int32_t m = model[i];
        // the LR delta reads its weight clip from `vol`
        if ((m >= qkb::kStandard && m <= qkb::kTerminalPlain) || m == qkb::kHestonLrDelta ||
            (m >= qkb::kControlVariates && m <= qkb::kQmcHalton))
            need_vol = true;
        // importance sampling reads its shift from `v0`
        if (m == qkb::kImportanceSampling) need_shift = true;
        if (m == qkb::kEuler || m == qkb::kMilstein || m == qkb::kLocalVol || m == qkb::kHeston ||
            m == qkb::kHestonLrDelta)
            need_steps = true;
        if (m == qkb::kHeston || m == qkb::kHestonLrDelta) need_heston = true;
    }
    if (need_vol && !vol) return fail_null("vol");
    if (need_heston) {
        const NamedPtr hp[] = {{v0, "v0"}, {kappa, "kappa"}, {theta, "theta"}, {sigma, "sigma"},
                               {rho, "rho"}};
        if (int32_t rc = check_nulls(hp)) return rc;
    }
    if (need_steps && !steps) return fail_null("steps");
    if (need_shift && !v0) return fail_null("v0");
    in->model = model;
    in->spot = spot;
    in->strike = strike;
    in->t = t;
    in->vol = vol;
    in->r = r;
    in->q = q;
    in->v0 = v0;
    in->kappa = kappa;
    in->theta = theta;
    in->sigma = sigma;
    in->rho = rho;
    in->option_type = option_type;
    in->paths = paths;
    in->steps = steps;
    in->seed = seed;
    in->n = n;
    return QK_OK;
}

}  // namespace


extern "C" {

void qk_abi_version(int32_t* major, int32_t* minor) {
    if (major) *major = QK_ABI_MAJOR;
    if (minor) *minor = QK_ABI_MINOR;
}

int32_t qk_plugin_get_api(int32_t host_abi_major, int32_t host_abi_minor,
                          const QKPluginAPI** out_api) {
    if (!out_api) return QK_ERR_NULL_PTR;
    if (host_abi_major != QK_ABI_MAJOR || host_abi_minor > QK_ABI_MINOR) {
        *out_api = nullptr;
        return QK_ERR_ABI_MISMATCH;
    }
    *out_api = &k_plugin_api;
    return QK_OK;
}

const char* qk_get_last_error(void) { return qkb::last_error(); }

int32_t qk_set_device(int32_t device) {
    cudaError_t e = cudaSetDevice(device);
    return e == cudaSuccess ? QK_OK : fail_cuda(e, "qk_set_device");
}

int32_t qk_get_device(int32_t* device) {
    if (!device) return fail_null("device");
    int d = -1;
    cudaError_t e = cudaGetDevice(&d);
    if (e != cudaSuccess) return fail_cuda(e, "qk_get_device");
    *device = d;
    return QK_OK;
}

void qk_clear_last_error(void) { qkb::clear_error(); }

// ---- terminal ---------------------------------------------------------------
int32_t qk_mcm_standard_monte_carlo_price_batch(const double* spot, const double* strike,
                                                const double* t, const double* vol,
                                                const double* r, const double* q,
                                                const int32_t* option_type, const int32_t* paths,
                                                const uint64_t* seed, int32_t n,
                                                double* out_prices) {
    return terminal_batch(qkb::kStandard, spot, strike, t, vol, r, q, option_type, paths, seed, n,
                          out_prices, nullptr, false, "qk_mcm_standard_monte_carlo_price_batch");
}

int32_t qk_mcm_standard_monte_carlo_price_se_batch(const double* spot, const double* strike,
                                                   const double* t, const double* vol,
                                                   const double* r, const double* q,
                                                   const int32_t* option_type,
                                                   const int32_t* paths, const uint64_t* seed,
                                                   int32_t n, double* out_prices,
                                                   double* out_stderr) {
    return terminal_batch(qkb::kStandard, spot, strike, t, vol, r, q, option_type, paths, seed, n,
                          out_prices, out_stderr, true,
                          "qk_mcm_standard_monte_carlo_price_se_batch");
}

double qk_mcm_standard_monte_carlo_price(double spot, double strike, double t, double vol,
                                         double r, double q, int32_t option_type, int32_t paths,
                                         uint64_t seed) {
    double out = nan_value();
    if (qk_mcm_standard_monte_carlo_price_batch(&spot, &strike, &t, &vol, &r, &q, &option_type,
                                                &paths, &seed, 1, &out) != QK_OK)
        return nan_value();
    return out;
}

int32_t qk_mcm_antithetic_variates_price_batch(const double* spot, const double* strike,
                                               const double* t, const double* vol,
                                               const double* r, const double* q,
                                               const int32_t* option_type, const int32_t* paths,
                                               const uint64_t* seed, int32_t n,
                                               double* out_prices) {
    return terminal_batch(qkb::kAntithetic, spot, strike, t, vol, r, q, option_type, paths, seed,
                          n, out_prices, nullptr, false, "qk_mcm_antithetic_variates_price_batch");
}

int32_t qk_mcm_antithetic_variates_price_se_batch(const double* spot, const double* strike,
                                                  const double* t, const double* vol,
                                                  const double* r, const double* q,
                                                  const int32_t* option_type,
                                                  const int32_t* paths, const uint64_t* seed,
                                                  int32_t n, double* out_prices,
                                                  double* out_stderr) {
    return terminal_batch(qkb::kAntithetic, spot, strike, t, vol, r, q, option_type, paths, seed,
                          n, out_prices, out_stderr, true,
                          "qk_mcm_antithetic_variates_price_se_batch");
}

double qk_mcm_antithetic_variates_price(double spot, double strike, double t, double vol,
                                        double r, double q, int32_t option_type, int32_t paths,
                                        uint64_t seed) {
    double out = nan_value();
    if (qk_mcm_antithetic_variates_price_batch(&spot, &strike, &t, &vol, &r, &q, &option_type,
                                               &paths, &seed, 1, &out) != QK_OK)
        return nan_value();
    return out;
}

// ---- one-factor stepwise -----------------------------------------------------
#define QK_STEPWISE_ENTRY(NAME, MODEL)                                                           \
    int32_t qk_mcm_##NAME##_price_batch(const double* spot, const double* strike,               \
                                        const double* t, const double* vol, const double* r,    \
                                        const double* q, const int32_t* option_type,            \
                                        const int32_t* paths, const int32_t* steps,             \
                                        const uint64_t* seed, int32_t n, double* out_prices) {  \
        return stepwise_batch(MODEL, spot, strike, t, vol, r, q, option_type, paths, steps, seed, \
                              n, out_prices, nullptr, false, "qk_mcm_" #NAME "_price_batch");   \
    }                                                                                           \
    int32_t qk_mcm_##NAME##_price_se_batch(const double* spot, const double* strike,            \
                                           const double* t, const double* vol,                  \
                                           const double* r, const double* q,                    \
                                           const int32_t* option_type, const int32_t* paths,    \
                                           const int32_t* steps, const uint64_t* seed,          \
                                           int32_t n, double* out_prices, double* out_stderr) { \
        return stepwise_batch(MODEL, spot, strike, t, vol, r, q, option_type, paths, steps, seed, \
                              n, out_prices, out_stderr, true,                                  \
                              "qk_mcm_" #NAME "_price_se_batch");                               \
    }                                                                                           \
    double qk_mcm_##NAME##_price(double spot, double strike, double t, double vol, double r,    \
                                 double q, int32_t option_type, int32_t paths, int32_t steps,   \
                                 uint64_t seed) {                                               \
        double out = nan_value();                                                               \
        if (qk_mcm_##NAME##_price_batch(&spot, &strike, &t, &vol, &r, &q, &option_type, &paths,  \
                                        &steps, &seed, 1, &out) != QK_OK)                       \
            return nan_value();                                                                 \
        return out;                                                                             \
    }

QK_STEPWISE_ENTRY(euler_maruyama, qkb::kEuler)
QK_STEPWISE_ENTRY(milstein, qkb::kMilstein)
QK_STEPWISE_ENTRY(local_vol_monte_carlo, qkb::kLocalVol)
#undef QK_STEPWISE_ENTRY

// ---- Heston --------------------------------------------------------------------
int32_t qk_mcm_heston_monte_carlo_price_batch(const double* spot, const double* strike,
                                              const double* t, const double* r, const double* q,
                                              const double* v0, const double* kappa,
                                              const double* theta, const double* sigma,
                                              const double* rho, const int32_t* option_type,
                                              const int32_t* paths, const int32_t* steps,
                                              const uint64_t* seed, int32_t n,
                                              double* out_prices) {
    return heston_batch(spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type, paths,
                        steps, seed, n, out_prices, nullptr, false,
                        "qk_mcm_heston_monte_carlo_price_batch");
}

int32_t qk_mcm_heston_monte_carlo_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr) {
    return heston_batch(spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type, paths,
                        steps, seed, n, out_prices, out_stderr, true,
                        "qk_mcm_heston_monte_carlo_price_se_batch");
}

double qk_mcm_heston_monte_carlo_price(double spot, double strike, double t, double r, double q,
                                       double v0, double kappa, double theta, double sigma,
                                       double rho, int32_t option_type, int32_t paths,
                                       int32_t steps, uint64_t seed) {
    double out = nan_value();
    if (qk_mcm_heston_monte_carlo_price_batch(&spot, &strike, &t, &r, &q, &v0, &kappa, &theta,
                                              &sigma, &rho, &option_type, &paths, &steps, &seed,
                                              1, &out) != QK_OK)
        return nan_value();
    return out;
}

int32_t qk_mcm_heston_monte_carlo_price_batch_noalloc(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr) {
    const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {r, "r"},
                             {q, "q"}, {v0, "v0"}, {kappa, "kappa"}, {theta, "theta"},
                             {sigma, "sigma"}, {rho, "rho"}, {option_type, "option_type"},
                             {paths, "paths"}, {steps, "steps"}, {seed, "seed"},
                             {out_prices, "out_prices"}};
    if (int32_t rc = check_nulls(ptrs)) return rc;
    if (n <= 0) return fail_size(n);
    const qkb::BatchInput in = heston_input(spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                            option_type, paths, steps, seed, n);
    cudaError_t e = cudaSuccess;
    int64_t tiles = 0;
    switch (qkb::noalloc_heston_batch(in, out_prices, out_stderr, &e, &tiles)) {
        case qkb::NoAllocStatus::kOk:
            return QK_OK;
        case qkb::NoAllocStatus::kTooManyOptions:
            set_error_fmt("bad batch size: %d options exceed the no-allocation limit of %d", n,
                          qkb::kNoAllocMaxOptions);
            return QK_ERR_BAD_SIZE;
        case qkb::NoAllocStatus::kTooManyTiles:
            set_error_fmt("bad batch size: %lld tiles exceed the no-allocation limit of %lld "
                          "(an option of P paths takes min(4096, ceil(ceil(P/2)/512)) tiles)",
                          (long long)tiles, (long long)qkb::kNoAllocMaxTiles);
            return QK_ERR_BAD_SIZE;
        default:
            return fail_cuda(e, "qk_mcm_heston_monte_carlo_price_batch_noalloc");
    }
}

// ---- Heston likelihood-ratio delta ------------------------------------------------
static int32_t lr_delta_batch(const double* spot, const double* strike, const double* t, const double* r,
                       const double* q, const double* v0, const double* kappa, const double* theta,
                       const double* sigma, const double* rho, const int32_t* option_type,
                       const int32_t* paths, const int32_t* steps, const uint64_t* seed,
                       const double* weight_clip, int32_t n, double* out_prices, double* out_se,
                       bool want_se, const char* where) {
    const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {r, "r"}, {q, "q"},
                             {v0, "v0"}, {kappa, "kappa"}, {theta, "theta"}, {sigma, "sigma"},
                             {rho, "rho"}, {option_type, "option_type"}, {paths, "paths"},
                             {steps, "steps"}, {seed, "seed"}, {weight_clip, "weight_clip"},
                             {out_prices, "out_prices"}};
    if (int32_t rc = check_nulls(ptrs)) return rc;
    if (want_se && !out_se) return fail_null("out_stderr");
    if (n <= 0) return fail_size(n);
    qkb::BatchInput in = heston_input(spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                      option_type, paths, steps, seed, n);
    in.uniform_model = qkb::kHestonLrDelta;
    in.weight_clip = weight_clip;
    return run_batch(in, 0, out_prices, out_se, where);
}

int32_t qk_mcm_heston_lr_delta_batch(const double* spot, const double* strike, const double* t,
                                     const double* r, const double* q, const double* v0,
                                     const double* kappa, const double* theta, const double* sigma,
                                     const double* rho, const int32_t* option_type,
                                     const int32_t* paths, const int32_t* steps,
                                     const uint64_t* seed, const double* weight_clip, int32_t n,
                                     double* out_prices) {
    return lr_delta_batch(spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type, paths,
                          steps, seed, weight_clip, n, out_prices, nullptr, false,
                          "qk_mcm_heston_lr_delta_batch");
}

int32_t qk_mcm_heston_lr_delta_se_batch(const double* spot, const double* strike, const double* t,
                                        const double* r, const double* q, const double* v0,
                                        const double* kappa, const double* theta,
                                        const double* sigma, const double* rho,
                                        const int32_t* option_type, const int32_t* paths,
                                        const int32_t* steps, const uint64_t* seed,
                                        const double* weight_clip, int32_t n, double* out_prices,
                                        double* out_stderr) {
    return lr_delta_batch(spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type, paths,
                          steps, seed, weight_clip, n, out_prices, out_stderr, true,
                          "qk_mcm_heston_lr_delta_se_batch");
}

double qk_mcm_heston_lr_delta(double spot, double strike, double t, double r, double q, double v0,
                              double kappa, double theta, double sigma, double rho,
                              int32_t option_type, int32_t paths, int32_t steps, uint64_t seed,
                              double weight_clip) {
    double out = nan_value();
    if (qk_mcm_heston_lr_delta_batch(&spot, &strike, &t, &r, &q, &v0, &kappa, &theta, &sigma, &rho,
                                     &option_type, &paths, &steps, &seed, &weight_clip, 1,
                                     &out) != QK_OK)
        return nan_value();
    return out;
}

// ---- terminal variance reduction ---------------------------------------------------
#define QK_VR_SEEDED(NAME, MODEL)                                                              \
    int32_t qk_mcm_##NAME##_price_batch(const double* spot, const double* strike, const double* t, \
                                        const double* vol, const double* r, const double* q,     \
                                        const int32_t* option_type, const int32_t* paths,        \
                                        const uint64_t* seed, int32_t n, double* out_prices) {   \
        return vr_batch(MODEL, spot, strike, t, vol, r, q, option_type, paths, nullptr, seed, n, \
                        out_prices, nullptr, false, "qk_mcm_" #NAME "_price_batch");            \
    }                                                                                          \
    int32_t qk_mcm_##NAME##_price_se_batch(                                                    \
        const double* spot, const double* strike, const double* t, const double* vol,          \
        const double* r, const double* q, const int32_t* option_type, const int32_t* paths,    \
        const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr) {             \
        return vr_batch(MODEL, spot, strike, t, vol, r, q, option_type, paths, nullptr, seed, n, \
                        out_prices, out_stderr, true, "qk_mcm_" #NAME "_price_se_batch");       \
    }                                                                                          \
    double qk_mcm_##NAME##_price(double spot, double strike, double t, double vol, double r,   \
                                 double q, int32_t option_type, int32_t paths, uint64_t seed) { \
        double out = nan_value();                                                              \
        if (qk_mcm_##NAME##_price_batch(&spot, &strike, &t, &vol, &r, &q, &option_type, &paths, \
                                        &seed, 1, &out) != QK_OK)                              \
            return nan_value();                                                                \
        return out;                                                                            \
    }

#define QK_VR_QMC(NAME, MODEL)                                                                 \
    int32_t qk_mcm_##NAME##_price_batch(const double* spot, const double* strike, const double* t, \
                                        const double* vol, const double* r, const double* q,     \
                                        const int32_t* option_type, const int32_t* paths,        \
                                        int32_t n, double* out_prices) {                         \
        return vr_batch(MODEL, spot, strike, t, vol, r, q, option_type, paths, nullptr, nullptr, \
                        n, out_prices, nullptr, false, "qk_mcm_" #NAME "_price_batch");         \
    }                                                                                          \
    int32_t qk_mcm_##NAME##_price_se_batch(                                                    \
        const double* spot, const double* strike, const double* t, const double* vol,          \
        const double* r, const double* q, const int32_t* option_type, const int32_t* paths,    \
        int32_t n, double* out_prices, double* out_stderr) {                                   \
        return vr_batch(MODEL, spot, strike, t, vol, r, q, option_type, paths, nullptr, nullptr, \
                        n, out_prices, out_stderr, true, "qk_mcm_" #NAME "_price_se_batch");    \
    }                                                                                          \
    double qk_mcm_##NAME##_price(double spot, double strike, double t, double vol, double r,   \
                                 double q, int32_t option_type, int32_t paths) {               \
        double out = nan_value();                                                              \
        if (qk_mcm_##NAME##_price_batch(&spot, &strike, &t, &vol, &r, &q, &option_type, &paths, \
                                        1, &out) != QK_OK)                                     \
            return nan_value();                                                                \
        return out;                                                                            \
    }

QK_VR_SEEDED(control_variates, qkb::kControlVariates)
QK_VR_SEEDED(stratified_sampling, qkb::kStratified)
QK_VR_QMC(quasi_monte_carlo_sobol, qkb::kQmcSobol)
QK_VR_QMC(quasi_monte_carlo_halton, qkb::kQmcHalton)
#undef QK_VR_SEEDED
#undef QK_VR_QMC

int32_t qk_mcm_importance_sampling_price_batch(const double* spot, const double* strike,
                                               const double* t, const double* vol, const double* r,
                                               const double* q, const int32_t* option_type,
                                               const int32_t* paths, const double* shift,
                                               const uint64_t* seed, int32_t n,
                                               double* out_prices) {
    return vr_batch(qkb::kImportanceSampling, spot, strike, t, vol, r, q, option_type, paths,
                    shift, seed, n, out_prices, nullptr, false,
                    "qk_mcm_importance_sampling_price_batch");
}

int32_t qk_mcm_importance_sampling_price_se_batch(const double* spot, const double* strike,
                                                  const double* t, const double* vol,
                                                  const double* r, const double* q,
                                                  const int32_t* option_type, const int32_t* paths,
                                                  const double* shift, const uint64_t* seed,
                                                  int32_t n, double* out_prices,
                                                  double* out_stderr) {
    return vr_batch(qkb::kImportanceSampling, spot, strike, t, vol, r, q, option_type, paths,
                    shift, seed, n, out_prices, out_stderr, true,
                    "qk_mcm_importance_sampling_price_se_batch");
}

double qk_mcm_importance_sampling_price(double spot, double strike, double t, double vol, double r,
                                        double q, int32_t option_type, int32_t paths, double shift,
                                        uint64_t seed) {
    double out = nan_value();
    if (qk_mcm_importance_sampling_price_batch(&spot, &strike, &t, &vol, &r, &q, &option_type,
                                               &paths, &shift, &seed, 1, &out) != QK_OK)
        return nan_value();
    return out;
}

// ---- Heston characteristic-function pricer -----------------------------------------
int32_t qk_cf_heston_price_cf_batch(const double* spot, const double* strike, const double* t,
                                    const double* r, const double* q, const double* v0,
                                    const double* kappa, const double* theta, const double* sigma,
                                    const double* rho, const int32_t* option_type,
                                    const int32_t* integration_steps,
                                    const double* integration_limit, int32_t n,
                                    double* out_prices) {
    const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {r, "r"}, {q, "q"},
                             {v0, "v0"}, {kappa, "kappa"}, {theta, "theta"}, {sigma, "sigma"},
                             {rho, "rho"}, {option_type, "option_type"},
                             {integration_steps, "integration_steps"},
                             {integration_limit, "integration_limit"}, {out_prices, "out_prices"}};
    if (int32_t rc = check_nulls(ptrs)) return rc;
    if (n <= 0) return fail_size(n);
    std::vector<qkb::CfOption> recs(static_cast<size_t>(n));
    for (int32_t i = 0; i < n; ++i)
        recs[i] = qkb::pack_cf_option(spot[i], strike[i], t[i], r[i], q[i], v0[i], kappa[i],
                                      theta[i], sigma[i], rho[i], option_type[i],
                                      integration_steps[i], integration_limit[i]);
    cudaError_t e = qkb::heston_cf_price_host(recs.data(), n, out_prices);
    return e == cudaSuccess ? QK_OK : fail_cuda(e, "qk_cf_heston_price_cf_batch");
}

// ---- Heston COS expansion ----------------------------------------------------------
int32_t qk_ftm_cos_fang_oosterlee_heston_price_batch(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* n_terms,
    const double* truncation_width, int32_t n, double* out_prices) {
    const NamedPtr ptrs[] = {{spot, "spot"}, {strike, "strike"}, {t, "t"}, {r, "r"}, {q, "q"},
                             {v0, "v0"}, {kappa, "kappa"}, {theta, "theta"}, {sigma, "sigma"},
                             {rho, "rho"}, {option_type, "option_type"}, {n_terms, "n_terms"},
                             {truncation_width, "truncation_width"}, {out_prices, "out_prices"}};
    if (int32_t rc = check_nulls(ptrs)) return rc;
    if (n <= 0) return fail_size(n);
    std::vector<qkb::CfOption> recs(static_cast<size_t>(n));
    for (int32_t i = 0; i < n; ++i)
        recs[i] = qkb::pack_cos_option(spot[i], strike[i], t[i], r[i], q[i], v0[i], kappa[i],
                                       theta[i], sigma[i], rho[i], option_type[i], n_terms[i],
                                       truncation_width[i]);
    cudaError_t e = qkb::heston_cf_price_host(recs.data(), n, out_prices);
    return e == cudaSuccess ? QK_OK : fail_cuda(e, "qk_ftm_cos_fang_oosterlee_heston_price_batch");
}

double qk_ftm_cos_fang_oosterlee_heston_price(double spot, double strike, double t, double r,
                                              double q, double v0, double kappa, double theta,
                                              double sigma, double rho, int32_t option_type,
                                              int32_t n_terms, double truncation_width) {
    double out = nan_value();
    if (qk_ftm_cos_fang_oosterlee_heston_price_batch(&spot, &strike, &t, &r, &q, &v0, &kappa,
                                                     &theta, &sigma, &rho, &option_type, &n_terms,
                                                     &truncation_width, 1, &out) != QK_OK)
        return nan_value();
    return out;
}

double qk_cf_heston_price_cf(double spot, double strike, double t, double r, double q, double v0,
                             double kappa, double theta, double sigma, double rho,
                             int32_t option_type, int32_t integration_steps,
                             double integration_limit) {
    double out = nan_value();
    if (qk_cf_heston_price_cf_batch(&spot, &strike, &t, &r, &q, &v0, &kappa, &theta, &sigma, &rho,
                                    &option_type, &integration_steps, &integration_limit, 1,
                                    &out) != QK_OK)
        return nan_value();
    return out;
}

// ---- mixed batch and plans -------------------------------------------------------
int32_t qk_mcm_mixed_price_batch(const int32_t* model, const double* spot, const double* strike,
                                 const double* t, const double* vol, const double* r,
                                 const double* q, const double* v0, const double* kappa,
                                 const double* theta, const double* sigma, const double* rho,
                                 const int32_t* option_type, const int32_t* paths,
                                 const int32_t* steps, const uint64_t* seed, int32_t n,
                                 double* out_prices, double* out_stderr) {
    qkb::BatchInput in;
    int32_t rc = mixed_input(model, spot, strike, t, vol, r, q, v0, kappa, theta, sigma, rho,
                             option_type, paths, steps, seed, n, &in);
    if (rc != QK_OK) return rc;
    if (!out_prices) return fail_null("out_prices");
    return run_batch(in, qkb::kFlagPersistent, out_prices, out_stderr, "qk_mcm_mixed_price_batch");
}

int32_t qk_mcm_mixed_price_batch_sharded(qk_dist* dist, const int32_t* model, const double* spot,
                                         const double* strike, const double* t, const double* vol,
                                         const double* r, const double* q, const double* v0,
                                         const double* kappa, const double* theta,
                                         const double* sigma, const double* rho,
                                         const int32_t* option_type, const int32_t* paths,
                                         const int32_t* steps, const uint64_t* seed, int32_t n,
                                         double* out_prices, double* out_stderr) {
    static const char* where = "qk_mcm_mixed_price_batch_sharded";
    if (!dist) return fail_null("dist");
    qkb::BatchInput in;
    int32_t rc = mixed_input(model, spot, strike, t, vol, r, q, v0, kappa, theta, sigma, rho,
                             option_type, paths, steps, seed, n, &in);
    if (rc != QK_OK) return rc;
    if (!out_prices) return fail_null("out_prices");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_cuda(e, where);
    // the tile geometry of the single-GPU mixed call, so the results match it
    qkb::Plan* plan = qkb::thread_scratch_plan(dev);
    std::string err;
    if ((e = plan->build(in, qkb::kFlagPersistent, &err)) != cudaSuccess) return fail_cuda(e, where);
    if ((rc = qkb::dist_execute(*plan, dist, nullptr, where)) != QK_OK) return rc;
    if ((e = plan->results(out_prices, out_stderr)) != cudaSuccess) return fail_cuda(e, where);
    return QK_OK;
}

int32_t qk_mcm_plan_shard_bounds(qk_mc_plan* plan, int32_t world, int64_t* bounds) {
    if (!plan) return fail_null("plan");
    if (!bounds) return fail_null("bounds");
    if (world <= 0) return fail_size(world);
    const std::vector<int64_t>& b = plan->plan.shard_bounds(world);
    std::memcpy(bounds, b.data(), sizeof(int64_t) * ((size_t)world + 1));
    return QK_OK;
}

int32_t qk_mcm_plan_execute_tiles(qk_mc_plan* plan, int64_t tile_begin, int64_t tile_end,
                                  void* stream) {
    static const char* where = "qk_mcm_plan_execute_tiles";
    if (!plan) return fail_null("plan");
    qkb::Plan& p = plan->plan;
    if (tile_begin < 0 || tile_end < tile_begin || tile_end > p.n_tiles()) {
        set_error_fmt("invalid input: tiles [%lld, %lld) outside [0, %lld) in %s",
                      (long long)tile_begin, (long long)tile_end, (long long)p.n_tiles(), where);
        return QK_ERR_INVALID_INPUT;
    }
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != p.device()) e = cudaSetDevice(p.device());
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : p.stream();
    if (e == cudaSuccess) e = p.order_after_upload(st);
    if (e == cudaSuccess) e = p.launch_tiles(st, tile_begin, tile_end, false);
    if (e == cudaSuccess) p.note_stream(st);
    if (prev >= 0 && prev != p.device()) cudaSetDevice(prev);
    return e == cudaSuccess ? QK_OK : fail_cuda(e, where);
}

int32_t qk_mcm_plan_device_partials(qk_mc_plan* plan, void** d_partials, int64_t* n_tiles,
                                    int32_t* bytes_per_tile) {
    if (!plan) return fail_null("plan");
    if (d_partials) *d_partials = plan->plan.d_partials();
    if (n_tiles) *n_tiles = plan->plan.n_tiles();
    if (bytes_per_tile) *bytes_per_tile = (int32_t)sizeof(qkb::TilePartial);
    return QK_OK;
}

int32_t qk_mcm_plan_finalize(qk_mc_plan* plan, void* stream) {
    if (!plan) return fail_null("plan");
    qkb::Plan& p = plan->plan;
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != p.device()) e = cudaSetDevice(p.device());
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : p.stream();
    if (e == cudaSuccess) e = p.order_after_upload(st);
    if (e == cudaSuccess) e = p.launch_finalize_all(st);
    if (e == cudaSuccess) p.note_stream(st);
    if (prev >= 0 && prev != p.device()) cudaSetDevice(prev);
    return e == cudaSuccess ? QK_OK : fail_cuda(e, "qk_mcm_plan_finalize");
}

int32_t qk_mcm_plan_execute_sharded(qk_mc_plan* plan, qk_dist* dist, void* stream) {
    if (!plan) return fail_null("plan");
    return qkb::dist_execute(plan->plan, dist, static_cast<cudaStream_t>(stream),
                             "qk_mcm_plan_execute_sharded");
}

int32_t qk_mcm_plan_create(const int32_t* model, const double* spot, const double* strike,
                           const double* t, const double* vol, const double* r, const double* q,
                           const double* v0, const double* kappa, const double* theta,
                           const double* sigma, const double* rho, const int32_t* option_type,
                           const int32_t* paths, const int32_t* steps, const uint64_t* seed,
                           int32_t n, int32_t flags, qk_mc_plan** out_plan) {
    if (!out_plan) return fail_null("out_plan");
    *out_plan = nullptr;
    qkb::BatchInput in;
    int32_t rc = mixed_input(model, spot, strike, t, vol, r, q, v0, kappa, theta, sigma, rho,
                             option_type, paths, steps, seed, n, &in);
    if (rc != QK_OK) return rc;
    qk_mc_plan* p = new qk_mc_plan();
    std::string err;
    cudaError_t e = p->plan.build(in, flags, &err);
    if (e != cudaSuccess) {
        delete p;
        return fail_cuda(e, "qk_mcm_plan_create");
    }
    *out_plan = p;
    return QK_OK;
}

int32_t qk_mcm_plan_execute(qk_mc_plan* plan, void* stream) {
    if (!plan) return fail_null("plan");
    cudaError_t e = plan->plan.execute(static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? QK_OK : fail_cuda(e, "qk_mcm_plan_execute");
}

int32_t qk_mcm_plan_results(qk_mc_plan* plan, double* out_prices, double* out_stderr) {
    if (!plan) return fail_null("plan");
    if (!out_prices) return fail_null("out_prices");
    cudaError_t e = plan->plan.results(out_prices, out_stderr);
    return e == cudaSuccess ? QK_OK : fail_cuda(e, "qk_mcm_plan_results");
}

int32_t qk_mcm_plan_device_results(qk_mc_plan* plan, double** d_prices, double** d_stderr) {
    if (!plan) return fail_null("plan");
    if (d_prices) *d_prices = plan->plan.d_price();
    if (d_stderr) *d_stderr = plan->plan.d_se();
    return QK_OK;
}

int32_t qk_mcm_plan_stats(qk_mc_plan* plan, double* simulate_ms, int32_t* launches,
                          int64_t* path_steps) {
    if (!plan) return fail_null("plan");
    cudaError_t e = plan->plan.sync_stats();
    if (e != cudaSuccess) return fail_cuda(e, "qk_mcm_plan_stats");
    if (simulate_ms) *simulate_ms = plan->plan.last_simulate_ms();
    if (launches) *launches = plan->plan.launches();
    if (path_steps) *path_steps = plan->plan.path_steps();
    return QK_OK;
}

int32_t qk_mcm_plan_config(qk_mc_plan* plan, int32_t* block, int32_t* units_per_thread,
                           int32_t* ctas) {
    if (!plan) return fail_null("plan");
    if (block) *block = plan->plan.block();
    if (units_per_thread) *units_per_thread = plan->plan.upt();
    if (ctas) *ctas = plan->plan.ctas();
    return QK_OK;
}

int32_t qk_mcm_plan_step_unroll(qk_mc_plan* plan, int32_t* step_unroll) {
    if (!plan) return fail_null("plan");
    if (!step_unroll) return fail_null("step_unroll");
    *step_unroll = plan->plan.step_unroll();
    return QK_OK;
}

int32_t qk_mcm_plan_destroy(qk_mc_plan* plan) {
    if (!plan) return QK_OK;
    delete plan;
    return QK_OK;
}

}  // extern "C"
