/*
 * qk_api.h -- C ABI of the B200 batch Monte Carlo pricing library
 * (libqk_b200.so).
 *
 * Part 1 is a drop-in for the Monte Carlo subset of yluoc/Quant-Kernel's
 * cpp/include/quantkernel/qk_api.h: the same names, argument order, types,
 * return codes and NaN-per-bad-element behaviour.  Each declaration cites the
 * reference declaration it replaces.  All pointers are host pointers; calls
 * are synchronous and thread-safe (one CUDA stream and one error buffer per
 * calling thread).  There is no CPU fallback: when CUDA is unusable the batch
 * calls return QK_ERR_RUNTIME_INIT and the scalar calls return NaN, both with
 * a message in qk_get_last_error().
 *
 * Part 2 (ABI 2.13) adds calls with no reference counterpart: price + standard
 * error batches, a mixed-model batch, and device-resident "plans".
 */
#ifndef QK_API_H
#define QK_API_H

#include "qk_abi.h"

#ifdef _WIN32
#define QK_EXPORT __declspec(dllexport)
#else
#define QK_EXPORT __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================= *
 * Part 1 -- reference-compatible entry points
 * ======================================================================= */

/* qk_api.h:16 */
QK_EXPORT void qk_abi_version(int32_t* major, int32_t* minor);
/* qk_api.h:17-19 */
QK_EXPORT int32_t qk_plugin_get_api(int32_t host_abi_major, int32_t host_abi_minor,
                                    const QKPluginAPI** out_api);
/* qk_api.h:20 */
QK_EXPORT const char* qk_get_last_error(void);
/* qk_api.h:21 */
QK_EXPORT void qk_clear_last_error(void);

/* qk_api.h:259-261 (estimate_terminal_antithetic, zero-vol forward branch) */
QK_EXPORT double qk_mcm_standard_monte_carlo_price(double spot, double strike, double t, double vol,
                                                   double r, double q, int32_t option_type,
                                                   int32_t paths, uint64_t seed);
/* qk_api.h:262-268 */
QK_EXPORT int32_t qk_mcm_standard_monte_carlo_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
    int32_t n, double* out_prices);

/* qk_api.h:269-271 (estimate_stepwise + make_bsm_euler_step) */
QK_EXPORT double qk_mcm_euler_maruyama_price(double spot, double strike, double t, double vol,
                                             double r, double q, int32_t option_type,
                                             int32_t paths, int32_t steps, uint64_t seed);
/* qk_api.h:300-305 */
QK_EXPORT int32_t qk_mcm_euler_maruyama_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices);

/* qk_api.h:272-274 (estimate_stepwise + make_bsm_milstein_step) */
QK_EXPORT double qk_mcm_milstein_price(double spot, double strike, double t, double vol, double r,
                                       double q, int32_t option_type, int32_t paths,
                                       int32_t steps, uint64_t seed);
/* qk_api.h:306-311 */
QK_EXPORT int32_t qk_mcm_milstein_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices);

/* qk_api.h:294-296 (estimate_terminal_antithetic) */
QK_EXPORT double qk_mcm_antithetic_variates_price(double spot, double strike, double t, double vol,
                                                  double r, double q, int32_t option_type,
                                                  int32_t paths, uint64_t seed);
/* qk_api.h:347-352 */
QK_EXPORT int32_t qk_mcm_antithetic_variates_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
    int32_t n, double* out_prices);

/* qk_api.h:359-364 (estimate_stepwise_2d + make_heston_euler_step) */
QK_EXPORT double qk_mcm_heston_monte_carlo_price(double spot, double strike, double t, double r,
                                                 double q, double v0, double kappa, double theta,
                                                 double sigma, double rho, int32_t option_type,
                                                 int32_t paths, int32_t steps, uint64_t seed);
/* qk_api.h:365-374 */
QK_EXPORT int32_t qk_mcm_heston_monte_carlo_price_batch(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices);

/* qk_api.h:375-380 (heston_lr_delta.cpp:37-132: likelihood-ratio delta,
 * antithetic pairs, score clipped to +-weight_clip) */
QK_EXPORT double qk_mcm_heston_lr_delta(double spot, double strike, double t, double r, double q,
                                        double v0, double kappa, double theta, double sigma,
                                        double rho, int32_t option_type, int32_t paths,
                                        int32_t steps, uint64_t seed, double weight_clip);
/* qk_api.h:381-392 */
QK_EXPORT int32_t qk_mcm_heston_lr_delta_batch(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, const double* weight_clip, int32_t n, double* out_prices);

/* qk_api.h:393-396 (local_vol_price_impl, constant sigma) */
QK_EXPORT double qk_mcm_local_vol_monte_carlo_price(double spot, double strike, double t,
                                                    double vol, double r, double q,
                                                    int32_t option_type, int32_t paths,
                                                    int32_t steps, uint64_t seed);
/* qk_api.h:397-403 */
QK_EXPORT int32_t qk_mcm_local_vol_monte_carlo_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices);

/* Terminal GBM with the reference's variance-reduction estimators. */
/* qk_api.h:291-293 (control_variates.cpp:10-52: control x = disc * S_T with
 * known mean spot e^{-qt}, beta from the same sample; paths >= 3) */
QK_EXPORT double qk_mcm_control_variates_price(double spot, double strike, double t, double vol,
                                               double r, double q, int32_t option_type,
                                               int32_t paths, uint64_t seed);
/* qk_api.h:341-346 */
QK_EXPORT int32_t qk_mcm_control_variates_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
    int32_t n, double* out_prices);
/* qk_api.h:288-290 (importance_sampling.cpp:11-36: normal shifted by `shift`,
 * likelihood-ratio weight exp(-shift y + shift^2/2)) */
QK_EXPORT double qk_mcm_importance_sampling_price(double spot, double strike, double t, double vol,
                                                  double r, double q, int32_t option_type,
                                                  int32_t paths, double shift, uint64_t seed);
/* qk_api.h:335-340 */
QK_EXPORT int32_t qk_mcm_importance_sampling_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const double* shift,
    const uint64_t* seed, int32_t n, double* out_prices);
/* qk_api.h:297-299 (stratified_sampling.cpp:11-35: one draw per stratum
 * [i/n, (i+1)/n), Acklam inverse normal) */
QK_EXPORT double qk_mcm_stratified_sampling_price(double spot, double strike, double t, double vol,
                                                  double r, double q, int32_t option_type,
                                                  int32_t paths, uint64_t seed);
/* qk_api.h:353-358 */
QK_EXPORT int32_t qk_mcm_stratified_sampling_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
    int32_t n, double* out_prices);
/* qk_api.h:278-280 (quasi_monte_carlo.cpp:10-32: one-dimensional Sobol points
 * 1..paths, Acklam inverse normal; deterministic, no seed) */
QK_EXPORT double qk_mcm_quasi_monte_carlo_sobol_price(double spot, double strike, double t,
                                                      double vol, double r, double q,
                                                      int32_t option_type, int32_t paths);
/* qk_api.h:318-322 */
QK_EXPORT int32_t qk_mcm_quasi_monte_carlo_sobol_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, int32_t n,
    double* out_prices);
/* qk_api.h:281-283 (quasi_monte_carlo.cpp:34-56: Halton base 2) */
QK_EXPORT double qk_mcm_quasi_monte_carlo_halton_price(double spot, double strike, double t,
                                                       double vol, double r, double q,
                                                       int32_t option_type, int32_t paths);
/* qk_api.h:323-327 */
QK_EXPORT int32_t qk_mcm_quasi_monte_carlo_halton_price_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, int32_t n,
    double* out_prices);

/* qk_api.h:53-55 (heston.cpp:7-53: little-trap characteristic function,
 * P1/P2 by ceil(integration_steps/64) panels of 64-point Gauss-Legendre on
 * [1e-8, integration_limit]; FP64 on the GPU, one CTA per option) */
QK_EXPORT double qk_cf_heston_price_cf(double spot, double strike, double t, double r, double q,
                                       double v0, double kappa, double theta, double sigma,
                                       double rho, int32_t option_type, int32_t integration_steps,
                                       double integration_limit);
/* qk_api.h:71-76 */
QK_EXPORT int32_t qk_cf_heston_price_cf_batch(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* integration_steps,
    const double* integration_limit, int32_t n, double* out_prices);

/* qk_api.h:463-468 (cos_method.cpp:30-58: Fang-Oosterlee COS expansion with
 * the Heston log-price characteristic function, n_terms cosine terms on
 * [c1 -/+ truncation_width sqrt(max(v0, theta) t)]; FP64 on the GPU, one CTA
 * per option) */
QK_EXPORT double qk_ftm_cos_fang_oosterlee_heston_price(double spot, double strike, double t,
                                                        double r, double q, double v0,
                                                        double kappa, double theta, double sigma,
                                                        double rho, int32_t option_type,
                                                        int32_t n_terms, double truncation_width);
/* qk_api.h:498-505 */
QK_EXPORT int32_t qk_ftm_cos_fang_oosterlee_heston_price_batch(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* n_terms,
    const double* truncation_width, int32_t n, double* out_prices);

/* ======================================================================= *
 * Part 2 -- additions in ABI 2.13 (no counterpart in the reference)
 * ======================================================================= */

/* Device selection for the calling thread (the library links its own CUDA
 * runtime, so a host framework's current device is not seen here).  Every
 * later call from this thread runs on `device`.  Returns QK_ERR_RUNTIME_INIT
 * for a device that does not exist. */
QK_EXPORT int32_t qk_set_device(int32_t device);
QK_EXPORT int32_t qk_get_device(int32_t* device);

/* Model codes for the mixed-model batch and for plans. */
#define QK_MC_STANDARD       0 /* terminal GBM, antithetic pairs, zero-vol forward branch */
#define QK_MC_ANTITHETIC     1 /* terminal GBM, antithetic pairs */
#define QK_MC_EULER          2 /* BSM Euler-Maruyama */
#define QK_MC_MILSTEIN       3 /* BSM Milstein */
#define QK_MC_LOCAL_VOL      4 /* constant local-vol Euler */
#define QK_MC_TERMINAL_PLAIN 5 /* terminal GBM, independent paths */
#define QK_MC_HESTON         6 /* Heston full-truncation Euler */
#define QK_MC_HESTON_LR_DELTA 7 /* Heston likelihood-ratio delta; `vol` holds weight_clip */
#define QK_MC_CONTROL_VARIATES 8 /* terminal GBM, control variate S_T */
#define QK_MC_IMPORTANCE_SAMPLING 9 /* terminal GBM, shifted normal; `v0` holds the shift */
#define QK_MC_STRATIFIED     10 /* terminal GBM, one draw per stratum */
#define QK_MC_QMC_SOBOL      11 /* terminal GBM, Sobol points (seed ignored) */
#define QK_MC_QMC_HALTON     12 /* terminal GBM, Halton base-2 points (seed ignored) */

/* Plan flags. */
#define QK_PLAN_PERSISTENT    0x1 /* one persistent work-stealing launch over all tiles */
#define QK_PLAN_GRAPH         0x2 /* replay execute() from a captured CUDA graph */
#define QK_PLAN_NO_ANTITHETIC 0x4 /* stepwise models: independent paths, not pairs */
#define QK_PLAN_TIMING        0x8 /* record CUDA events around the simulate kernel */
#define QK_PLAN_AUTOTUNE      0x10 /* choose block size / units per thread / step
                                      * unrolling by timing; for batches of several model
                                      * families also the mode: one persistent kernel or
                                      * one grid per family (the latter not when
                                      * QK_PLAN_PERSISTENT is given) */
#define QK_PLAN_FAMILY_GRIDS  0x20 /* several model families: one grid per family group,
                                      * back to back, instead of the persistent kernel */
#define QK_PLAN_STEP_UNROLL2  0x40 /* stepwise single-family plans (Euler, Milstein and
                                      * local vol at 1, 2 or 4 units per thread, Heston at
                                      * 1 or 2): two Philox step blocks per loop iteration
                                      * (same results bit for bit; the autotuner also
                                      * tries it) */

/* Price + standard error batches.  Same inputs as the Part 1 batch calls;
 * out_stderr[i] is the standard error of out_prices[i] (NaN where no
 * simulation ran: invalid input, t <= 1e-12, the zero-vol branch). */
QK_EXPORT int32_t qk_mcm_standard_monte_carlo_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
    int32_t n, double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_antithetic_variates_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
    int32_t n, double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_euler_maruyama_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_milstein_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_local_vol_monte_carlo_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_heston_monte_carlo_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr);
/* Variance-reduction estimators.  Standard errors: control variates -- the
 * residual variance of payoff - beta * control over n - 2; stratified -- the
 * squared differences of neighbouring strata pairs (conservative); importance
 * sampling -- the weighted payoffs' sample variance; quasi-Monte Carlo -- the
 * i.i.d. formula applied to the points (an indicator, not a confidence bound:
 * the points are not random). */
QK_EXPORT int32_t qk_mcm_control_variates_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
    int32_t n, double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_importance_sampling_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const double* shift,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_stratified_sampling_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, const uint64_t* seed,
    int32_t n, double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_quasi_monte_carlo_sobol_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, int32_t n,
    double* out_prices, double* out_stderr);
QK_EXPORT int32_t qk_mcm_quasi_monte_carlo_halton_price_se_batch(
    const double* spot, const double* strike, const double* t, const double* vol, const double* r,
    const double* q, const int32_t* option_type, const int32_t* paths, int32_t n,
    double* out_prices, double* out_stderr);

/* Heston batch that allocates no memory.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc: services whose host framework owns
 * every device allocation (a caching allocator or a capped pool), processes
 * that must not grow their GPU footprint after start-up, and latency-bound
 * paths that cannot afford an allocation or the synchronisation of a free.
 * Same inputs and outputs as qk_mcm_heston_monte_carlo_price_se_batch (host
 * arrays; out_stderr may be NULL) and the same kernels and results; every
 * device buffer lives in one fixed 16.6 MiB array per GPU, held until the
 * process exits.  Limits: n <= 4096 options and at most 262,144 tiles in
 * total, where an option of P paths takes min(4096, ceil(ceil(P/2) / 512))
 * tiles (1024 options of 262,144 paths fill the limit; past 2^22 paths an
 * option's tiles grow instead of multiplying); larger batches return
 * QK_ERR_BAD_SIZE before any GPU work.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) and creates the
 * library's non-blocking stream for this entry point, with that device
 * current, so make it before any stream capture; later calls use only that
 * stream (never the legacy default stream).  Calls share the array, which
 * keeps the last call's contents (every call overwrites what it reads, so
 * nothing needs clearing); two calls running on the GPU at once would race on
 * it, so this entry point serialises its calls with a lock and returns only
 * after the results are copied back. */
QK_EXPORT int32_t qk_mcm_heston_monte_carlo_price_batch_noalloc(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr);

QK_EXPORT int32_t qk_mcm_heston_lr_delta_se_batch(
    const double* spot, const double* strike, const double* t, const double* r, const double* q,
    const double* v0, const double* kappa, const double* theta, const double* sigma,
    const double* rho, const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, const double* weight_clip, int32_t n, double* out_prices,
    double* out_stderr);

/* Mixed-model batch: option i is priced with model[i] (QK_MC_*).  Fields a
 * model does not use are ignored and may hold anything (vol for Heston;
 * v0..rho for the BSM models; steps for the terminal models; seed for the
 * quasi-Monte Carlo models).  QK_MC_IMPORTANCE_SAMPLING reads its shift from
 * v0.  Runs as one
 * persistent work-stealing launch.  out_stderr may be NULL. */
QK_EXPORT int32_t qk_mcm_mixed_price_batch(
    const int32_t* model, const double* spot, const double* strike, const double* t,
    const double* vol, const double* r, const double* q, const double* v0, const double* kappa,
    const double* theta, const double* sigma, const double* rho, const int32_t* option_type,
    const int32_t* paths, const int32_t* steps, const uint64_t* seed, int32_t n,
    double* out_prices, double* out_stderr);

/* Plans: validate and upload a batch once, then run it many times with the
 * inputs resident in GPU memory.  A plan belongs to the device that was
 * current when it was created.  execute() is asynchronous on `stream` (a
 * cudaStream_t; NULL = the plan's own stream); results() synchronises that
 * stream and copies prices (and standard errors, if out_stderr != NULL) to
 * host memory.  Plans are not thread-safe: one thread per plan at a time. */
typedef struct qk_mc_plan qk_mc_plan;

QK_EXPORT int32_t qk_mcm_plan_create(
    const int32_t* model, const double* spot, const double* strike, const double* t,
    const double* vol, const double* r, const double* q, const double* v0, const double* kappa,
    const double* theta, const double* sigma, const double* rho, const int32_t* option_type,
    const int32_t* paths, const int32_t* steps, const uint64_t* seed, int32_t n, int32_t flags,
    qk_mc_plan** out_plan);
QK_EXPORT int32_t qk_mcm_plan_execute(qk_mc_plan* plan, void* stream);
QK_EXPORT int32_t qk_mcm_plan_results(qk_mc_plan* plan, double* out_prices, double* out_stderr);
/* Device pointers to the plan's result arrays (n doubles each). */
QK_EXPORT int32_t qk_mcm_plan_device_results(qk_mc_plan* plan, double** d_prices,
                                             double** d_stderr);
/* Milliseconds of the last execute()'s simulate kernel (QK_PLAN_TIMING), and
 * the number of kernels one execute() launches. */
QK_EXPORT int32_t qk_mcm_plan_stats(qk_mc_plan* plan, double* simulate_ms, int32_t* launches,
                                    int64_t* path_steps);
/* The launch shape in use: block size; units per thread (> 0: one
 * single-family grid; 0: the persistent kernel; -1: one grid per family
 * group); CTAs of the persistent kernel. */
QK_EXPORT int32_t qk_mcm_plan_config(qk_mc_plan* plan, int32_t* block, int32_t* units_per_thread,
                                     int32_t* ctas);
/* Step blocks per loop iteration of the plan's simulate kernel (1 or 2; 1 for
 * terminal, variance-reduction and multi-family plans). */
QK_EXPORT int32_t qk_mcm_plan_step_unroll(qk_mc_plan* plan, int32_t* step_unroll);
QK_EXPORT int32_t qk_mcm_plan_destroy(qk_mc_plan* plan);

/* ----------------------------------------------------------------------- *
 * One batch across several GPUs (ABI 2.13, no counterpart in the reference,
 * which prices a batch with OpenMP threads on one host).  One rank per GPU
 * (a process or a thread each); every rank builds the same plan from the
 * same inputs.  A sharded execute simulates this rank's contiguous range of
 * the plan's tiles (balanced by path-steps), exchanges every rank's tile
 * sums over NCCL (one grouped broadcast step) and finalizes all options on
 * every rank, so results() gives the whole batch, bit for bit what a
 * single-GPU execute gives.  NCCL is loaded at run time (libnccl.so.2, or the
 * path in QK_B200_NCCL_PATH); without it these calls return
 * QK_ERR_RUNTIME_INIT ("nccl unavailable: ...").  The collective blocks
 * until every rank has joined it: a rank that never joins holds the others
 * until qk_dist_abort() is called on them (from another thread) or they are
 * stopped.
 * ----------------------------------------------------------------------- */
#define QK_DIST_ID_BYTES 128
typedef struct qk_dist qk_dist;

/* A new communicator id (QK_DIST_ID_BYTES bytes), made once on one rank and
 * handed to every rank (file, socket, the launcher's own store). */
QK_EXPORT int32_t qk_dist_unique_id(uint8_t* out_id);
/* Joins rank `rank` of `world` on the calling thread's current device
 * (qk_set_device first).  All ranks must call it with the same id. */
QK_EXPORT int32_t qk_dist_create(const uint8_t* id, int32_t world, int32_t rank, qk_dist** out);
QK_EXPORT int32_t qk_dist_info(const qk_dist* dist, int32_t* world, int32_t* rank,
                               int32_t* device);
/* Ends the communicator's pending and future collectives with an error. */
QK_EXPORT int32_t qk_dist_abort(qk_dist* dist);
QK_EXPORT int32_t qk_dist_destroy(qk_dist* dist);
/* The partition rule of the sharded execute, on any list of costs: bounds
 * (world + 1 entries) of contiguous ranges with near-equal total cost;
 * bounds[r] is the item boundary whose cumulative cost is nearest r/world of
 * the total (ties: the earlier one).  Host only (no GPU, no NCCL). */
QK_EXPORT int32_t qk_dist_partition(const double* cost, int64_t n, int32_t world,
                                    int64_t* bounds);
/* This rank's share of a plan on `stream` (NULL: the plan's stream), then
 * qk_mcm_plan_results() as after qk_mcm_plan_execute().  The plan must live
 * on the communicator's device, and every rank's plan must have the same
 * tiling: same inputs, flags and launch shape (a shape chosen by
 * QK_PLAN_AUTOTUNE, or cached from another plan's tuning, can differ between
 * ranks).  Each call first max-reduces a fingerprint of the tiling over the
 * ranks (one small collective and a wait for it) and returns
 * QK_ERR_INVALID_INPUT on every rank when they differ. */
QK_EXPORT int32_t qk_mcm_plan_execute_sharded(qk_mc_plan* plan, qk_dist* dist, void* stream);
/* The pieces of a sharded execute, for callers that move the tile sums with
 * their own transport: the partition (world + 1 tile bounds, host only), the
 * simulate kernels over tiles [tile_begin, tile_end) only, the plan's device
 * array of per-tile sums (n_tiles records of bytes_per_tile bytes, indexed by
 * tile), and the finalize kernel over every option (after every tile's sums
 * are in place).  execute_tiles over each range of the partition, in any
 * order, then finalize, gives what execute() gives. */
QK_EXPORT int32_t qk_mcm_plan_shard_bounds(qk_mc_plan* plan, int32_t world, int64_t* bounds);
QK_EXPORT int32_t qk_mcm_plan_execute_tiles(qk_mc_plan* plan, int64_t tile_begin,
                                            int64_t tile_end, void* stream);
QK_EXPORT int32_t qk_mcm_plan_device_partials(qk_mc_plan* plan, void** d_partials,
                                              int64_t* n_tiles, int32_t* bytes_per_tile);
QK_EXPORT int32_t qk_mcm_plan_finalize(qk_mc_plan* plan, void* stream);
/* qk_mcm_mixed_price_batch across the ranks of `dist`: every rank passes the
 * whole batch and receives every result (equal to the single-GPU call's). */
QK_EXPORT int32_t qk_mcm_mixed_price_batch_sharded(
    qk_dist* dist, const int32_t* model, const double* spot, const double* strike,
    const double* t, const double* vol, const double* r, const double* q, const double* v0,
    const double* kappa, const double* theta, const double* sigma, const double* rho,
    const int32_t* option_type, const int32_t* paths, const int32_t* steps,
    const uint64_t* seed, int32_t n, double* out_prices, double* out_stderr);

/* ======================================================================= *
 * Part 3 -- Heston surrogate (ABI 2.13, no counterpart in the reference)
 * ======================================================================= */

/* Tensor-core building block of the surrogate: C = A . B^T with A [m x k] and
 * B [n x k] bf16 row-major DEVICE pointers (16-byte aligned, k % 64 == 0,
 * n % 64 == 0), fp32 output.  With splits > 1 the k range is cut into `splits`
 * equal parts (k % (64 * splits) == 0) and c holds `splits` partial slabs
 * [splits][m][n].  Asynchronous on `stream` (NULL = default stream). */
QK_EXPORT int32_t qk_sur_gemm_bf16(const void* a, const void* b, float* c, int32_t m, int32_t n,
                                   int32_t k, int32_t splits, void* stream);

/* The surrogate: an MLP 9 -> 256 -> 256 -> 256 -> 1 (SiLU, BF16 weights and
 * activations, FP32 accumulation, FP32 master weights) from the features
 *   f = (S/K, T, r, q, v0, kappa, theta, sigma, rho)
 * to the Heston call price / S.  Inputs are normalised to [-1, 1] over the
 * training box [box_lo, box_hi] (a dimension with lo == hi maps to 0).  The
 * network learns a residual: price / S = base + MLP, with base the
 * Black-Scholes call / S at the Heston mean variance over [0, T],
 *   vbar = theta + (v0 - theta) (1 - exp(-kappa T)) / (kappa T),
 * computed in FP64 from the raw features (targets given to set_dataset and
 * gradients are price / S; the model subtracts the base itself).  It is
 * trained on the GPU by the library's own tcgen05 forward/backward GEMMs and
 * Adam kernels on labels the caller produces (normally this library's Heston
 * Monte Carlo).  Arrays are host arrays unless marked DEVICE; features are
 * row-major n x 9. */
typedef struct qk_sur_model qk_sur_model;

QK_EXPORT int32_t qk_sur_heston_create(const double* box_lo, const double* box_hi, uint64_t seed,
                                       qk_sur_model** out_model);
QK_EXPORT int32_t qk_sur_heston_destroy(qk_sur_model* model);
QK_EXPORT int32_t qk_sur_heston_set_dataset(qk_sur_model* model, const double* features,
                                            const double* target, int64_t n);
/* Adam (beta 0.9/0.999, eps 1e-8), lr cosine-decayed from `lr` over all steps of
 * this call, minibatch `batch` (a multiple of 128), a fresh permutation per
 * epoch.  out_epoch_loss (may be NULL) receives each epoch's mean MSE. */
QK_EXPORT int32_t qk_sur_heston_train(qk_sur_model* model, int32_t epochs, int32_t batch,
                                      double lr, uint64_t shuffle_seed, double* out_epoch_loss);
/* price / S for each row of features (no box check). */
QK_EXPORT int32_t qk_sur_heston_predict(qk_sur_model* model, const double* features, int64_t n,
                                        double* out);
/* Device-resident inference: x_rows = normalised bf16 rows [n][64] (DEVICE,
 * 16-byte aligned) as qk_sur_heston_features(_device) writes them: the nine
 * features in columns 0..8 and zeros in columns 9..63 (this call reads
 * columns 0..15 only), base = the rows' base (DEVICE, fp32; NULL only for a
 * model loaded from a checkpoint without a base), y = price / S (DEVICE,
 * fp32); asynchronous on `stream` (NULL = model's). */
QK_EXPORT int32_t qk_sur_heston_predict_device(qk_sur_model* model, const void* x_rows,
                                               const float* base, int64_t n, float* y,
                                               void* stream);
/* The same inference as three layer-by-layer GEMM launches per 65,536 rows
 * (activations round-trip through device memory): the reference the fused
 * kernel behind qk_sur_heston_predict_device is tested against (same bits). */
QK_EXPORT int32_t qk_sur_heston_predict_device_layered(qk_sur_model* model, const void* x_rows,
                                                       const float* base, int64_t n, float* y,
                                                       void* stream);
/* Normalised bf16 rows [n][64] (HOST output buffer of n*64 uint16) and, when
 * out_base is not NULL, each row's base (n floats). */
QK_EXPORT int32_t qk_sur_heston_features(qk_sur_model* model, const double* features, int64_t n,
                                         void* out_rows, float* out_base);
/* The same on the device: features n x 9 FP64 (DEVICE) -> rows [n][64] bf16
 * (DEVICE, 16-byte aligned) and base (DEVICE, n floats), one launch,
 * asynchronous on `stream` (NULL = model's).  Rows equal qk_sur_heston_features'
 * bit for bit; the base can differ in the last FP32 bit (device exp/erfc). */
QK_EXPORT int32_t qk_sur_heston_features_device(qk_sur_model* model, const double* features,
                                                int64_t n, void* rows, float* base, void* stream);
/* Loss (mean squared error) and its 134,401 gradients for one batch (n a
 * multiple of 128), without an update; replaces the model's dataset. */
QK_EXPORT int32_t qk_sur_heston_gradients(qk_sur_model* model, const double* features,
                                          const double* target, int32_t n, double* grads,
                                          double* loss);
/* Parameters in the order W1[256][9], b1, W2[256][256], b2, W3[256][256], b3,
 * w4[256], b4 (134,401 values). */
QK_EXPORT int32_t qk_sur_heston_parameters(qk_sur_model* model, double* out);
QK_EXPORT int32_t qk_sur_heston_set_parameters(qk_sur_model* model, const double* in);
QK_EXPORT int32_t qk_sur_heston_save(qk_sur_model* model, const char* path);
QK_EXPORT int32_t qk_sur_heston_load(qk_sur_model* model, const char* path);
/* Prices a Heston batch: options whose features lie in the training box are
 * priced by the surrogate (puts by put-call parity), the others by the Heston
 * Monte Carlo with fallback_paths x fallback_steps and seed fallback_seed + i.
 * out_source[i]: 0 surrogate, 1 Monte Carlo fallback, 2 no simulation (invalid
 * input -> NaN, or t <= 1e-12 -> intrinsic value).  May be NULL. */
QK_EXPORT int32_t qk_sur_heston_price_batch(
    qk_sur_model* model, const double* spot, const double* strike, const double* t,
    const double* r, const double* q, const double* v0, const double* kappa, const double* theta,
    const double* sigma, const double* rho, const int32_t* option_type, int32_t n,
    int32_t fallback_paths, int32_t fallback_steps, uint64_t fallback_seed, double* out_prices,
    int32_t* out_source);

#ifdef __cplusplus
}
#endif

#endif /* QK_API_H */
