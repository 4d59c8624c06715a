/*
 * qk_oracle.h -- CPU oracle for the batch Monte Carlo pricing path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it, and only as the checker.
 *
 * Three groups of functions:
 *
 *  1. Exact restatement of the reference MC pricers (yluoc/Quant-Kernel,
 *     cpp/src/common/mc_engine.h:15-136, cpp/src/common/model_concepts.h:93-266,
 *     cpp/src/algorithms/monte_carlo_methods/ *): same MT19937-64 stream, same
 *     libstdc++ polar normal, same draw order and the same floating-point
 *     expression order, so prices match the reference bit for bit.  Each
 *     pricer also returns the standard error the reference never computes.
 *
 *  2. FP64 closed forms: Black-Scholes-Merton (with erfc) and the Heston
 *     characteristic-function price (Gauss-Legendre P1/P2 integration).
 *
 *  3. "Philox replay": the reference step functions in FP64, driven by the
 *     GPU kernels' counter-based Philox4x32-10 + Box-Muller stream.  Given the
 *     same seed, the GPU's FP32 estimate and this FP64 estimate see identical
 *     normals, so their difference isolates FP32 path-state rounding.
 */
#ifndef QK_ORACLE_H
#define QK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- 1. random streams -------------------------------------------------- */
typedef struct {
    uint64_t mt[312];
    int32_t  idx;
    int32_t  has_saved;
    double   saved;
} qko_normal_gen;

void     qko_gen_init(qko_normal_gen* g, uint64_t seed);
uint64_t qko_mt64_next(qko_normal_gen* g);
double   qko_gen_canonical(qko_normal_gen* g);
double   qko_gen_normal(qko_normal_gen* g);
/* Fill out[0..n) with the first n normals of seed's stream (fixture helper). */
void     qko_normals(uint64_t seed, int32_t n, double* out);

/* ---- 1. reference pricers (bit-exact) + standard error ------------------ */
/* Every pricer returns the price and, when se != NULL, writes the standard
 * error of that price (NaN when it is undefined: special cases, < 2 samples). */
double qko_standard_mc(double spot, double strike, double t, double vol, double r, double q,
                       int32_t option_type, int32_t paths, uint64_t seed, double* se);
double qko_antithetic(double spot, double strike, double t, double vol, double r, double q,
                      int32_t option_type, int32_t paths, uint64_t seed, double* se);
double qko_terminal_plain(double spot, double strike, double t, double vol, double r, double q,
                          int32_t option_type, int32_t paths, uint64_t seed, double* se);
double qko_euler(double spot, double strike, double t, double vol, double r, double q,
                 int32_t option_type, int32_t paths, int32_t steps, uint64_t seed, double* se);
double qko_milstein(double spot, double strike, double t, double vol, double r, double q,
                    int32_t option_type, int32_t paths, int32_t steps, uint64_t seed, double* se);
double qko_local_vol(double spot, double strike, double t, double vol, double r, double q,
                     int32_t option_type, int32_t paths, int32_t steps, uint64_t seed, double* se);
double qko_heston(double spot, double strike, double t, double r, double q,
                  double v0, double kappa, double theta, double sigma, double rho,
                  int32_t option_type, int32_t paths, int32_t steps, uint64_t seed, double* se);

/* heston_lr_delta.cpp:37-132: likelihood-ratio delta with antithetic pairs
 * (the RNG state is copied before each pair and replayed negated). */
double qko_heston_lr_delta(double spot, double strike, double t, double r, double q,
                           double v0, double kappa, double theta, double sigma, double rho,
                           int32_t option_type, int32_t paths, int32_t steps, uint64_t seed,
                           double weight_clip, double* se);

/* Terminal GBM with the variance-reduction estimators (control_variates.cpp,
 * importance_sampling.cpp, stratified_sampling.cpp, quasi_monte_carlo.cpp).
 * Standard errors as the GPU defines them (see qk_oracle.c). */
double qko_control_variates(double spot, double strike, double t, double vol, double r, double q,
                            int32_t option_type, int32_t paths, uint64_t seed, double* se);
double qko_importance_sampling(double spot, double strike, double t, double vol, double r,
                               double q, int32_t option_type, int32_t paths, double shift,
                               uint64_t seed, double* se);
double qko_stratified(double spot, double strike, double t, double vol, double r, double q,
                      int32_t option_type, int32_t paths, uint64_t seed, double* se);
double qko_qmc_sobol(double spot, double strike, double t, double vol, double r, double q,
                     int32_t option_type, int32_t paths, double* se);
double qko_qmc_halton(double spot, double strike, double t, double vol, double r, double q,
                      int32_t option_type, int32_t paths, double* se);

/* Batch forms (OpenMP over options when built with it).  out_se may be NULL. */
void qko_heston_batch(const double* spot, const double* strike, const double* t,
                      const double* r, const double* q, const double* v0,
                      const double* kappa, const double* theta, const double* sigma,
                      const double* rho, const int32_t* option_type, const int32_t* paths,
                      const int32_t* steps, const uint64_t* seed, int32_t n,
                      double* out, double* out_se);
/* model: 0 = standard MC (antithetic terminal), 1 = antithetic variates,
 *        2 = Euler, 3 = Milstein, 4 = local vol (constant), 5 = terminal plain,
 *        8 = control variates, 10 = stratified, 11 = QMC Sobol, 12 = QMC Halton */
void qko_bsm_family_batch(int32_t model, const double* spot, const double* strike,
                          const double* t, const double* vol, const double* r,
                          const double* q, const int32_t* option_type, const int32_t* paths,
                          const int32_t* steps, const uint64_t* seed, int32_t n,
                          double* out, double* out_se);

/* ---- 2. closed forms ---------------------------------------------------- */
double qko_bsm_price(double spot, double strike, double t, double vol, double r, double q,
                     int32_t option_type);
double qko_heston_cf_price(double spot, double strike, double t, double r, double q,
                           double v0, double kappa, double theta, double sigma, double rho,
                           int32_t option_type, int32_t integration_steps,
                           double integration_limit);

/* cos_method.cpp:30-58: Heston price by the Fang-Oosterlee COS expansion. */
double qko_heston_cos_price(double spot, double strike, double t, double r, double q,
                            double v0, double kappa, double theta, double sigma, double rho,
                            int32_t option_type, int32_t n_terms, double truncation_width);
/* First-order rounding-error scale of the COS price (defined in qk_oracle.c). */
double qko_heston_cos_error_scale(double spot, double strike, double t, double r, double q,
                              double v0, double kappa, double theta, double sigma, double rho,
                              int32_t option_type, int32_t n_terms, double truncation_width);

/* ---- 3. Philox replay of the GPU stream --------------------------------- */
void qko_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* The terminal kernels' four FP64 normals of quad c0: counters (c0, c1, 0, c3)
 * and (c0, c1 + 1, 0, c3), one Box-Muller pair each; see qk_oracle.c. */
void qko_philox_normals4(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c3, double z[4]);
/* The Heston kernels' six normals of one call (three Box-Muller pairs). */
void qko_philox_normals6(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c3, double z[6]);
/* model as in qko_bsm_family_batch, plus 6 = Heston (uses v0..rho; vol ignored)
 * and 7 = Heston likelihood-ratio delta (vol holds weight_clip).
 * antithetic: 1 = pairs (GPU default), 0 = independent paths. */
double qko_philox_price(int32_t model, double spot, double strike, double t, double vol,
                        double r, double q, double v0, double kappa, double theta,
                        double sigma, double rho, int32_t option_type, int32_t paths,
                        int32_t steps, uint64_t seed, int32_t antithetic, double* se);

/* Variance-reduction models 8-12 (9 = importance sampling with `shift`) on
 * the GPU's Philox stream, FP64, with the GPU's estimators. */
double qko_philox_vr_price(int32_t model, double spot, double strike, double t, double vol,
                           double r, double q, double shift, int32_t option_type, int32_t paths,
                           uint64_t seed, double* se);

#ifdef __cplusplus
}
#endif
#endif /* QK_ORACLE_H */
