/*
 * qk_oracle.c -- CPU oracle for the batch Monte Carlo pricing path.
 *
 * TEST INFRASTRUCTURE ONLY (see qk_oracle.h).  Compiled with
 * -ffp-contract=off so that every expression rounds exactly as written, the
 * way the reference's x86-64 build (no FMA) evaluates it.
 *
 * Citations are into yluoc/Quant-Kernel.
 */
#include "qk_oracle.h"

#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <string.h>

#define QKO_CALL 0
#define QKO_PUT 1
#define QKO_EPS 1e-12 /* monte_carlo_methods/common/internal_util.h:13 */

static double qko_nan(void) {
    /* math_util.h:12-16 writes the quiet NaN bit pattern 0x7FF8000000000000. */
    uint64_t bits = UINT64_C(0x7FF8000000000000);
    double out;
    memcpy(&out, &bits, sizeof out);
    return out;
}

static int qko_finite(double x) {
    /* math_util.h:18-23: finite iff the exponent field is not all ones. */
    uint64_t bits;
    memcpy(&bits, &x, sizeof bits);
    return (bits & UINT64_C(0x7FF0000000000000)) != UINT64_C(0x7FF0000000000000);
}

/* std::max(a, b) is (a < b) ? b : a.  The reference's NaN behaviour follows
 * from this exact form, so the oracle keeps it rather than fmax(). */
static double smax(double a, double b) { return (a < b) ? b : a; }

/* option_util.h:33-38: payoff, NaN for an unknown option type. */
static double intrinsic(double x, double y, int32_t option_type) {
    if (option_type == QKO_CALL) return smax(0.0, x - y);
    if (option_type == QKO_PUT) return smax(0.0, y - x);
    return qko_nan();
}

static int valid_option_type(int32_t ot) { return ot == QKO_CALL || ot == QKO_PUT; }

/* option_util.h:42-50. */
static int valid_common_inputs(double spot, double strike, double t, double vol, double r,
                               double q, int32_t ot) {
    if (!valid_option_type(ot)) return 0;
    if (!qko_finite(spot) || !qko_finite(strike) || !qko_finite(t) || !qko_finite(vol) ||
        !qko_finite(r) || !qko_finite(q))
        return 0;
    return spot > 0.0 && strike > 0.0 && t >= 0.0 && vol >= 0.0;
}

/* monte_carlo_methods/common/internal_util.h:24-26. */
static int valid_mc_counts(int32_t paths, int32_t steps) { return paths > 1 && steps > 0; }

/* ===================================================================== *
 * MT19937-64 (Matsumoto & Nishimura, "Mersenne Twister 64-bit", 2000),
 * with the parameters that the C++ standard fixes for std::mt19937_64.
 * ===================================================================== */
#define MT_N 312
#define MT_M 156
#define MT_UPPER UINT64_C(0xFFFFFFFF80000000)
#define MT_LOWER UINT64_C(0x000000007FFFFFFF)

static void mt_seed(qko_normal_gen* g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < MT_N; ++i) {
        uint64_t prev = g->mt[i - 1];
        g->mt[i] = UINT64_C(6364136223846793005) * (prev ^ (prev >> 62)) + (uint64_t)i;
    }
    g->idx = MT_N;
}

static void mt_twist(qko_normal_gen* g) {
    for (int k = 0; k < MT_N; ++k) {
        uint64_t x = (g->mt[k] & MT_UPPER) | (g->mt[(k + 1) % MT_N] & MT_LOWER);
        uint64_t xa = x >> 1;
        if (x & 1u) xa ^= UINT64_C(0xB5026F5AA96619E9);
        g->mt[k] = g->mt[(k + MT_M) % MT_N] ^ xa;
    }
    g->idx = 0;
}

uint64_t qko_mt64_next(qko_normal_gen* g) {
    if (g->idx >= MT_N) mt_twist(g);
    uint64_t y = g->mt[g->idx++];
    y ^= (y >> 29) & UINT64_C(0x5555555555555555);
    y ^= (y << 17) & UINT64_C(0x71D67FFFEDA60000);
    y ^= (y << 37) & UINT64_C(0xFFF7EEE000000000);
    y ^= y >> 43;
    return y;
}

void qko_gen_init(qko_normal_gen* g, uint64_t seed) {
    /* mc_engine.h:15-23: one engine + one normal_distribution per option. */
    mt_seed(g, seed);
    g->has_saved = 0;
    g->saved = 0.0;
}

/* libstdc++ (GCC 13) generate_canonical<double, 53> over a 64-bit engine:
 * one draw, double(x) / 2^64, and a result that rounds up to 1 replaced by
 * the largest double below 1. */
double qko_gen_canonical(qko_normal_gen* g) {
    double u = (double)qko_mt64_next(g) / 18446744073709551616.0;
    if (u >= 1.0) u = nextafter(1.0, 0.0);
    return u;
}

/* libstdc++ normal_distribution<double>: Marsaglia's polar method.  Each
 * accepted (x, y) yields y * m now and caches x * m for the next call. */
double qko_gen_normal(qko_normal_gen* g) {
    if (g->has_saved) {
        g->has_saved = 0;
        return g->saved * 1.0 + 0.0;
    }
    double x, y, r2;
    do {
        x = 2.0 * qko_gen_canonical(g) - 1.0;
        y = 2.0 * qko_gen_canonical(g) - 1.0;
        r2 = x * x + y * y;
    } while (r2 > 1.0 || r2 == 0.0);
    const double mult = sqrt(-2.0 * log(r2) / r2);
    g->saved = x * mult;
    g->has_saved = 1;
    return (y * mult) * 1.0 + 0.0;
}

void qko_normals(uint64_t seed, int32_t n, double* out) {
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    for (int32_t i = 0; i < n; ++i) out[i] = qko_gen_normal(&g);
}

/* ===================================================================== *
 * Running moments for the standard error.  The price sums stay plain
 * double additions in the reference's order (bit-exactness); the squared
 * sums only feed the standard error.
 * ===================================================================== */
static double se_from_moments(double disc, double sum, double sumsq, double n) {
    if (!(n >= 2.0)) return qko_nan();
    double mean = sum / n;
    double var = (sumsq - n * mean * mean) / (n - 1.0);
    if (var < 0.0) var = 0.0;
    return disc * sqrt(var / n);
}

/* model_concepts.h:93-102 make_bsm_terminal. */
static double bsm_terminal(double vol, double r, double q, double spot, double t, double z) {
    double drift = (r - q - 0.5 * vol * vol) * t;
    double diffusion = vol * sqrt(smax(t, 0.0)) * z;
    return spot * exp(drift + diffusion);
}

/* mc_engine.h:32-53 estimate_terminal_antithetic with the payoff accumulator.
 * Standard error over the n/2 pair means (the lone odd path is left out of
 * the variance, it is in the mean). */
static double est_terminal_antithetic(double spot, double strike, double t, double vol, double r,
                                      double q, int32_t ot, int32_t n_paths, uint64_t seed,
                                      double disc, double* se) {
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    double sum = 0.0, psum = 0.0, psq = 0.0;
    const int32_t n_pairs = n_paths / 2;
    for (int32_t i = 0; i < n_pairs; ++i) {
        const double z = qko_gen_normal(&g);
        const double st_up = bsm_terminal(vol, r, q, spot, t, z);
        const double st_dn = bsm_terminal(vol, r, q, spot, t, -z);
        const double a = intrinsic(st_up, strike, ot);
        const double b = intrinsic(st_dn, strike, ot);
        sum += a;
        sum += b;
        const double m = 0.5 * (a + b);
        psum += m;
        psq += m * m;
    }
    if ((n_paths & 1) != 0) {
        const double z = qko_gen_normal(&g);
        const double st = bsm_terminal(vol, r, q, spot, t, z);
        sum += intrinsic(st, strike, ot);
    }
    const double mean = sum / (double)n_paths;
    if (se) *se = se_from_moments(disc, psum, psq, (double)n_pairs);
    return disc * mean;
}

/* standard_monte_carlo.cpp:11-33. */
double qko_standard_mc(double spot, double strike, double t, double vol, double r, double q,
                       int32_t ot, int32_t paths, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths <= 1) return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    if (vol <= QKO_EPS) {
        const double fwd = spot * exp((r - q) * t);
        return exp(-r * t) * intrinsic(fwd, strike, ot);
    }
    const double disc = exp(-r * t);
    return est_terminal_antithetic(spot, strike, t, vol, r, q, ot, paths, seed, disc, se);
}

/* antithetic_variates.cpp:11-29 (no zero-vol branch). */
double qko_antithetic(double spot, double strike, double t, double vol, double r, double q,
                      int32_t ot, int32_t paths, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths <= 1) return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    return est_terminal_antithetic(spot, strike, t, vol, r, q, ot, paths, seed, disc, se);
}

/* mc_engine.h:62-75 estimate_terminal (the plain loop; the reference runs it
 * under importance sampling, here with the BSM terminal model and payoff). */
double qko_terminal_plain(double spot, double strike, double t, double vol, double r, double q,
                          int32_t ot, int32_t paths, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths <= 1) return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    double sum = 0.0, sq = 0.0;
    for (int32_t i = 0; i < paths; ++i) {
        const double z = qko_gen_normal(&g);
        const double p = intrinsic(bsm_terminal(vol, r, q, spot, t, z), strike, ot);
        sum += p;
        sq += p * p;
    }
    if (se) *se = se_from_moments(disc, sum, sq, (double)paths);
    return disc * (sum / (double)paths);
}

/* mc_engine.h:84-103 estimate_stepwise with
 *   kind 0: make_bsm_euler_step    (model_concepts.h:136-143)
 *   kind 1: make_bsm_milstein_step (model_concepts.h:150-158) */
static double est_stepwise(int kind, double spot, double strike, double t, double vol,
                           double drift, int32_t ot, int32_t n_paths, int32_t steps,
                           uint64_t seed, double disc, double* se) {
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    const double dt = t / (double)steps;
    const double sqrt_dt = sqrt(dt);
    double sum = 0.0, sq = 0.0;
    for (int32_t i = 0; i < n_paths; ++i) {
        double s = spot;
        for (int32_t j = 0; j < steps; ++j) {
            double dw = sqrt_dt * qko_gen_normal(&g);
            if (kind == 0)
                s = smax(1e-12, s + drift * s * dt + vol * s * dw);
            else
                s = smax(1e-12, s + drift * s * dt + vol * s * dw +
                                    0.5 * vol * vol * s * (dw * dw - dt));
        }
        const double p = intrinsic(s, strike, ot);
        sum += p;
        sq += p * p;
    }
    if (se) *se = se_from_moments(disc, sum, sq, (double)n_paths);
    return disc * (sum / (double)n_paths);
}

/* euler_maruyama.cpp:11-28. */
double qko_euler(double spot, double strike, double t, double vol, double r, double q,
                 int32_t ot, int32_t paths, int32_t steps, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || !valid_mc_counts(paths, steps))
        return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    return est_stepwise(0, spot, strike, t, vol, r - q, ot, paths, steps, seed, disc, se);
}

/* milstein.cpp:11-28. */
double qko_milstein(double spot, double strike, double t, double vol, double r, double q,
                    int32_t ot, int32_t paths, int32_t steps, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || !valid_mc_counts(paths, steps))
        return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    return est_stepwise(1, spot, strike, t, vol, r - q, ot, paths, steps, seed, disc, se);
}

/* local_vol_monte_carlo.cpp:20-48 (local_vol_price_impl) with the constant
 * sigma_fn of model_concepts.h:240-266 and the entry checks of :57-73.  The
 * reference discounts as disc * sum / paths here, not disc * (sum / paths). */
double qko_local_vol(double spot, double strike, double t, double vol, double r, double q,
                     int32_t ot, int32_t paths, int32_t steps, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || !valid_mc_counts(paths, steps))
        return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    const double dt = t / (double)steps;
    const double sqrt_dt = sqrt(dt);
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    double sum = 0.0, sq = 0.0;
    for (int32_t i = 0; i < paths; ++i) {
        double s = spot;
        double current_t = 0.0;
        for (int32_t j = 0; j < steps; ++j) {
            const double dw = sqrt_dt * qko_gen_normal(&g);
            const double sig = vol; /* sigma_fn(s, current_t) */
            s = smax(1e-12, s + (r - q) * s * dt + sig * s * dw);
            current_t += dt;
        }
        (void)current_t;
        const double p = intrinsic(s, strike, ot);
        sum += p;
        sq += p * p;
    }
    if (se) *se = se_from_moments(disc, sum, sq, (double)paths);
    return disc * sum / (double)paths;
}

/* heston_monte_carlo.cpp:11-36 driving mc_engine.h:113-136
 * estimate_stepwise_2d with make_heston_euler_step (model_concepts.h:205-226). */
double qko_heston(double spot, double strike, double t, double r, double q, double v0,
                  double kappa, double theta, double sigma, double rho, int32_t ot,
                  int32_t paths, int32_t steps, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_option_type(ot) || spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0 ||
        kappa < 0.0 || theta < 0.0 || sigma < 0.0 || rho < -1.0 || rho > 1.0 ||
        !valid_mc_counts(paths, steps))
        return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    const double rho_comp = sqrt(smax(1.0 - rho * rho, 0.0));
    const double dt = t / (double)steps;
    const double sqrt_dt = sqrt(dt);
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    double sum = 0.0, sq = 0.0;
    for (int32_t i = 0; i < paths; ++i) {
        double s = spot;
        double v = v0;
        for (int32_t j = 0; j < steps; ++j) {
            const double z1 = qko_gen_normal(&g);
            const double z2 = qko_gen_normal(&g);
            const double v_pos = smax(v, 0.0);
            const double sqrt_v = sqrt(v_pos);
            const double dw1 = sqrt_dt * z1;
            const double dw2 = sqrt_dt * (rho * z1 + rho_comp * z2);
            const double s_next = s * exp((r - q - 0.5 * v_pos) * dt + sqrt_v * dw1);
            const double v_next = smax(0.0, v + kappa * (theta - v_pos) * dt + sigma * sqrt_v * dw2);
            s = smax(s_next, 1e-12);
            v = v_next;
        }
        const double p = intrinsic(s, strike, ot);
        sum += p;
        sq += p * p;
    }
    if (se) *se = se_from_moments(disc, sum, sq, (double)paths);
    return disc * (sum / (double)paths);
}

/* std::min(a, b) is (b < a) ? b : a. */
static double smin(double a, double b) { return (b < a) ? b : a; }

/* heston_lr_delta.cpp:37-132.  Standard error over the pair samples
 * (pf w - pa w) / 2; the unpaired path of an odd count is in the mean only. */
double qko_heston_lr_delta(double spot, double strike, double t, double r, double q, double v0,
                           double kappa, double theta, double sigma, double rho, int32_t ot,
                           int32_t paths, int32_t steps, uint64_t seed, double weight_clip,
                           double* se) {
    if (se) *se = qko_nan();
    if (!valid_option_type(ot) || spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0 ||
        kappa < 0.0 || theta < 0.0 || sigma < 0.0 || rho < -1.0 || rho > 1.0 ||
        !valid_mc_counts(paths, steps) || weight_clip <= 0.0)
        return qko_nan();
    if (t <= QKO_EPS) {
        if (ot == QKO_CALL) return (spot > strike) ? 1.0 : 0.0;
        return (spot < strike) ? -1.0 : 0.0;
    }
    const double disc = exp(-r * t);
    const double dt = t / (double)steps;
    const double sqrt_dt = sqrt(dt);
    const double sqrt_v0 = sqrt(smax(v0, 0.0));
    const double rho_comp = sqrt(smax(1.0 - rho * rho, 0.0));
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    double sum = 0.0, ysum = 0.0, ysq = 0.0;
    const int32_t n_pairs = paths / 2;
#define LR_STEP(z1_, z2_)                                                                      \
    do {                                                                                       \
        const double v_pos = smax(v, 0.0);                                                     \
        const double sqrt_v = sqrt(v_pos);                                                     \
        const double dw1 = sqrt_dt * (z1_);                                                    \
        const double dw2 = sqrt_dt * (rho * (z1_) + rho_comp * (z2_));                         \
        const double s_next = s * exp((r - q - 0.5 * v_pos) * dt + sqrt_v * dw1);              \
        v = smax(0.0, v + kappa * (theta - v_pos) * dt + sigma * sqrt_v * dw2);                \
        s = smax(s_next, 1e-12);                                                               \
    } while (0)
    for (int32_t i = 0; i < n_pairs; ++i) {
        qko_normal_gen saved = g;
        double s = spot, v = v0, z1_first = 0.0;
        for (int32_t j = 0; j < steps; ++j) {
            const double z1 = qko_gen_normal(&g);
            const double z2 = qko_gen_normal(&g);
            if (j == 0) z1_first = z1;
            LR_STEP(z1, z2);
        }
        const double pf = intrinsic(s, strike, ot);
        double score = (sqrt_v0 > 1e-15) ? z1_first / (sqrt_v0 * sqrt_dt * spot) : 0.0;
        score = smax(-weight_clip, smin(weight_clip, score));
        s = spot;
        v = v0;
        for (int32_t j = 0; j < steps; ++j) {
            const double z1 = -qko_gen_normal(&saved);
            const double z2 = -qko_gen_normal(&saved);
            LR_STEP(z1, z2);
        }
        const double pa = intrinsic(s, strike, ot);
        const double y = pf * score + pa * (-score);
        sum += y;
        ysum += 0.5 * y;
        ysq += 0.25 * y * y;
    }
    if ((paths & 1) != 0) {
        double s = spot, v = v0, z1_first = 0.0;
        for (int32_t j = 0; j < steps; ++j) {
            const double z1 = qko_gen_normal(&g);
            const double z2 = qko_gen_normal(&g);
            if (j == 0) z1_first = z1;
            LR_STEP(z1, z2);
        }
        const double p = intrinsic(s, strike, ot);
        double score = (sqrt_v0 > 1e-15) ? z1_first / (sqrt_v0 * sqrt_dt * spot) : 0.0;
        score = smax(-weight_clip, smin(weight_clip, score));
        sum += p * score;
    }
#undef LR_STEP
    if (se) *se = se_from_moments(disc, ysum, ysq, (double)n_pairs);
    return disc * sum / (double)paths;
}

/* ===================================================================== *
 * 1b. Terminal GBM with the reference's variance-reduction estimators.
 * ===================================================================== */

/* Acklam's inverse normal CDF as the reference evaluates it
 * (monte_carlo_methods/common/internal_util.h:42-90; P. J. Acklam, "An
 * algorithm for computing the inverse normal cumulative distribution
 * function", 2003): same coefficients, same Horner order. */
static double acklam_inv(double p) {
    static const double a1 = -3.969683028665376e+01, a2 = 2.209460984245205e+02,
                        a3 = -2.759285104469687e+02, a4 = 1.383577518672690e+02,
                        a5 = -3.066479806614716e+01, a6 = 2.506628277459239e+00;
    static const double b1 = -5.447609879822406e+01, b2 = 1.615858368580409e+02,
                        b3 = -1.556989798598866e+02, b4 = 6.680131188771972e+01,
                        b5 = -1.328068155288572e+01;
    static const double c1 = -7.784894002430293e-03, c2 = -3.223964580411365e-01,
                        c3 = -2.400758277161838e+00, c4 = -2.549732539343734e+00,
                        c5 = 4.374664141464968e+00, c6 = 2.938163982698783e+00;
    static const double d1 = 7.784695709041462e-03, d2 = 3.224671290700398e-01,
                        d3 = 2.445134137142996e+00, d4 = 3.754408661907416e+00;
    const double p_low = 0.02425, p_high = 1.0 - p_low;
    if (p <= 0.0 || p >= 1.0) return qko_nan();
    if (p < p_low) {
        const double t = sqrt(-2.0 * log(p));
        return (((((c1 * t + c2) * t + c3) * t + c4) * t + c5) * t + c6) /
               ((((d1 * t + d2) * t + d3) * t + d4) * t + 1.0);
    }
    if (p > p_high) {
        const double t = sqrt(-2.0 * log(1.0 - p));
        return -(((((c1 * t + c2) * t + c3) * t + c4) * t + c5) * t + c6) /
               ((((d1 * t + d2) * t + d3) * t + d4) * t + 1.0);
    }
    const double t = p - 0.5;
    const double r = t * t;
    return (((((a1 * r + a2) * r + a3) * r + a4) * r + a5) * r + a6) * t /
           (((((b1 * r + b2) * r + b3) * r + b4) * r + b5) * r + 1.0);
}

/* std::clamp(u, 1e-12, 1 - 1e-12) */
static double clamp_unit(double u) {
    return (u < 1e-12) ? 1e-12 : (((1.0 - 1e-12) < u) ? 1.0 - 1e-12 : u);
}

/* internal_util.h:104-119: bit j of gray(i) contributes 1 << (31 - j). */
static double sobol_point(uint32_t i) {
    if (i == 0u) return 0.0;
    uint32_t gray = i ^ (i >> 1), x = 0u;
    for (uint32_t bit = 0; gray != 0u; ++bit, gray >>= 1)
        if (gray & 1u) x ^= (1u << (31u - bit));
    return ((double)x + 0.5) / 4294967296.0;
}

/* internal_util.h:121-130: radical inverse in `base`. */
static double halton_point(uint32_t i, uint32_t base) {
    double f = 1.0, r = 0.0;
    while (i > 0u) {
        f /= (double)base;
        r += f * (double)(i % base);
        i /= base;
    }
    return r;
}

/* Standard errors shared with the GPU (none of these exist in the reference):
 * control variates -- residual variance of payoff - beta * control over
 * n - 2, from sums of the payoff p and the centred control c = S_T - E[S_T];
 * the degenerate-control branch falls back to the plain sample variance. */
static double cv_se(double disc, double sp, double spp, double sc, double scc, double scp,
                    double n) {
    const double mp = sp / n, mc = sc / n;
    const double vc = scc / n - mc * mc, vp = spp / n - mp * mp;
    if (disc * disc * vc <= QKO_EPS) return n >= 2.0 ? disc * sqrt(smax(vp, 0.0) / (n - 1.0)) : qko_nan();
    const double cov = scp / n - mc * mp;
    return disc * sqrt(smax(vp - cov * (cov / vc), 0.0) / (n - 2.0));
}

/* control_variates.cpp:10-52. */
double qko_control_variates(double spot, double strike, double t, double vol, double r, double q,
                            int32_t ot, int32_t paths, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths <= 2) return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    const double disc = exp(-r * t);
    const double expected_x = spot * exp(-q * t);
    const double mean_st = spot * exp((r - q) * t);
    double sum_y = 0.0, sum_x = 0.0, sum_xx = 0.0, sum_xy = 0.0;
    double sp = 0.0, spp = 0.0, sc = 0.0, scc = 0.0, scp = 0.0;
    for (int32_t i = 0; i < paths; ++i) {
        const double z = qko_gen_normal(&g);
        const double st = bsm_terminal(vol, r, q, spot, t, z);
        const double x = disc * st;
        const double pay = intrinsic(st, strike, ot);
        const double y = disc * pay;
        sum_y += y;
        sum_x += x;
        sum_xx += x * x;
        sum_xy += x * y;
        const double c = st - mean_st;
        sp += pay;
        spp += pay * pay;
        sc += c;
        scc += c * c;
        scp += c * pay;
    }
    if (se) *se = cv_se(disc, sp, spp, sc, scc, scp, (double)paths);
    const double mean_y = sum_y / (double)paths;
    const double mean_x = sum_x / (double)paths;
    const double var_x = (sum_xx / (double)paths) - mean_x * mean_x;
    if (var_x <= QKO_EPS) return mean_y;
    const double cov_xy = (sum_xy / (double)paths) - mean_x * mean_y;
    const double beta = cov_xy / var_x;
    return mean_y - beta * (mean_x - expected_x);
}

/* importance_sampling.cpp:11-36 driving mc_engine.h:62-75 estimate_terminal. */
double qko_importance_sampling(double spot, double strike, double t, double vol, double r,
                               double q, int32_t ot, int32_t paths, double shift, uint64_t seed,
                               double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths <= 1 || !qko_finite(shift))
        return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    double sum = 0.0, sq = 0.0;
    for (int32_t i = 0; i < paths; ++i) {
        const double z = qko_gen_normal(&g);
        const double st = bsm_terminal(vol, r, q, spot, t, z + shift);
        const double y = z + shift;
        const double weight = exp(-shift * y + 0.5 * shift * shift);
        const double a = intrinsic(st, strike, ot) * weight;
        sum += a;
        sq += a * a;
    }
    if (se) *se = se_from_moments(disc, sum, sq, (double)paths);
    return disc * (sum / (double)paths);
}

/* stratified_sampling.cpp:11-35; uniform_real_distribution(0, 1) is one
 * generate_canonical draw, u * (1 - 0) + 0. */
double qko_stratified(double spot, double strike, double t, double vol, double r, double q,
                      int32_t ot, int32_t paths, uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths <= 1) return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    qko_normal_gen g;
    qko_gen_init(&g, seed);
    const double disc = exp(-r * t);
    double sum = 0.0, dsq = 0.0, prev = 0.0;
    for (int32_t i = 0; i < paths; ++i) {
        double u = ((double)i + (qko_gen_canonical(&g) * (1.0 - 0.0) + 0.0)) / (double)paths;
        u = clamp_unit(u);
        const double z = acklam_inv(u);
        const double st = bsm_terminal(vol, r, q, spot, t, z);
        const double a = intrinsic(st, strike, ot);
        sum += a;
        if (i & 1) dsq += (prev - a) * (prev - a);
        prev = a;
    }
    if (se) *se = disc * sqrt(dsq) / (double)paths;
    return disc * (sum / (double)paths);
}

/* quasi_monte_carlo.cpp:10-56 (kind 0: Sobol, 1: Halton base 2). */
static double qmc_price(int kind, double spot, double strike, double t, double vol, double r,
                        double q, int32_t ot, int32_t paths, double* se) {
    if (se) *se = qko_nan();
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths <= 1) return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    double sum = 0.0, sq = 0.0;
    for (int32_t i = 1; i <= paths; ++i) {
        double u = kind == 0 ? sobol_point((uint32_t)i) : halton_point((uint32_t)i, 2u);
        u = clamp_unit(u);
        const double z = acklam_inv(u);
        const double st = bsm_terminal(vol, r, q, spot, t, z);
        const double a = intrinsic(st, strike, ot);
        sum += a;
        sq += a * a;
    }
    if (se) *se = se_from_moments(disc, sum, sq, (double)paths);
    return disc * (sum / (double)paths);
}

double qko_qmc_sobol(double spot, double strike, double t, double vol, double r, double q,
                     int32_t ot, int32_t paths, double* se) {
    return qmc_price(0, spot, strike, t, vol, r, q, ot, paths, se);
}

double qko_qmc_halton(double spot, double strike, double t, double vol, double r, double q,
                      int32_t ot, int32_t paths, double* se) {
    return qmc_price(1, spot, strike, t, vol, r, q, ot, paths, se);
}

void qko_heston_batch(const double* spot, const double* strike, const double* t,
                      const double* r, const double* q, const double* v0, const double* kappa,
                      const double* theta, const double* sigma, const double* rho,
                      const int32_t* ot, const int32_t* paths, const int32_t* steps,
                      const uint64_t* seed, int32_t n, double* out, double* out_se) {
#pragma omp parallel for schedule(dynamic)
    for (int32_t i = 0; i < n; ++i) {
        double se;
        out[i] = qko_heston(spot[i], strike[i], t[i], r[i], q[i], v0[i], kappa[i], theta[i],
                            sigma[i], rho[i], ot[i], paths[i], steps[i], seed[i], &se);
        if (out_se) out_se[i] = se;
    }
}

void qko_bsm_family_batch(int32_t model, const double* spot, const double* strike,
                          const double* t, const double* vol, const double* r, const double* q,
                          const int32_t* ot, const int32_t* paths, const int32_t* steps,
                          const uint64_t* seed, int32_t n, double* out, double* out_se) {
#pragma omp parallel for schedule(dynamic)
    for (int32_t i = 0; i < n; ++i) {
        double se = qko_nan(), p;
        const int32_t st = steps ? steps[i] : 1;
        switch (model) {
            case 0: p = qko_standard_mc(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], seed[i], &se); break;
            case 1: p = qko_antithetic(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], seed[i], &se); break;
            case 2: p = qko_euler(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], st, seed[i], &se); break;
            case 3: p = qko_milstein(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], st, seed[i], &se); break;
            case 4: p = qko_local_vol(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], st, seed[i], &se); break;
            case 5: p = qko_terminal_plain(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], seed[i], &se); break;
            case 8: p = qko_control_variates(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], seed[i], &se); break;
            case 10: p = qko_stratified(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], seed[i], &se); break;
            case 11: p = qko_qmc_sobol(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], &se); break;
            case 12: p = qko_qmc_halton(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i], paths[i], &se); break;
            default: p = qko_nan(); break;
        }
        out[i] = p;
        if (out_se) out_se[i] = se;
    }
}

/* ===================================================================== *
 * 2. Closed forms.
 * ===================================================================== */

static double norm_cdf_exact(double x) { return 0.5 * erfc(-x / sqrt(2.0)); }

/* black_scholes_merton.cpp:7-33 with an erfc-based normal CDF (the
 * reference uses the A&S 7.1.26 approximation, max error ~1.5e-7). */
double qko_bsm_price(double spot, double strike, double t, double vol, double r, double q,
                     int32_t ot) {
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot)) return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    if (vol <= QKO_EPS) {
        double fwd = spot * exp((r - q) * t);
        return exp(-r * t) * intrinsic(fwd, strike, ot);
    }
    double sqrt_t = sqrt(t);
    double d1 = (log(spot / strike) + (r - q + 0.5 * vol * vol) * t) / (vol * sqrt_t);
    double d2 = d1 - vol * sqrt_t;
    double df = exp(-r * t), qf = exp(-q * t);
    if (ot == QKO_CALL) return spot * qf * norm_cdf_exact(d1) - strike * df * norm_cdf_exact(d2);
    return strike * df * norm_cdf_exact(-d2) - spot * qf * norm_cdf_exact(-d1);
}

/* 64-point Gauss-Legendre rule on [-1, 1]: the 32 positive nodes and their
 * weights, computed once by Newton's method on the Legendre recurrence. */
static double clamp01(double x) {
    const double lo = (0.0 < x) ? x : 0.0; /* std::max(0.0, x) */
    return (1.0 < lo) ? 1.0 : lo;           /* std::min(1.0, lo) */
}

static double gl_x[32], gl_w[32];
static int gl_ready = 0;

static void gl_init(void) {
    if (gl_ready) return;
    const int n = 64;
    for (int i = 0; i < 32; ++i) {
        /* Tricomi's initial guess for root i (descending from 1). */
        double x = cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = pk;
            }
            dp = n * (x * p1 - p0) / (x * x - 1.0);
            double dx = p1 / dp;
            x -= dx;
            if (fabs(dx) < 1e-16) break;
        }
        /* store ascending: index 31 - i */
        gl_x[31 - i] = x;
        gl_w[31 - i] = 2.0 / ((1.0 - x * x) * dp * dp);
    }
    gl_ready = 1;
}

/* heston.cpp:7-53 (little-trap characteristic function) with the P1/P2
 * integration of closed_form_semi_analytical/common/internal_util.h:80-142:
 * ceil(steps/64) panels of the 64-point rule on [1e-8, limit]. */
double qko_heston_cf_price(double spot, double strike, double t, double r, double q, double v0,
                           double kappa, double theta, double sigma, double rho, int32_t ot,
                           int32_t integration_steps, double integration_limit) {
    if (!valid_option_type(ot)) return qko_nan();
    if (!qko_finite(spot) || !qko_finite(strike) || !qko_finite(t) || !qko_finite(r) ||
        !qko_finite(q) || !qko_finite(v0) || !qko_finite(kappa) || !qko_finite(theta) ||
        !qko_finite(sigma) || !qko_finite(rho))
        return qko_nan();
    if (spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0 || kappa <= 0.0 || theta < 0.0 ||
        sigma <= 0.0 || rho <= -1.0 || rho >= 1.0)
        return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    if (integration_steps < 16 || integration_limit <= 1e-6) return qko_nan();
    gl_init();

    const double sig2 = sigma * sigma;
    const double kts2 = kappa * theta / sig2;
    const double drift = log(spot) + (r - q) * t;
    const double lk = log(strike);

#define HESTON_CF(u_, out_)                                                               \
    do {                                                                                  \
        double complex iu_ = I * (u_);                                                    \
        double complex beta_ = kappa - rho * sigma * iu_;                                 \
        double complex d_ = csqrt(beta_ * beta_ + sig2 * (iu_ + (u_) * (u_)));            \
        double complex bmd_ = beta_ - d_;                                                 \
        double complex g_ = bmd_ / (beta_ + d_);                                          \
        double complex e_ = cexp(-d_ * t);                                                \
        double complex C_ = iu_ * drift + kts2 * (bmd_ * t - 2.0 * clog((1.0 - g_ * e_) / (1.0 - g_))); \
        double complex D_ = (bmd_ / sig2) * ((1.0 - e_) / (1.0 - g_ * e_));               \
        (out_) = cexp(C_ + D_ * v0);                                                      \
    } while (0)

    double complex phi_mi;
    HESTON_CF(-I, phi_mi);
    const double phi_abs = cabs(phi_mi);
    const int panels = (integration_steps + 63) / 64 > 1 ? (integration_steps + 63) / 64 : 1;
    const double a = 1e-8, b = integration_limit;
    const double width = (b - a) / panels;
    double s1 = 0.0, s2 = 0.0;
    for (int p = 0; p < panels; ++p) {
        const double pa = a + p * width;
        const double mid = pa + 0.5 * width, half = 0.5 * width;
        for (int i = 0; i < 32; ++i) {
            for (int side = 0; side < 2; ++side) {
                const double u = side ? mid + half * gl_x[i] : mid - half * gl_x[i];
                const double complex rot = cexp(-I * u * lk) / (I * u);
                double complex c2;
                HESTON_CF(u, c2);
                s2 += half * gl_w[i] * creal(rot * c2);
                if (phi_abs >= 1e-14) {
                    double complex c1;
                    HESTON_CF(u - I, c1);
                    s1 += half * gl_w[i] * creal(rot * c1 / phi_mi);
                }
            }
        }
    }
#undef HESTON_CF
    /* clamp01 (internal_util.h:25-27) is std::min(1, std::max(0, x)), which
     * maps NaN to 0; p1 is NaN unless |phi(-i)| >= 1e-14 holds, which fails
     * for a NaN phi(-i) too (kappa = rho sigma: beta + d = 0 at u = -i). */
    double p2 = 0.5 + s2 / M_PI;
    double p1 = 0.5 + s1 / M_PI;
    p2 = clamp01(p2);
    p1 = clamp01(p1);
    if (!(phi_abs >= 1e-14)) return qko_nan();
    const double call = spot * exp(-q * t) * p1 - strike * exp(-r * t) * p2;
    if (ot == QKO_CALL) return call;
    /* put-call parity */
    return call - spot * exp(-q * t) + strike * exp(-r * t);
}

/* cos_method.cpp:30-58 (Heston COS, Fang-Oosterlee) with the Heston log-price
 * characteristic function of charfn_concepts.h:54-78 and the sum of
 * cos_method.h:13-57, in the same expression order. */
static double complex heston_log_charfn(double spot, double r, double q, double v0, double kappa,
                                        double theta, double sigma, double rho, double complex u,
                                        double t, double* mag) {
    const double complex i = CMPLX(0.0, 1.0);
    const double complex iu = i * u;
    const double complex a = kappa - rho * sigma * iu;
    const double complex b = sigma * sigma * (iu + u * u);
    const double complex d = csqrt(a * a + b);
    const double complex g = (a - d) / (a + d);
    const double complex edt = cexp(-d * t);
    const double complex lg = clog((1.0 - g * edt) / (1.0 - g));
    const double complex C = (kappa * theta / (sigma * sigma)) * ((a - d) * t - 2.0 * lg);
    const double complex D = ((a - d) / (sigma * sigma)) * (1.0 - edt) / (1.0 - g * edt);
    if (mag) {
        /* Sizes of the exponent's parts before they cancel.  a - d is a
         * difference of two numbers of size |a| + |d|, so its rounding error
         * is of that size, and 1/sigma^2 carries it into C and D. */
        const double ad = cabs(a) + cabs(d);
        *mag = cabs(u) * (fabs(log(spot)) + fabs((r - q) * t)) +
               fabs(kappa * theta / (sigma * sigma)) * (ad * t + 2.0 * (cabs(lg) + 1.0)) +
               fabs(v0) * ad / (sigma * sigma) * cabs(1.0 - edt) / cabs(1.0 - g * edt);
    }
    return cexp(iu * log(spot) + iu * (r - q) * t + C + D * v0);
}

/* The COS price, and in *err_scale (when not NULL) a first-order scale of its
 * rounding error: exp(-r t) sum_k |w_k f_k u_k| (1 + M_k), M_k the size of
 * term k's exponent parts (and of its phase u a) before they cancel.  An
 * absolute error e in an exponent is a relative error e in its exp(), so
 * another correctly working evaluation (other libm, other summation order)
 * lands within a modest multiple of DBL_EPSILON x this scale. */
static double heston_cos_impl(double spot, double strike, double t, double r, double q, double v0,
                              double kappa, double theta, double sigma, double rho, int32_t ot,
                              int32_t n_terms, double truncation_width, double* err_scale);

double qko_heston_cos_price(double spot, double strike, double t, double r, double q, double v0,
                            double kappa, double theta, double sigma, double rho, int32_t ot,
                            int32_t n_terms, double truncation_width) {
    return heston_cos_impl(spot, strike, t, r, q, v0, kappa, theta, sigma, rho, ot, n_terms,
                           truncation_width, NULL);
}

double qko_heston_cos_error_scale(double spot, double strike, double t, double r, double q,
                              double v0, double kappa, double theta, double sigma, double rho,
                              int32_t ot, int32_t n_terms, double truncation_width) {
    double a = 0.0;
    heston_cos_impl(spot, strike, t, r, q, v0, kappa, theta, sigma, rho, ot, n_terms,
                    truncation_width, &a);
    return a;
}

static double heston_cos_impl(double spot, double strike, double t, double r, double q, double v0,
                              double kappa, double theta, double sigma, double rho, int32_t ot,
                              int32_t n_terms, double truncation_width, double* err_scale) {
    if (!valid_option_type(ot)) return qko_nan();
    if (!qko_finite(spot) || !qko_finite(strike) || !qko_finite(t) || !qko_finite(r) ||
        !qko_finite(q) || !qko_finite(v0) || !qko_finite(kappa) || !qko_finite(theta) ||
        !qko_finite(sigma) || !qko_finite(rho) || !qko_finite(truncation_width))
        return qko_nan();
    if (spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0) return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    if (n_terms < 8 || truncation_width <= 0.0) return qko_nan();
    const double eff_var = smax(v0, theta);
    const double c1 = log(spot) + (r - q - 0.5 * eff_var) * t;
    const double c2 = eff_var * t;
    const double a = c1 - truncation_width * sqrt(smax(c2, 0.0));
    const double b = c1 + truncation_width * sqrt(smax(c2, 0.0));
    if (!(b > a + QKO_EPS)) return qko_nan();
    const double log_strike = log(strike);
    const double c = (log_strike < a ? a : log_strike) > b ? b : (log_strike < a ? a : log_strike);
    const double dd = b;
    double call = 0.0;
    if (c < dd) {
        const double interval = b - a;
        const double inv = 1.0 / interval;
        double sum = 0.0;
        for (int32_t k = 0; k < n_terms; ++k) {
            const double u = (double)k * M_PI * inv;
            double chi, psi;
            if (k == 0) {
                chi = exp(dd) - exp(c);
                psi = dd - c;
            } else {
                const double ud = u * (dd - a), uc = u * (c - a);
                const double exp_d = exp(dd), exp_c = exp(c);
                chi = ((cos(ud) * exp_d - cos(uc) * exp_c) + u * (sin(ud) * exp_d - sin(uc) * exp_c)) /
                      (1.0 + u * u);
                psi = (sin(ud) - sin(uc)) / u;
            }
            const double u_k = 2.0 * inv * (chi - strike * psi);
            double mag = 0.0;
            const double complex phi = heston_log_charfn(spot, r, q, v0, kappa, theta, sigma, rho,
                                                         CMPLX(u, 0.0), t, err_scale ? &mag : NULL);
            const double f_k = creal(phi * cexp(-CMPLX(0.0, 1.0) * (u * a)));
            const double weight = (k == 0) ? 0.5 : 1.0;
            sum += weight * f_k * u_k;
            if (err_scale) *err_scale += fabs(weight * f_k * u_k) * (1.0 + mag + fabs(u * a));
        }
        call = exp(-r * t) * sum;
        if (err_scale) *err_scale *= exp(-r * t);
    }
    call = smax(0.0, call);
    if (ot == QKO_CALL) return call;
    return call - spot * exp(-q * t) + strike * exp(-r * t);
}

/* ===================================================================== *
 * 3. Philox replay.
 *
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with a
 * Weyl-sequence key schedule.
 *
 * The GPU kernels draw their normals from this counter layout:
 *   key      = (low 32 bits of seed, high 32 bits of seed)
 *   counter  = (unit, block, 0, c3)   c3 = 0 antithetic pairs, 1 plain paths
 * Terminal models (FP64 normals): normal k of the option (k = pair index, or
 *   path index when plain) is slot k % 4 of quad k / 4; the quad's counters
 *   (k / 4, 0, 0, c3) and (k / 4, 1, 0, c3) each give one FP64 Box-Muller pair
 *   from 52-bit words  ub = x0 << 20 | x1 >> 12,  gb = x2 << 20 | x3 >> 12:
 *     u  = (ub + 0.5) * 2^-52,         g = (gb + 0.5) * 2^-51 - 1
 *     n0 = sqrt(-2 ln u) cos(pi g),    n1 = sqrt(-2 ln u) sin(pi g)
 *   (control variates and importance sampling use the same quads, c3 = 1).
 * One-factor stepwise models: six normals per call as for Heston below;
 *   step j of unit u is block j / 6, normal j % 6.
 * Heston: one call gives six normals, three Box-Muller pairs with 23-bit
 *   radii from x0 >> 9, x1 >> 9, x2 >> 9 and angles of 16, 16 and 18 bits
 *   from x3 & 0xFFFF, x3 >> 16 and (x0 & 0x1FF) | (x1 & 0x1FF) << 9;
 *   step j of unit u is block j / 3, (z1, z2) = pair j % 3.
 * ===================================================================== */
void qko_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = (uint64_t)UINT32_C(0xD2511F53) * c0;
        const uint64_t p1 = (uint64_t)UINT32_C(0xCD9E8D57) * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += UINT32_C(0x9E3779B9);
        k1 += UINT32_C(0xBB67AE85);
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* FP64 Box-Muller pair from one call's four words (52-bit radius and angle
 * words; both conversions below are exact). */
static void box_muller_f64(const uint32_t x[4], double* za, double* zb) {
    const uint64_t ub = ((uint64_t)x[0] << 20) | (x[1] >> 12);
    const uint64_t gb = ((uint64_t)x[2] << 20) | (x[3] >> 12);
    const double u = ((double)ub + 0.5) * 0x1p-52;
    const double g = ((double)gb + 0.5) * 0x1p-51 - 1.0;
    const double rad = sqrt(-2.0 * log(u));
    *za = rad * cos(M_PI * g);
    *zb = rad * sin(M_PI * g);
}

/* Box-Muller from a 23-bit radius word and an n-bit angle word. */
static void box_muller_bits(uint32_t ub, uint32_t gb, int n, double* za, double* zb) {
    const double u = ((double)ub + 0.5) * 0x1p-23;
    const double g = ((double)gb + 0.5) * ldexp(1.0, -(n - 1)) - 1.0;
    const double rad = sqrt(-2.0 * log(u));
    *za = rad * cos(M_PI * g);
    *zb = rad * sin(M_PI * g);
}

void qko_philox_normals6(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c3, double z[6]) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const uint32_t ctr[4] = {c0, c1, 0u, c3};
    uint32_t x[4];
    qko_philox4x32_10(ctr, key, x);
    box_muller_bits(x[0] >> 9, x[3] & 0xFFFFu, 16, &z[0], &z[1]);
    box_muller_bits(x[1] >> 9, x[3] >> 16, 16, &z[2], &z[3]);
    box_muller_bits(x[2] >> 9, (x[0] & 0x1FFu) | ((x[1] & 0x1FFu) << 9), 18, &z[4], &z[5]);
}

void qko_philox_normals4(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c3, double z[4]) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const uint32_t ctr0[4] = {c0, c1, 0u, c3};
    const uint32_t ctr1[4] = {c0, c1 + 1u, 0u, c3};
    uint32_t x[4];
    qko_philox4x32_10(ctr0, key, x);
    box_muller_f64(x, &z[0], &z[1]);
    qko_philox4x32_10(ctr1, key, x);
    box_muller_f64(x, &z[2], &z[3]);
}

/* One simulated path of unit u under sign sg (+1 / -1) for the stepwise
 * models, FP64 with the reference step functions. */
static double replay_path(int32_t model, double spot, double t, double vol, double r, double q,
                          double v0, double kappa, double theta, double sigma, double rho,
                          int32_t steps, uint64_t seed, uint32_t unit, uint32_t c3, double sg) {
    double z4[4];
    if (model == 0 || model == 1 || model == 5) {
        qko_philox_normals4(seed, unit / 4u, 0u, c3, z4);
        return bsm_terminal(vol, r, q, spot, t, sg * z4[unit % 4u]);
    }
    const double dt = t / (double)steps;
    const double sqrt_dt = sqrt(dt);
    if (model == 6 || model == 7) {
        const double rho_comp = sqrt(smax(1.0 - rho * rho, 0.0));
        double s = spot, v = v0, z6[6];
        for (int32_t j = 0; j < steps; ++j) {
            if (j % 3 == 0) qko_philox_normals6(seed, unit, (uint32_t)(j / 3), c3, z6);
            const double z1 = sg * z6[2 * (j % 3)];
            const double z2 = sg * z6[2 * (j % 3) + 1];
            const double v_pos = smax(v, 0.0);
            const double sqrt_v = sqrt(v_pos);
            const double dw1 = sqrt_dt * z1;
            const double dw2 = sqrt_dt * (rho * z1 + rho_comp * z2);
            const double s_next = s * exp((r - q - 0.5 * v_pos) * dt + sqrt_v * dw1);
            v = smax(0.0, v + kappa * (theta - v_pos) * dt + sigma * sqrt_v * dw2);
            s = smax(s_next, 1e-12);
        }
        return s;
    }
    double s = spot, z6[6];
    const double drift = r - q;
    for (int32_t j = 0; j < steps; ++j) {
        if (j % 6 == 0) qko_philox_normals6(seed, unit, (uint32_t)(j / 6), c3, z6);
        const double dw = sqrt_dt * (sg * z6[j % 6]);
        if (model == 3)
            s = smax(1e-12, s + drift * s * dt + vol * s * dw + 0.5 * vol * vol * s * (dw * dw - dt));
        else
            s = smax(1e-12, s + drift * s * dt + vol * s * dw);
    }
    return s;
}

double qko_philox_price(int32_t model, double spot, double strike, double t, double vol,
                        double r, double q, double v0, double kappa, double theta, double sigma,
                        double rho, int32_t ot, int32_t paths, int32_t steps, uint64_t seed,
                        int32_t antithetic, double* se) {
    if (se) *se = qko_nan();
    /* entry checks and special cases of the matching reference pricer */
    if (model == 7) {
        const double clip = vol;
        if (!valid_option_type(ot) || spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0 ||
            kappa < 0.0 || theta < 0.0 || sigma < 0.0 || rho < -1.0 || rho > 1.0 ||
            !valid_mc_counts(paths, steps) || !(clip > 0.0))
            return qko_nan();
        if (t <= QKO_EPS) {
            if (ot == QKO_CALL) return (spot > strike) ? 1.0 : 0.0;
            return (spot < strike) ? -1.0 : 0.0;
        }
        const double disc = exp(-r * t);
        const double sqrt_dt = sqrt(t / (double)steps);
        const double sqrt_v0 = sqrt(smax(v0, 0.0));
        double sum = 0.0, ysum = 0.0, ysq = 0.0, ny = 0.0;
        const int32_t units = antithetic ? paths - paths / 2 : paths;
        const int32_t n_pairs = paths / 2;
        for (int32_t u = 0; u < units; ++u) {
            double z6[6];
            qko_philox_normals6(seed, (uint32_t)u, 0u, antithetic ? 0u : 1u, z6);
            double w = (sqrt_v0 > 1e-15) ? z6[0] / (sqrt_v0 * sqrt_dt * spot) : 0.0;
            w = smax(-clip, smin(clip, w));
            const double a = intrinsic(replay_path(6, spot, t, vol, r, q, v0, kappa, theta, sigma,
                                                   rho, steps, seed, (uint32_t)u,
                                                   antithetic ? 0u : 1u, 1.0), strike, ot) * w;
            if (antithetic && u < n_pairs) {
                const double b = intrinsic(replay_path(6, spot, t, vol, r, q, v0, kappa, theta,
                                                       sigma, rho, steps, seed, (uint32_t)u, 0u,
                                                       -1.0), strike, ot) * (-w);
                sum += a + b;
                const double m = 0.5 * (a + b);
                ysum += m;
                ysq += m * m;
                ny += 1.0;
            } else if (antithetic) {
                sum += a;
            } else {
                sum += a;
                ysum += a;
                ysq += a * a;
                ny += 1.0;
            }
        }
        if (se) *se = se_from_moments(disc, ysum, ysq, ny);
        return disc * (sum / (double)paths);
    }
    if (model == 6) {
        if (!valid_option_type(ot) || spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0 ||
            kappa < 0.0 || theta < 0.0 || sigma < 0.0 || rho < -1.0 || rho > 1.0 ||
            !valid_mc_counts(paths, steps))
            return qko_nan();
    } else {
        int counts_ok = (model == 0 || model == 1 || model == 5) ? paths > 1
                                                                : valid_mc_counts(paths, steps);
        if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || !counts_ok) return qko_nan();
    }
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    if (model == 0 && vol <= QKO_EPS) {
        const double fwd = spot * exp((r - q) * t);
        return exp(-r * t) * intrinsic(fwd, strike, ot);
    }
    const double disc = exp(-r * t);
    double sum = 0.0, ysum = 0.0, ysq = 0.0, ny = 0.0;
    if (antithetic) {
        const int32_t n_pairs = paths / 2;
        for (int32_t p = 0; p < n_pairs; ++p) {
            double a = intrinsic(replay_path(model, spot, t, vol, r, q, v0, kappa, theta, sigma,
                                             rho, steps, seed, (uint32_t)p, 0u, 1.0),
                                 strike, ot);
            double b = intrinsic(replay_path(model, spot, t, vol, r, q, v0, kappa, theta, sigma,
                                             rho, steps, seed, (uint32_t)p, 0u, -1.0),
                                 strike, ot);
            sum += a + b;
            const double m = 0.5 * (a + b);
            ysum += m;
            ysq += m * m;
            ny += 1.0;
        }
        if (paths & 1) {
            sum += intrinsic(replay_path(model, spot, t, vol, r, q, v0, kappa, theta, sigma, rho,
                                         steps, seed, (uint32_t)n_pairs, 0u, 1.0),
                             strike, ot);
        }
    } else {
        for (int32_t p = 0; p < paths; ++p) {
            double a = intrinsic(replay_path(model, spot, t, vol, r, q, v0, kappa, theta, sigma,
                                             rho, steps, seed, (uint32_t)p, 1u, 1.0),
                                 strike, ot);
            sum += a;
            ysum += a;
            ysq += a * a;
            ny += 1.0;
        }
    }
    if (se) *se = se_from_moments(disc, ysum, ysq, ny);
    return disc * (sum / (double)paths);
}

/* Philox replay of the variance-reduction models (8-12), FP64, the GPU's
 * stream and estimators:
 *   8 control variates, 9 importance sampling: path i uses normal slot i % 4
 *     of counter (i / 4, 0, 0, 1);
 *   10 stratified: U_i = (x + 0.5) 2^-32 from word i % 4 of counter
 *     (i / 4, 0, 0, 2);  11 / 12: the reference's points (no randomness). */
double qko_philox_vr_price(int32_t model, double spot, double strike, double t, double vol,
                           double r, double q, double shift, int32_t ot, int32_t paths,
                           uint64_t seed, double* se) {
    if (se) *se = qko_nan();
    const int32_t min_paths = model == 8 ? 3 : 2;
    if (!valid_common_inputs(spot, strike, t, vol, r, q, ot) || paths < min_paths ||
        !qko_finite(shift))
        return qko_nan();
    if (t <= QKO_EPS) return intrinsic(spot, strike, ot);
    const double disc = exp(-r * t);
    const double d0 = (r - q - 0.5 * vol * vol) * t;
    const double d1 = vol * sqrt(smax(t, 0.0));
    const double mean_st = spot * exp((r - q) * t);
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    double sp = 0.0, spp = 0.0, sc = 0.0, scc = 0.0, scp = 0.0, dsq = 0.0, prev = 0.0;
    for (int32_t i = 0; i < paths; ++i) {
        double z;
        if (model == 11 || model == 12) {
            const double u = model == 11 ? sobol_point((uint32_t)i + 1u)
                                         : halton_point((uint32_t)i + 1u, 2u);
            z = acklam_inv(clamp_unit(u));
        } else if (model == 10) {
            const uint32_t ctr[4] = {(uint32_t)i / 4u, 0u, 0u, 2u};
            uint32_t x[4];
            qko_philox4x32_10(ctr, key, x);
            const double ui = ((double)x[i % 4] + 0.5) * 0x1p-32;
            z = acklam_inv(clamp_unit(((double)i + ui) / (double)paths));
        } else {
            double z4[4];
            qko_philox_normals4(seed, (uint32_t)i / 4u, 0u, 1u, z4);
            z = z4[i % 4];
        }
        double w = 1.0;
        if (model == 9) {
            z = z + shift;
            w = exp(-shift * z + 0.5 * shift * shift);
        }
        const double st = spot * exp(d0 + d1 * z);
        const double a = intrinsic(st, strike, ot) * w;
        sp += a;
        spp += a * a;
        if (model == 8) {
            const double c = st - mean_st;
            sc += c;
            scc += c * c;
            scp += c * a;
        }
        if (model == 10 && (i & 1)) dsq += (prev - a) * (prev - a);
        prev = a;
    }
    const double n = (double)paths;
    if (model == 8) {
        const double mp = sp / n, mc = sc / n, vc = scc / n - mc * mc;
        if (se) *se = cv_se(disc, sp, spp, sc, scc, scp, n);
        if (disc * disc * vc <= QKO_EPS) return disc * mp;
        const double beta = (scp / n - mc * mp) / vc;
        return disc * (mp - beta * mc);
    }
    if (model == 10) {
        if (se) *se = disc * sqrt(dsq) / n;
    } else if (se) {
        *se = se_from_moments(disc, sp, spp, n);
    }
    return disc * (sp / n);
}
