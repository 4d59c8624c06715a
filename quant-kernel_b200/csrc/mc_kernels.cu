// mc_kernels.cu -- hand-written sm_100a Monte Carlo kernels.
//
// Work decomposition.  A batch is a list of options; option i is split into
// `tiles` tiles of BLOCK * UPT * unit_iters simulation units (a unit is an
// antithetic pair or a plain path for the stepwise models, and a quad of four
// normals for the terminal models).  A CTA simulates one tile at a time: each
// thread carries UPT units in registers through all time steps, drawing its
// normals from Philox4x32-10 keyed by the option's seed and countered by
// (unit, step block) -- so a path's normals depend only on (seed, path index),
// never on the batch, the launch shape or the scheduling.  Per-thread FP64
// double-double sums of y and y^2 (y = pair mean or payoff) are reduced
// warp -> CTA in a fixed order and written to the tile's slot; the finalize
// kernel merges an option's slots in tile order.  Results are therefore
// deterministic and a batch reproduces the scalar call bit for bit.
//
// Reference loops restated (yluoc/Quant-Kernel):
//   terminal   mc_engine.h:32-75   + model_concepts.h:93-102
//   stepwise   mc_engine.h:84-103  + model_concepts.h:136-158, 240-266
//   Heston     mc_engine.h:113-136 + model_concepts.h:205-226
//   variance reduction (terminal GBM, FP64 path arithmetic)
//              control_variates.cpp:10-52, importance_sampling.cpp:11-36,
//              stratified_sampling.cpp:11-35, quasi_monte_carlo.cpp:10-56
// Heston keeps log(S/spot) instead of S: the reference's s * exp(a) step with
// the std::max(s, 1e-12) floor is the same map as x + a floored at
// log(1e-12/spot), and it removes the per-step exp; sqrt(v) times the
// Box-Muller radius is taken as one square root.
#include "mc_device.cuh"
#include "mc_launch.h"

#include <cstdio>

namespace qkb {

namespace {

// ----------------------------------------------------------------------------
// Per-thread accumulation of one tile.
// ----------------------------------------------------------------------------
struct Acc {
    DD sy{0.0, 0.0};
    DD q{0.0, 0.0};
    double lone = 0.0;
    double cx = 0.0, cxx = 0.0, cxy = 0.0;  // control variates only
    __device__ __forceinline__ void add_pair(double a, double b) {
        const double y = __dmul_rn(0.5, __dadd_rn(a, b));
        sy = dd_add(sy, y);
        q = dd_add(q, __dmul_rn(y, y));
    }
    __device__ __forceinline__ void add_lone(double a) { lone = __dadd_rn(lone, a); }
    __device__ __forceinline__ void add_plain(double a) {
        sy = dd_add(sy, a);
        q = dd_add(q, __dmul_rn(a, a));
    }
};

// ----------------------------------------------------------------------------
// Inverse normal CDF: P. J. Acklam's rational approximation (2003; relative
// error < 1.15e-9), the one the reference evaluates
// (monte_carlo_methods/common/internal_util.h:42-90).  Coefficients and the
// Horner order are the published ones so that quasi-Monte Carlo prices, which
// have no randomness, agree with the reference to rounding.
// ----------------------------------------------------------------------------
__device__ __forceinline__ double acklam_inv(double p) {
    if (p <= 0.0 || p >= 1.0) return __longlong_as_double(0x7FF8000000000000ll);
    constexpr double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                             1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    constexpr double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                             6.680131188771972e+01, -1.328068155288572e+01};
    constexpr double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                             -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    constexpr double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                             3.754408661907416e+00};
    constexpr double p_low = 0.02425;
    const bool lo = p < p_low, hi = p > 1.0 - p_low;
    if (lo || hi) {
        const double t = sqrt(-2.0 * log(lo ? p : 1.0 - p));
        double num = c[0];
#pragma unroll
        for (int i = 1; i < 6; ++i) num = num * t + c[i];
        double den = d[0];
#pragma unroll
        for (int i = 1; i < 4; ++i) den = den * t + d[i];
        den = den * t + 1.0;
        return (lo ? num : -num) / den;
    }
    const double t = p - 0.5;
    const double r = t * t;
    double num = a[0];
#pragma unroll
    for (int i = 1; i < 6; ++i) num = num * r + a[i];
    double den = b[0];
#pragma unroll
    for (int i = 1; i < 5; ++i) den = den * r + b[i];
    den = den * r + 1.0;
    return num * t / den;
}

// std::clamp(u, 1e-12, 1 - 1e-12) (a NaN stays NaN).
__device__ __forceinline__ double clamp_unit(double u) {
    return u < 1e-12 ? 1e-12 : ((1.0 - 1e-12) < u ? 1.0 - 1e-12 : u);
}

// ----------------------------------------------------------------------------
// Terminal GBM (models 0, 1, 5), FP64 throughout like the reference's
// make_bsm_terminal: S_T = spot exp(d0 + d1 z) with d0 = (r - q - vol^2/2) t
// and d1 = vol sqrt(t) from the host, in that expression order (the down
// path's d1 (-z) is -(d1 z) exactly, as in the reference).  Unit = quad of four
// FP64 normals (two Philox calls).  Normal k serves pair k (antithetic) or
// path k (plain); with an odd antithetic path count, normal n_pairs drives the
// lone last path.
// ----------------------------------------------------------------------------
template <int UPT, bool ANTI>
__device__ __forceinline__ void sim_terminal(const McOption& o, uint32_t unit0, uint32_t stride,
                                             uint32_t k0, uint32_t k1, Acc& acc) {
    const double d0 = o.d[0], d1 = o.d[1];
    const uint32_t n_pairs = (uint32_t)o.paths >> 1;
    const uint32_t n_norm = ANTI ? (uint32_t)(o.paths - (int32_t)n_pairs) : (uint32_t)o.paths;
    const bool odd = (o.paths & 1) != 0;
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
        const uint32_t unit = unit0 + (uint32_t)k * stride;
        if (unit * 4u >= n_norm) continue;
        double z[4];
        normals4_f64(unit, ANTI ? 0u : 1u, k0, k1, z);
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t idx = unit * 4u + (uint32_t)s;
            if (idx >= n_norm) break;
            const double dz = __dmul_rn(d1, z[s]);
            const double su = o.spot * exp(__dadd_rn(d0, dz));
            const double a = payoff(su, o.strike, o.option_type);
            if (ANTI) {
                if (idx < n_pairs) {
                    const double sd = o.spot * exp(__dadd_rn(d0, -dz));
                    acc.add_pair(a, payoff(sd, o.strike, o.option_type));
                } else if (odd) {
                    acc.add_lone(a);
                }
            } else {
                acc.add_plain(a);
            }
        }
    }
}

// ----------------------------------------------------------------------------
// One-factor stepwise BSM (Euler / local vol: MIL = false; Milstein: true).
// State is s = S/spot in FP32 and the step is the reference's additive form
//   s' = max(s + s * inc, 1e-12/spot),  inc = (r-q)dt + vol sqrt(dt) z
//   [Milstein: + c (z^2 - 1), c = vol^2 dt / 2]
// evaluated as one fused s + s * inc.  One Philox call feeds six steps
// (Philox6: three Box-Muller pairs).  SU step blocks run per loop iteration
// (their Philox calls first): the same normals and arithmetic for every SU,
// more independent work per iteration for larger SU (the autotuner's step
// unrolling).
// ----------------------------------------------------------------------------
template <int UPT, bool ANTI, bool MIL, int SU>
__device__ __forceinline__ void sim_stepwise(const McOption& o, uint32_t unit0, uint32_t stride,
                                             uint32_t k0, uint32_t k1, Acc& acc) {
    // Philox6 normals are z / kBmRadius: the vol and Milstein constants take
    // the factor (b z = (b kBmRadius)(z / kBmRadius), likewise c z^2)
    const float m0 = o.p[0], b = o.p[1] * kBmRadius, fl = o.p[2], c = o.p[3] * kBmRadius2;
    const int32_t steps = o.steps;
    const uint32_t units = (uint32_t)o.units;
    const uint32_t c3 = ANTI ? 0u : 1u;
    float su[UPT], sd[UPT];
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
        su[k] = 1.0f;
        sd[k] = 1.0f;
    }
    // PK: units 2p and 2p + 1 of the thread form one packed pair (lane 0, lane
    // 1) for every multiply and FMA of the step; the floors stay per lane.
    // Same operations in the same order as the scalar step, so the same bits.
    constexpr bool PK = (UPT % 2) == 0;
    constexpr int NP = PK ? UPT / 2 : 1;
    float2 su2[NP], sd2[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        su2[p] = f2(1.0f);
        sd2[p] = f2(1.0f);
    }
    const float2 m02 = f2(m0), b2 = f2(b), c2 = f2(c);
    // One step s of a step block (the block's Box-Muller pair s / 2 is drawn
    // at even s), packed (units 2p, 2p + 1 as one pair) or scalar.
    float2 zp2[NP][2];
    float zp[UPT][2];
    auto step = [&](const Philox6 (&r)[UPT], int s) {
        if constexpr (PK) {
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                if ((s & 1) == 0) philox6_pair2(r[2 * p], r[2 * p + 1], s >> 1, zp2[p][0], zp2[p][1]);
                const float2 zz = zp2[p][s & 1];
                float2 iu, id;
                if (MIL) {
                    iu = fma2(fma2(c2, zz, b2), zz, m02);
                    id = fma2(fma2(neg2(c2), zz, b2), neg2(zz), m02);
                } else {
                    iu = fma2(b2, zz, m02);
                    id = fma2(neg2(b2), zz, m02);
                }
                const float2 u = fma2(su2[p], iu, su2[p]);
                su2[p] = f2(fmaxf(u.x, fl), fmaxf(u.y, fl));
                if (ANTI) {
                    const float2 d = fma2(sd2[p], id, sd2[p]);
                    sd2[p] = f2(fmaxf(d.x, fl), fmaxf(d.y, fl));
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < UPT; ++k) {
                if ((s & 1) == 0) r[k].pair(s >> 1, zp[k][0], zp[k][1]);
                const float zz = zp[k][s & 1];
                float iu, id;
                if (MIL) {
                    iu = fma_rn(fma_rn(c, zz, b), zz, m0);
                    id = fma_rn(fma_rn(-c, zz, b), -zz, m0);
                } else {
                    iu = fma_rn(b, zz, m0);
                    id = fma_rn(-b, zz, m0);
                }
                su[k] = fmaxf(fma_rn(su[k], iu, su[k]), fl);
                if (ANTI) sd[k] = fmaxf(fma_rn(sd[k], id, sd[k]), fl);
            }
        }
    };
    auto philox_block = [&](Philox6 (&r)[UPT], uint32_t bk) {
#pragma unroll
        for (int k = 0; k < UPT; ++k)
            r[k].x = philox4x32_10(unit0 + (uint32_t)k * stride, bk, 0u, c3, k0, k1);
    };
    // steps <= kMaxSteps (checked when packing), so j0 + 12 never wraps
    uint32_t blk = 0;  // step block j / 6
    if constexpr (SU == 1) {
        // whole blocks of six steps with no branch between the steps and the
        // next block's Philox call after the first step, then the steps
        // left (as in the Heston kernel)
        const int32_t full = steps - steps % 6;
        int32_t j0 = 0;
        Philox6 r[UPT];
        philox_block(r, 0u);
#pragma unroll 2
        for (; j0 < full; j0 += 6, ++blk) {
            Philox6 nx[UPT];
            step(r, 0);
            philox_block(nx, blk + 1u);
#pragma unroll
            for (int s = 1; s < 6; ++s) step(r, s);
#pragma unroll
            for (int k = 0; k < UPT; ++k) r[k] = nx[k];
        }
        if (j0 < steps) {
            const int32_t m = steps - j0;
#pragma unroll
            for (int s = 0; s < 5; ++s)
                if (s < m) step(r, s);
        }
    } else {
        for (int32_t j0 = 0; j0 < steps; j0 += 6 * SU, blk += SU) {
            Philox6 rb[SU][UPT];
#pragma unroll
            for (int sb = 0; sb < SU; ++sb) philox_block(rb[sb], blk + (uint32_t)sb);
#pragma unroll
            for (int sb = 0; sb < SU; ++sb) {
                const int32_t j = j0 + 6 * sb;
                const int32_t m = (steps - j) < 6 ? (steps - j) : 6;
#pragma unroll
                for (int s = 0; s < 6; ++s)
                    if (s < m) step(rb[sb], s);
            }
        }
    }
    if constexpr (PK) {
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            su[2 * p] = su2[p].x;
            su[2 * p + 1] = su2[p].y;
            sd[2 * p] = sd2[p].x;
            sd[2 * p + 1] = sd2[p].y;
        }
    }
    const uint32_t n_pairs = (uint32_t)o.paths >> 1;
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
        const uint32_t unit = unit0 + (uint32_t)k * stride;
        if (unit >= units) continue;
        const double pu = payoff(o.spot * (double)su[k], o.strike, o.option_type);
        if (ANTI) {
            if (unit < n_pairs)
                acc.add_pair(pu, payoff(o.spot * (double)sd[k], o.strike, o.option_type));
            else
                acc.add_lone(pu);
        } else {
            acc.add_plain(pu);
        }
    }
}

// ----------------------------------------------------------------------------
// Heston full-truncation Euler.  State (x, v) with x = log(S/spot), or y =
// x - j (r-q)dt after j steps where the drift is small (DF below):
//   x' = max_nan(x + (r-q)dt - v dt/2 + sqrt(v) sqrt(dt) z1, log(1e-12/spot))
//   v' = max(v (1 - kappa dt) + kappa theta dt
//            + sigma sqrt(dt) sqrt(v) (rho z1 + sqrt(1-rho^2) z2), 0)
// v >= 0 after every step (and v0 >= 0 is validated), so the reference's
// v_pos = max(v, 0) is v itself.  One Philox call feeds three steps of a unit
// (six normals: Philox6); SU step blocks per loop iteration as in
// sim_stepwise.  With Box-Muller z1 = r cos a, z2 = r sin a, r = sqrt(-2 ln u),
// the step needs sqrt(v) r = sqrt(v r^2) only: one square root per path and
// step instead of one per path and step plus one per pair.
// ----------------------------------------------------------------------------
//
// LR = true: the likelihood-ratio delta of heston_lr_delta.cpp:37-132.  Each
// path's payoff is weighted by the score of its first spot step,
// w = clamp(z1_0 / (sqrt(v0) sqrt(dt) S0), -clip, clip); the antithetic path's
// score is -w.
//
// DF (drift in floor) selects the state: y = x - j (r-q)dt (one add fewer per
// path and step) or x itself.  y is used while |(r-q)dt| steps <= 1: then y
// stays as small as x, so FP32 rounds it no worse, and the floor
// log(1e-12/spot) - j (r-q)dt stays exact to FP32 rounding.  Larger or
// non-finite drifts, which the reference accepts for Heston (no finiteness
// check on r and q), keep x, whose floor is exact at any drift.
template <int UPT, bool ANTI, bool LR, int SU, bool DF>
__device__ __forceinline__ void sim_heston_form(const McOption& o, uint32_t unit0, uint32_t stride,
                                                uint32_t k0, uint32_t k1, Acc& acc) {
    // the normals enter as kBmRadius sqrt(w) (c, s) (Philox6::parts): the two
    // constants that multiply them take the factor kBmRadius
    const float cmu = o.p[0], hdt = o.p[1], sqdt = o.p[2] * kBmRadius, kdt = o.p[3], kth = o.p[4];
    const float xsq = o.p[5] * kBmRadius, rho = o.p[6], rhoc = o.p[7], v0 = o.p[8], xfl = o.p[9];
    const float omk = 1.0f - kdt;
    const float xr = xsq * rho, xc = xsq * rhoc;
    const int32_t steps = o.steps;
    const uint32_t units = (uint32_t)o.units;
    const uint32_t c3 = ANTI ? 0u : 1u;
    // DF: xu, xd hold y = x - j (r-q)dt after j steps: the drift leaves the
    // per-step update and enters the floor instead, y_j >= log(1e-12/spot) -
    // j (r-q)dt, the same map as x_j >= log(1e-12/spot)
    float xu[UPT], vu[UPT], xd[UPT], vd[UPT];
    float fl = xfl;
    float zfirst[UPT];
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
        xu[k] = 0.0f;
        xd[k] = 0.0f;
        vu[k] = v0;
        vd[k] = v0;
        zfirst[k] = 0.0f;
    }
    // PK: units 2p and 2p + 1 of the thread form one packed pair (lane 0, lane
    // 1) for every multiply and FMA of the step; the square roots and the
    // floors stay per lane.  Same operations in the same order as the scalar
    // step, so the same bits.
    constexpr bool PK = (UPT % 2) == 0;
    constexpr int NP = PK ? UPT / 2 : 1;
    float2 xu2[NP], vu2[NP], xd2[NP], vd2[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        xu2[p] = f2(0.0f);
        xd2[p] = f2(0.0f);
        vu2[p] = f2(v0);
        vd2[p] = f2(v0);
    }
    const float2 sqdt2 = f2(sqdt), xr2 = f2(xr), xc2 = f2(xc), nhdt2 = f2(-hdt), omk2 = f2(omk),
                 kth2 = f2(kth), cmu2 = f2(cmu);
    // One step s of a step block: packed (units 2p, 2p + 1 as one pair) or
    // scalar; `first` marks step 0 of the path (the LR score's normal).
    auto step = [&](const Philox6 (&r)[UPT], int s, bool first) {
        if (DF) fl -= cmu;  // the floor of y after this step
        if constexpr (PK) {
            const float flo = DF ? fl : xfl;
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                float2 w, c1, s1;
                philox6_parts2(r[2 * p], r[2 * p + 1], s, w, c1, s1);
                if (LR && first) {
                    zfirst[2 * p] = ptx_sqrt(w.x) * c1.x;
                    zfirst[2 * p + 1] = ptx_sqrt(w.y) * c1.y;
                }
                const float2 sz1 = mul2(sqdt2, c1);
                const float2 xw = fma2(xr2, c1, mul2(xc2, s1));
                {
                    const float2 q = mul2(vu2[p], w);
                    const float2 sv = f2(ptx_sqrt(q.x), ptx_sqrt(q.y));
                    const float2 x = DF ? fma2(sv, sz1, fma2(nhdt2, vu2[p], xu2[p]))
                                        : add2(xu2[p], fma2(sv, sz1, fma2(nhdt2, vu2[p], cmu2)));
                    xu2[p] = f2(ptx_max_nan(x.x, flo), ptx_max_nan(x.y, flo));
                    const float2 v = fma2(sv, xw, fma2(vu2[p], omk2, kth2));
                    vu2[p] = f2(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f));
                }
                if (ANTI) {
                    const float2 q = mul2(vd2[p], w);
                    const float2 sv = f2(ptx_sqrt(q.x), ptx_sqrt(q.y));
                    const float2 x = DF ? fma2(sv, neg2(sz1), fma2(nhdt2, vd2[p], xd2[p]))
                                        : add2(xd2[p], fma2(sv, neg2(sz1), fma2(nhdt2, vd2[p], cmu2)));
                    xd2[p] = f2(ptx_max_nan(x.x, flo), ptx_max_nan(x.y, flo));
                    const float2 v = fma2(sv, neg2(xw), fma2(vd2[p], omk2, kth2));
                    vd2[p] = f2(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f));
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < UPT; ++k) {
                // z1 = kBmRadius sqrt(w) c, z2 = kBmRadius sqrt(w) s; the
                // step needs sqrt(v) z1 and sqrt(v) z2 only, so sqrt(w)
                // joins the variance's square root: sqrt(v w)
                float w, c1, s1;
                r[k].parts(s, w, c1, s1);
                if (LR && first) zfirst[k] = ptx_sqrt(w) * c1;
                const float sz1 = sqdt * c1;
                const float xw = fma_rn(xr, c1, xc * s1);
                {
                    const float sv = ptx_sqrt(vu[k] * w);
                    if (DF)
                        xu[k] = ptx_max_nan(fma_rn(sv, sz1, fma_rn(-hdt, vu[k], xu[k])), fl);
                    else
                        xu[k] = ptx_max_nan(xu[k] + fma_rn(sv, sz1, fma_rn(-hdt, vu[k], cmu)), xfl);
                    vu[k] = fmaxf(fma_rn(sv, xw, fma_rn(vu[k], omk, kth)), 0.0f);
                }
                if (ANTI) {
                    const float sv = ptx_sqrt(vd[k] * w);
                    if (DF)
                        xd[k] = ptx_max_nan(fma_rn(sv, -sz1, fma_rn(-hdt, vd[k], xd[k])), fl);
                    else
                        xd[k] = ptx_max_nan(xd[k] + fma_rn(sv, -sz1, fma_rn(-hdt, vd[k], cmu)), xfl);
                    vd[k] = fmaxf(fma_rn(sv, -xw, fma_rn(vd[k], omk, kth)), 0.0f);
                }
            }
        }
    };
    auto philox_block = [&](Philox6 (&r)[UPT], uint32_t b) {
#pragma unroll
        for (int k = 0; k < UPT; ++k)
            r[k].x = philox4x32_10(unit0 + (uint32_t)k * stride, b, 0u, c3, k0, k1);
    };
    // steps <= kMaxSteps (checked when packing), so j0 + 6 never wraps
    uint32_t blk = 0;  // step block j / 3
    if constexpr (SU == 1) {
        // whole blocks of three steps with no branch between the steps (so
        // one step's special-function work can be scheduled among the next
        // step's arithmetic), then the one or two steps left.  The next
        // block's Philox calls are issued inside the block -- the first half
        // of the units' after the block's first step, the rest after its
        // second -- so their integer work interleaves with the steps'
        // special-function work (the same words: the same bits); the loop is
        // unrolled twice so that the two sets of words swap without copies.
        const int32_t full = steps - steps % 3;
        int32_t j0 = 0;
        Philox6 r[UPT];
        philox_block(r, 0u);
#pragma unroll 2
        for (; j0 < full; j0 += 3, ++blk) {
            Philox6 nx[UPT];
            step(r, 0, j0 == 0);
#pragma unroll
            for (int k = 0; k < UPT / 2; ++k)
                nx[k].x = philox4x32_10(unit0 + (uint32_t)k * stride, blk + 1u, 0u, c3, k0, k1);
            step(r, 1, false);
#pragma unroll
            for (int k = UPT / 2; k < UPT; ++k)
                nx[k].x = philox4x32_10(unit0 + (uint32_t)k * stride, blk + 1u, 0u, c3, k0, k1);
            step(r, 2, false);
#pragma unroll
            for (int k = 0; k < UPT; ++k) r[k] = nx[k];
        }
        if (j0 < steps) {
            step(r, 0, j0 == 0);
            if (j0 + 1 < steps) step(r, 1, false);
        }
    } else {
        for (int32_t j0 = 0; j0 < steps; j0 += 3 * SU, blk += SU) {
            Philox6 rb[SU][UPT];
#pragma unroll
            for (int sb = 0; sb < SU; ++sb) philox_block(rb[sb], blk + (uint32_t)sb);
#pragma unroll
            for (int sb = 0; sb < SU; ++sb) {
                const int32_t j = j0 + 3 * sb;
                const int32_t m = (steps - j) < 3 ? (steps - j) : 3;
#pragma unroll
                for (int s = 0; s < 3; ++s)
                    if (s < m) step(rb[sb], s, j == 0 && s == 0);
            }
        }
    }
    if constexpr (PK) {
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            xu[2 * p] = xu2[p].x;
            xu[2 * p + 1] = xu2[p].y;
            xd[2 * p] = xd2[p].x;
            xd[2 * p + 1] = xd2[p].y;
        }
    }
    const uint32_t n_pairs = (uint32_t)o.paths >> 1;
    const double drift = DF ? (double)steps * (double)cmu : 0.0;  // x = y + steps (r-q)dt
    // score scale 1 / (sqrt(v0) sqrt(dt) S0) for z1 = kBmRadius zfirst; v0 = 0
    // is a constant-zero option
    const double wscale = LR ? kBmRadiusD / ((double)ptx_sqrt(v0) * (double)o.p[2] * o.spot) : 0.0;
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
        const uint32_t unit = unit0 + (uint32_t)k * stride;
        if (unit >= units) continue;
        double w = 1.0;
        if (LR) w = fmin(o.weight_clip, fmax(-o.weight_clip, (double)zfirst[k] * wscale));
        const double pu = payoff(o.spot * exp((double)xu[k] + drift), o.strike, o.option_type) * w;
        if (ANTI) {
            if (unit < n_pairs)
                acc.add_pair(pu, payoff(o.spot * exp((double)xd[k] + drift), o.strike, o.option_type) * (LR ? -w : 1.0));
            else
                acc.add_lone(pu);
        } else {
            acc.add_plain(pu);
        }
    }
}

template <int UPT, bool ANTI, bool LR, int SU>
__device__ __forceinline__ void sim_heston(const McOption& o, uint32_t unit0, uint32_t stride,
                                           uint32_t k0, uint32_t k1, Acc& acc) {
    // uniform per option (and so per CTA); a NaN drift takes the x state
    if (fabsf(o.p[0]) * (float)o.steps <= 1.0f)
        sim_heston_form<UPT, ANTI, LR, SU, true>(o, unit0, stride, k0, k1, acc);
    else
        sim_heston_form<UPT, ANTI, LR, SU, false>(o, unit0, stride, k0, k1, acc);
}

// ----------------------------------------------------------------------------
// Terminal GBM with a variance-reduction estimator (models 8-12).  Unit = quad
// of four consecutive paths 4u .. 4u+3; the path arithmetic is FP64 like the
// reference's: S_T = spot exp(d0 + d1 z).
//   control variates   z from the plain FP64 normal stream of the terminal
//                      models (normals4_f64, c3 = 1); sums of the payoff and
//                      of the centred control c = S_T - E[S_T]
//   importance         z from the same FP64 normal stream, y = z + shift,
//                      payoff(S_T(y)) exp(-shift y + shift^2 / 2)
//   stratified         u = (i + U_i) / n with U_i uniform (Philox stream
//                      c3 = 2), z = Acklam(u); q collects (y_2k - y_2k+1)^2 of
//                      neighbouring strata, which are in the same quad
//   Sobol / Halton     u = the i-th point (1-based) of the base-2 van der
//                      Corput sequence in Gray-code order (Sobol, dimension
//                      one) or natural order (Halton base 2), z = Acklam(u)
// ----------------------------------------------------------------------------
template <int UPT>
__device__ __forceinline__ void sim_vr(const McOption& o, uint32_t unit0, uint32_t stride,
                                       uint32_t k0, uint32_t k1, Acc& acc) {
    const uint32_t n = (uint32_t)o.paths;
    const int32_t m = o.model;
    const double d0 = o.d[0], d1 = o.d[1], shift = o.d[2], mean_st = o.d[3];
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
        const uint32_t unit = unit0 + (uint32_t)k * stride;
        if (unit * 4u >= n) continue;
        double z[4];
        if (m == kQmcSobol || m == kQmcHalton) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const uint32_t i1 = unit * 4u + (uint32_t)s + 1u;
                // quasi_monte_carlo.cpp:23-24 / 46-47 with internal_util.h:104-130:
                // bit j of the (Gray-coded) index goes to bit 31 - j.
                const uint32_t x = __brev(m == kQmcSobol ? (i1 ^ (i1 >> 1)) : i1);
                const double u = m == kQmcSobol ? ((double)x + 0.5) / 4294967296.0
                                                : (double)x * 0x1p-32;
                z[s] = acklam_inv(clamp_unit(u));
            }
        } else if (m == kStratified) {
            const U4 w = philox4x32_10(unit, 0u, 0u, 2u, k0, k1);
            const uint32_t bits[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const double ui = ((double)bits[s] + 0.5) * 0x1p-32;
                const double u = ((double)(unit * 4u + (uint32_t)s) + ui) / (double)n;
                z[s] = acklam_inv(clamp_unit(u));
            }
        } else {
            normals4_f64(unit, 1u, k0, k1, z);
        }
        double y[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const bool valid = unit * 4u + (uint32_t)s < n;
            double zz = z[s];
            double w = 1.0;
            if (m == kImportanceSampling) {
                zz = z[s] + shift;
                w = exp(-shift * zz + 0.5 * shift * shift);
            }
            const double st = o.spot * exp(d0 + d1 * zz);
            const double pay = payoff(st, o.strike, o.option_type) * w;
            y[s] = pay;
            if (!valid) continue;
            acc.sy = dd_add(acc.sy, pay);
            if (m != kStratified) acc.q = dd_add(acc.q, pay * pay);
            if (m == kControlVariates) {
                const double c = st - mean_st;
                acc.cx += c;
                acc.cxx += c * c;
                acc.cxy += c * pay;
            }
        }
        if (m == kStratified) {
#pragma unroll
            for (int s = 0; s < 4; s += 2) {
                if (unit * 4u + (uint32_t)s + 1u < n) {
                    const double dy = y[s] - y[s + 1];
                    acc.q = dd_add(acc.q, dy * dy);
                }
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Fixed-order CTA reduction of (sy, q) into the tile's slot.
// ----------------------------------------------------------------------------
template <int BLOCK, bool CV>
__device__ __forceinline__ void reduce_tile(Acc acc, TilePartial* __restrict__ out, DD* smem) {
    constexpr int W = BLOCK / 32;
    DD a = acc.sy, b = acc.q;
    double lone = acc.lone;  // nonzero in at most one thread: plain sums are exact
    double cx = acc.cx, cxx = acc.cxx, cxy = acc.cxy;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a = dd_merge(a, dd_shfl_down(a, off));
        b = dd_merge(b, dd_shfl_down(b, off));
        lone = __dadd_rn(lone, __shfl_down_sync(0xffffffffu, lone, off));
        if (CV) {
            cx = __dadd_rn(cx, __shfl_down_sync(0xffffffffu, cx, off));
            cxx = __dadd_rn(cxx, __shfl_down_sync(0xffffffffu, cxx, off));
            cxy = __dadd_rn(cxy, __shfl_down_sync(0xffffffffu, cxy, off));
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        smem[warp] = a;
        smem[W + warp] = b;
        smem[2 * W + warp] = DD{lone, 0.0};
        if (CV) {
            smem[3 * W + warp] = DD{cx, cxx};
            smem[4 * W + warp] = DD{cxy, 0.0};
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DD ta = smem[0], tb = smem[W];
        double tl = smem[2 * W].hi;
        double tx = 0.0, txx = 0.0, txy = 0.0;
        if (CV) {
            tx = smem[3 * W].hi;
            txx = smem[3 * W].lo;
            txy = smem[4 * W].hi;
        }
#pragma unroll
        for (int w = 1; w < W; ++w) {
            ta = dd_merge(ta, smem[w]);
            tb = dd_merge(tb, smem[W + w]);
            tl = __dadd_rn(tl, smem[2 * W + w].hi);
            if (CV) {
                tx = __dadd_rn(tx, smem[3 * W + w].hi);
                txx = __dadd_rn(txx, smem[3 * W + w].lo);
                txy = __dadd_rn(txy, smem[4 * W + w].hi);
            }
        }
        TilePartial t;
        t.sy_hi = ta.hi;
        t.sy_lo = ta.lo;
        t.q_hi = tb.hi;
        t.q_lo = tb.lo;
        t.lone = tl;
        t.cx = tx;
        t.cxx = txx;
        t.cxy = txy;
        *out = t;
    }
    __syncthreads();
}

// Option owning `tile`: the last i with tile_begin[i] <= tile (tile_begin is
// non-decreasing, n + 1 entries, tile_begin[n] = total tiles).
__device__ __forceinline__ int32_t find_option(const int64_t* __restrict__ tile_begin, int32_t n,
                                               int64_t tile) {
    int32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(tile_begin + mid) <= tile)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <int FAMILY, int UPT, bool ANTI, int SU>
__device__ __forceinline__ void sim_family(const McOption& o, uint32_t unit0, uint32_t stride,
                                           uint32_t k0, uint32_t k1, Acc& acc) {
    if (FAMILY == kFamTerminal) sim_terminal<UPT, ANTI>(o, unit0, stride, k0, k1, acc);
    if (FAMILY == kFamEuler) sim_stepwise<UPT, ANTI, false, SU>(o, unit0, stride, k0, k1, acc);
    if (FAMILY == kFamMilstein) sim_stepwise<UPT, ANTI, true, SU>(o, unit0, stride, k0, k1, acc);
    if (FAMILY == kFamHeston) sim_heston<UPT, ANTI, false, SU>(o, unit0, stride, k0, k1, acc);
    if (FAMILY == kFamHestonLr) sim_heston<UPT, ANTI, true, SU>(o, unit0, stride, k0, k1, acc);
    if (FAMILY == kFamVr) sim_vr<UPT>(o, unit0, stride, k0, k1, acc);
}

// One tile: all UPT * unit_iters units of every thread, then the reduction.
template <int FAMILY, int BLOCK, int UPT, bool ANTI, int SU = 1>
__device__ __forceinline__ void run_tile(const McOption& o, int64_t tile, TilePartial* partials,
                                         DD* smem) {
    const uint32_t k0 = (uint32_t)o.seed, k1 = (uint32_t)(o.seed >> 32);
    const int64_t local = tile - o.tile_begin;
    const uint32_t per_iter = (uint32_t)(BLOCK * UPT);
    const uint32_t first = (uint32_t)(local * (int64_t)per_iter * o.unit_iters);
    Acc acc;
    for (int32_t it = 0; it < o.unit_iters; ++it) {
        const uint32_t base = first + (uint32_t)it * per_iter;
        if (base >= (uint32_t)o.units) break;
        sim_family<FAMILY, UPT, ANTI, SU>(o, base + threadIdx.x, (uint32_t)BLOCK, k0, k1, acc);
    }
    reduce_tile<BLOCK, FAMILY == kFamVr>(acc, partials + tile, smem);
}

// ----------------------------------------------------------------------------
// Kernel 1a: single-family simulate, grid-stride over tiles [tile0, tile0 +
// n_tiles) of the options opts[0, n).
// ----------------------------------------------------------------------------
// No register cap: the kernel is issue- and special-function-bound, and
// forcing 64 registers (4 CTAs of 256 per SM) added instructions and ran
// slower on B200 than the compiler's 70 (3 CTAs).
template <int FAMILY, int BLOCK, int UPT, bool ANTI, int SU>
__global__ void __launch_bounds__(BLOCK)
    mc_simulate_kernel(const McOption* __restrict__ opts, const int64_t* __restrict__ tile_begin,
                       int32_t n, int64_t tile0, int64_t n_tiles, TilePartial* __restrict__ partials) {
    __shared__ DD smem[5 * (BLOCK / 32)];
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const int64_t tile = tile0 + t;  // tile_begin holds absolute tile indices
        const int32_t oi = find_option(tile_begin, n, tile);
        const McOption o = opts[oi];
        run_tile<FAMILY, BLOCK, UPT, ANTI, SU>(o, tile, partials, smem);
    }
}

// ----------------------------------------------------------------------------
// Kernel 1b: persistent work-stealing simulate for mixed batches.  One CTA per
// resident slot; each CTA takes the next tile from a global counter until the
// list is exhausted.  The records are in work order, in runs ("groups") of one
// (family, antithetic) pair, so consecutive claims mostly fall in one group:
// a CTA enters a group's loop once -- one call of that family's code, compiled
// and register-allocated on its own -- and keeps claiming and simulating
// tiles inside it until a claim lands past the group, with the owning record
// found by a forward search from the previous one (claims only grow).  The
// next tile is claimed when the current one starts and its index is only read
// when the current one ends, so the atomic's round trip overlaps the
// simulation.  The counter is reset by the finalize kernel of the same
// execute, so a captured graph can replay without a memset.  The counter only
// grows: all CTAs together claim at most n_tiles + gridDim.x indices, so every
// loop ends.
// ----------------------------------------------------------------------------

// Last record i in [lo, hi) with tile_begin[i] <= tile, given tile_begin[lo] <=
// tile and tile_begin non-decreasing: gallop forward, then bisect.
__device__ __forceinline__ int32_t advance_option(const int64_t* __restrict__ tile_begin,
                                                  int32_t lo, int32_t hi, int64_t tile) {
    int32_t step = 1;
    while (lo + step < hi && __ldg(tile_begin + lo + step) <= tile) {
        lo += step;
        step <<= 1;
    }
    int32_t top = (lo + step < hi ? lo + step : hi) - 1;
    while (lo < top) {
        const int32_t mid = (lo + top + 1) >> 1;
        if (__ldg(tile_begin + mid) <= tile)
            lo = mid;
        else
            top = mid - 1;
    }
    return lo;
}

// Tiles of one group, from `tile` (claimed, inside the group) until a claim
// lands past the group; returns that claim.
template <int FAMILY, int BLOCK, int UPT, bool ANTI>
__device__ __noinline__ int64_t run_group(const McOption* __restrict__ opts,
                                          const int64_t* __restrict__ tile_begin, int32_t opt_lo,
                                          int32_t opt_hi, int64_t tile_hi,
                                          TilePartial* __restrict__ partials,
                                          unsigned long long* __restrict__ work_counter, DD* smem,
                                          long long* s_tile, int64_t tile) {
    int32_t oi = advance_option(tile_begin, opt_lo, opt_hi, tile);
    McOption o = opts[oi];
    for (;;) {
        // claim the next tile now; thread 0 first uses the result below
        long long next = 0;
        if (threadIdx.x == 0) next = (long long)atomicAdd(work_counter, 1ull);
        run_tile<FAMILY, BLOCK, UPT, ANTI>(o, tile, partials, smem);  // ends in a CTA barrier
        if (threadIdx.x == 0) *s_tile = next;
        __syncthreads();
        // every thread reads s_tile here, and the next write to it follows the
        // barrier at the end of the next tile
        tile = *s_tile;
        if (tile >= tile_hi) return tile;
        if (tile >= o.tile_begin + o.tiles) {
            oi = advance_option(tile_begin, oi + 1, opt_hi, tile);
            o = opts[oi];
        }
    }
}

// Eight 128-thread CTAs per SM (64 registers): every family body is compiled
// within that budget; five, six and seven CTAs per SM measured slower on the
// mixed benchmark batch (52.1, 51.7, 51.2 vs 51.0 ms).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
    mc_persistent_kernel(const McOption* __restrict__ opts, const int64_t* __restrict__ tile_begin,
                         int64_t n_tiles, TilePartial* __restrict__ partials,
                         unsigned long long* __restrict__ work_counter,
                         const GroupTable* __restrict__ groups) {
    __shared__ DD smem[5 * (BLOCK / 32)];
    __shared__ long long s_tile;
    if (threadIdx.x == 0) s_tile = (long long)atomicAdd(work_counter, 1ull);
    __syncthreads();
    int64_t tile = s_tile;
    const int32_t count = groups->count;
    int32_t g = 0;
    while (tile < n_tiles) {
        // claims only grow, so the group index only moves forward
        while (g < count && tile >= groups->tile_hi[g]) ++g;
        if (g >= count) break;  // the groups cover every tile; defensive
        const int32_t lo = groups->opt_lo[g], hi = groups->opt_hi[g];
        const int64_t th = groups->tile_hi[g];
        switch (groups->code[g]) {
#define QK_GROUP(FAM, UPT, ANTI)                                                                  \
    case FAM * 2 + (ANTI ? 1 : 0):                                                               \
        tile = run_group<FAM, BLOCK, UPT, ANTI>(opts, tile_begin, lo, hi, th, partials,          \
                                                work_counter, smem, &s_tile, tile);              \
        break;
            QK_GROUP(kFamTerminal, kFamilyUpt<kFamTerminal>, true)
            QK_GROUP(kFamTerminal, kFamilyUpt<kFamTerminal>, false)
            QK_GROUP(kFamEuler, kFamilyUpt<kFamEuler>, true)
            QK_GROUP(kFamEuler, kFamilyUpt<kFamEuler>, false)
            QK_GROUP(kFamMilstein, kFamilyUpt<kFamMilstein>, true)
            QK_GROUP(kFamMilstein, kFamilyUpt<kFamMilstein>, false)
            QK_GROUP(kFamHeston, kFamilyUpt<kFamHeston>, true)
            QK_GROUP(kFamHeston, kFamilyUpt<kFamHeston>, false)
            QK_GROUP(kFamHestonLr, kFamilyUpt<kFamHestonLr>, true)
            QK_GROUP(kFamHestonLr, kFamilyUpt<kFamHestonLr>, false)
            QK_GROUP(kFamVr, kFamilyUpt<kFamVr>, false)
#undef QK_GROUP
            default:
                tile = n_tiles;  // unknown code: the host never builds one
                break;
        }
    }
}

// ----------------------------------------------------------------------------
// Kernel 2: finalize.  One warp per option merges the option's tile slots in
// tile order (lane-strided, then a fixed shuffle tree), then writes price and
// standard error.  Also resets the work counter for the next execute.
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    mc_finalize_kernel(const McOption* __restrict__ opts, int32_t n,
                       const TilePartial* __restrict__ partials, double* __restrict__ out_price,
                       double* __restrict__ out_se, const int32_t* __restrict__ out_index,
                       unsigned long long* __restrict__ work_counter) {
    if (work_counter != nullptr && blockIdx.x == 0 && threadIdx.x == 0) *work_counter = 0ull;
    const int32_t warp = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const McOption& o = opts[warp];
    const int32_t dst = out_index != nullptr ? out_index[warp] : warp;
    if (o.mode != kModeSimulate) {
        if (lane == 0) {
            out_price[dst] = o.const_price;
            out_se[dst] = __longlong_as_double(0x7FF8000000000000ll);
        }
        return;
    }
    DD sy{0.0, 0.0}, q{0.0, 0.0};
    double lone = 0.0, cx = 0.0, cxx = 0.0, cxy = 0.0;
    for (int32_t t = lane; t < o.tiles; t += 32) {
        const TilePartial p = partials[o.tile_begin + t];
        sy = dd_merge(sy, DD{p.sy_hi, p.sy_lo});
        q = dd_merge(q, DD{p.q_hi, p.q_lo});
        lone = __dadd_rn(lone, p.lone);
        cx = __dadd_rn(cx, p.cx);
        cxx = __dadd_rn(cxx, p.cxx);
        cxy = __dadd_rn(cxy, p.cxy);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sy = dd_merge(sy, dd_shfl_down(sy, off));
        q = dd_merge(q, dd_shfl_down(q, off));
        lone = __dadd_rn(lone, __shfl_down_sync(0xffffffffu, lone, off));
        cx = __dadd_rn(cx, __shfl_down_sync(0xffffffffu, cx, off));
        cxx = __dadd_rn(cxx, __shfl_down_sync(0xffffffffu, cxx, off));
        cxy = __dadd_rn(cxy, __shfl_down_sync(0xffffffffu, cxy, off));
    }
    if (lane == 0) {
        const double s = sy.hi + sy.lo;
        const double qq = q.hi + q.lo;
        const double np = (double)o.paths;
        const double nan = __longlong_as_double(0x7FF8000000000000ll);
        double price, se = nan;
        if (o.model == kControlVariates) {
            // control_variates.cpp:40-51 with x = disc S_T and y = disc payoff;
            // the control is summed centred on E[S_T], so mean_x - E[x] is
            // disc * mc and the disc factors cancel in beta.
            const double mp = s / np, mc = cx / np;
            const double vc = cxx / np - mc * mc;
            const double vp = qq / np - mp * mp;
            if (o.disc * o.disc * vc <= 1e-12) {
                price = o.disc * mp;
                if (np >= 2.0) se = o.disc * sqrt(fmax(vp, 0.0) / (np - 1.0));
            } else {
                const double cov = cxy / np - mc * mp;
                const double beta = cov / vc;
                price = o.disc * (mp - beta * mc);
                // residual variance of payoff - beta * control
                const double res = vp - cov * beta;
                se = o.disc * sqrt(fmax(res, 0.0) / (np - 2.0));
            }
        } else if (o.model == kStratified) {
            price = o.disc * (s / np);
            // paired strata: Var(mean) ~ sum over pairs (y_a - y_b)^2 / n^2
            se = o.disc * sqrt(qq) / np;
        } else {
            // sum of all path payoffs: two per pair, plus the unpaired path
            const double total = o.antithetic ? __dadd_rn(2.0 * s, lone) : s;
            price = o.disc * (total / np);
            const double ns = (double)o.samples;
            if (ns >= 2.0) {
                const double mean = s / ns;
                double var = (qq - ns * mean * mean) / (ns - 1.0);
                if (var < 0.0) var = 0.0;
                se = o.disc * sqrt(var / ns);
            }
        }
        out_price[dst] = price;
        out_se[dst] = se;
    }
}

template <int FAMILY, int BLOCK, int UPT, bool ANTI, int SU>
cudaError_t launch_one(const SimArgs& a, cudaStream_t st) {
    const int64_t cap = (int64_t)a.max_ctas;
    const unsigned grid = (unsigned)(a.n_tiles < cap ? a.n_tiles : cap);
    mc_simulate_kernel<FAMILY, BLOCK, UPT, ANTI, SU>
        <<<grid, BLOCK, 0, st>>>(a.opts, a.tile_begin, a.n, a.tile0, a.n_tiles, a.partials);
    return cudaGetLastError();
}

constexpr bool is_stepwise(int family) {
    return family == kFamEuler || family == kFamMilstein || family == kFamHeston ||
           family == kFamHestonLr;
}

// Step unrolling 2 where step_unroll2_compiled() says so.
template <int FAMILY, int BLOCK, bool ANTI>
cudaError_t launch_upt(int upt, int su, const SimArgs& a, cudaStream_t st) {
    if constexpr (is_stepwise(FAMILY)) {
        if (su == 2) {
            if (!step_unroll2_compiled(FAMILY, upt)) return cudaErrorInvalidValue;
            switch (upt) {
                case 1: return launch_one<FAMILY, BLOCK, 1, ANTI, 2>(a, st);
                case 2: return launch_one<FAMILY, BLOCK, 2, ANTI, 2>(a, st);
                default:
                    if constexpr (step_unroll2_compiled(FAMILY, 4))
                        return launch_one<FAMILY, BLOCK, 4, ANTI, 2>(a, st);
                    return cudaErrorInvalidValue;
            }
        }
    }
    if (su != 1) return cudaErrorInvalidValue;
    switch (upt) {
        case 1: return launch_one<FAMILY, BLOCK, 1, ANTI, 1>(a, st);
        case 2: return launch_one<FAMILY, BLOCK, 2, ANTI, 1>(a, st);
        case 4: return launch_one<FAMILY, BLOCK, 4, ANTI, 1>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int FAMILY, bool ANTI>
cudaError_t launch_block(int block, int upt, int su, const SimArgs& a, cudaStream_t st) {
    switch (block) {
        case 128: return launch_upt<FAMILY, 128, ANTI>(upt, su, a, st);
        case 256: return launch_upt<FAMILY, 256, ANTI>(upt, su, a, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int FAMILY>
cudaError_t launch_anti(bool anti, int block, int upt, int su, const SimArgs& a, cudaStream_t st) {
    return anti ? launch_block<FAMILY, true>(block, upt, su, a, st)
                : launch_block<FAMILY, false>(block, upt, su, a, st);
}

}  // namespace

int family_of(int32_t model) {
    switch (model) {
        case kStandard:
        case kAntithetic:
        case kTerminalPlain: return kFamTerminal;
        case kEuler:
        case kLocalVol: return kFamEuler;
        case kMilstein: return kFamMilstein;
        case kHestonLrDelta: return kFamHestonLr;
        case kControlVariates:
        case kImportanceSampling:
        case kStratified:
        case kQmcSobol:
        case kQmcHalton: return kFamVr;
        default: return kFamHeston;
    }
}

cudaError_t launch_simulate(int family, bool anti, int block, int upt, int su, const SimArgs& a,
                            cudaStream_t st) {
    if (a.n_tiles <= 0) return cudaSuccess;
    switch (family) {
        case kFamTerminal: return launch_anti<kFamTerminal>(anti, block, upt, su, a, st);
        case kFamEuler: return launch_anti<kFamEuler>(anti, block, upt, su, a, st);
        case kFamMilstein: return launch_anti<kFamMilstein>(anti, block, upt, su, a, st);
        case kFamHeston: return launch_anti<kFamHeston>(anti, block, upt, su, a, st);
        case kFamHestonLr: return launch_anti<kFamHestonLr>(anti, block, upt, su, a, st);
        case kFamVr: return launch_block<kFamVr, false>(block, upt, su, a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_persistent(int block, const SimArgs& a, const GroupTable* groups,
                              unsigned long long* work_counter, cudaStream_t st) {
    if (a.n_tiles <= 0) return cudaSuccess;
    const int64_t cap = (int64_t)a.max_ctas;
    const unsigned grid = (unsigned)(a.n_tiles < cap ? a.n_tiles : cap);
    if (block == 128)
        mc_persistent_kernel<128><<<grid, 128, 0, st>>>(a.opts, a.tile_begin, a.n_tiles,
                                                        a.partials, work_counter, groups);
    else if (block == 256)
        mc_persistent_kernel<256><<<grid, 256, 0, st>>>(a.opts, a.tile_begin, a.n_tiles,
                                                        a.partials, work_counter, groups);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_finalize(const McOption* opts, int32_t n, const TilePartial* partials,
                            double* out_price, double* out_se, const int32_t* out_index,
                            unsigned long long* work_counter, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int64_t threads = (int64_t)n * 32;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    mc_finalize_kernel<<<grid, 256, 0, st>>>(opts, n, partials, out_price, out_se, out_index,
                                             work_counter);
    return cudaGetLastError();
}

int max_resident_ctas(int family_or_persistent, int block, int upt, int device) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    int per_sm = 0;
    cudaError_t e = cudaSuccess;
    if (family_or_persistent < 0) {
        e = block == 128 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc_persistent_kernel<128>, 128, 0)
                         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc_persistent_kernel<256>, 256, 0);
    } else {
        // Occupancy of the Heston variant bounds the others (most registers).
        if (block == 128) {
            e = upt == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc_simulate_kernel<kFamHeston, 128, 1, true, 1>, 128, 0)
              : upt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc_simulate_kernel<kFamHeston, 128, 2, true, 1>, 128, 0)
                         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc_simulate_kernel<kFamHeston, 128, 4, true, 1>, 128, 0);
        } else {
            e = upt == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc_simulate_kernel<kFamHeston, 256, 1, true, 1>, 256, 0)
              : upt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc_simulate_kernel<kFamHeston, 256, 2, true, 1>, 256, 0)
                         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc_simulate_kernel<kFamHeston, 256, 4, true, 1>, 256, 0);
        }
    }
    if (e != cudaSuccess || per_sm <= 0) return 0;
    return sms * per_sm;
}

}  // namespace qkb
