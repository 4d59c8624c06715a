// cf_kernels.cu -- batch Heston Fourier pricers on the GPU.
//
// 1. Characteristic-function price (heston_cf_kernel):
// Restates yluoc/Quant-Kernel closed_form_semi_analytical/heston/heston.cpp:7-53
// (little-trap characteristic function) and the P1/P2 integration of
// closed_form_semi_analytical/common/internal_util.h:80-142:
// ceil(steps/64) panels of the 64-point Gauss-Legendre rule on [1e-8, limit],
// two characteristic-function values per node.  One 128-thread CTA prices one
// option: threads take nodes round-robin, accumulate in FP64 and reduce in a
// fixed order, so results are deterministic.  The rule's nodes and weights are
// computed on the host (Newton on the Legendre recurrence) and held in
// constant memory.
//
// 2. COS expansion (heston_cos_kernel): yluoc/Quant-Kernel
// fourier_transform_methods/cos_method/cos_method.cpp:30-58 with the
// log-price characteristic function of common/charfn_concepts.h:54-78 and
// the cosine sum of cos_method.h:13-57: n_terms terms on [a, b], one CTA per
// option, terms round-robin over the threads, FP64, fixed-order reduction.
#include "cf_kernels.h"

#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "mc_plan.h"
#include "qk_fault.h"

namespace qkb {

namespace {

__constant__ double c_gl_x[32];
__constant__ double c_gl_w[32];

struct Cx {
    double re, im;
};
__device__ __forceinline__ Cx cx(double r, double i) { return Cx{r, i}; }
__device__ __forceinline__ Cx operator+(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ Cx operator-(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ Cx operator*(double s, Cx a) { return cx(s * a.re, s * a.im); }
__device__ __forceinline__ Cx operator/(Cx a, Cx b) {
    // Smith's algorithm (scaled division)
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re, d = b.re + b.im * r;
        return cx((a.re + a.im * r) / d, (a.im - a.re * r) / d);
    }
    const double r = b.re / b.im, d = b.re * r + b.im;
    return cx((a.re * r + a.im) / d, (a.im * r - a.re) / d);
}
__device__ __forceinline__ Cx cexp_(Cx a) {
    double s, c;
    sincos(a.im, &s, &c);
    const double e = exp(a.re);
    return cx(e * c, e * s);
}
// Principal logarithm.  Near |a| = 1 the real part is 0.5 log1p(x^2 + y^2 - 1)
// with x^2 and y^2 split into exact FMA products: log(hypot(x, y)) would carry
// an absolute error of one ulp of 1 there, which the 1/u factor of the P1/P2
// integrands magnifies at small u.
__device__ __forceinline__ Cx clog_(Cx a) {
    const double ax = fabs(a.re), ay = fabs(a.im);
    const double big = fmax(ax, ay), small = fmin(ax, ay);
    const double hb = big * big;
    double lr;
    if (hb >= 0.5 && hb <= 2.0) {
        const double lb = fma(big, big, -hb);
        const double hs = small * small;
        const double ls = fma(small, small, -hs);
        const double s = hb - 1.0;  // exact for hb in [0.5, 2]
        const double t = s + hs;    // two-sum of s and hs
        const double bp = t - s;
        const double err = (s - (t - bp)) + (hs - bp);
        lr = 0.5 * log1p(t + (err + lb + ls));
    } else {
        lr = log(hypot(a.re, a.im));
    }
    return cx(lr, atan2(a.im, a.re));
}
// Principal square root (branch cut on the negative real axis).  The smaller
// component comes from a division, not from sqrt(|a| - |re|), which cancels
// when |im| << |re|.
__device__ __forceinline__ Cx csqrt_(Cx a) {
    const double m = hypot(a.re, a.im);
    if (m == 0.0) return cx(0.0, a.im);
    if (a.re >= 0.0) {
        const double t = sqrt(0.5 * (m + a.re));
        return cx(t, a.im / (2.0 * t));
    }
    const double t = sqrt(0.5 * (m - a.re));
    return cx(fabs(a.im) / (2.0 * t), copysign(t, a.im));
}

// Complex product and quotient for the characteristic function, with the
// multiply-adds fused explicitly (one rounding per component) and Smith's
// scaled division taking one reciprocal instead of two quotients.
__device__ __forceinline__ Cx fmul(Cx a, Cx b) {
    return cx(fma(a.re, b.re, -(a.im * b.im)), fma(a.re, b.im, a.im * b.re));
}
__device__ __forceinline__ Cx fdiv(Cx a, Cx b) {
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re, inv = 1.0 / fma(b.im, r, b.re);
        return cx(fma(a.im, r, a.re) * inv, fma(-a.re, r, a.im) * inv);
    }
    const double r = b.re / b.im, inv = 1.0 / fma(b.re, r, b.im);
    return cx(fma(a.re, r, a.im) * inv, fma(a.im, r, -a.re) * inv);
}

struct HestonCf {
    double kappa, theta_k_s2, rho_sigma, sigma2, inv_sigma2, v0, t, drift;
    // heston.cpp:33-44.  Not inlined: the body is large and is called at three
    // places; one copy keeps the kernel inside the instruction cache.
    __device__ __noinline__ Cx operator()(Cx u) const {
        const Cx iu = cx(-u.im, u.re);
        const Cx beta = cx(kappa, 0.0) - rho_sigma * iu;
        const Cx d = csqrt_(fmul(beta, beta) + sigma2 * (iu + fmul(u, u)));
        const Cx bmd = beta - d;
        const Cx g = fdiv(bmd, beta + d);
        const Cx e = cexp_(cx(-d.re * t, -d.im * t));
        const Cx one = cx(1.0, 0.0);
        const Cx one_ge = one - fmul(g, e);
        const Cx C = drift * iu + theta_k_s2 * (t * bmd - 2.0 * clog_(fdiv(one_ge, one - g)));
        const Cx D = fmul(inv_sigma2 * bmd, fdiv(one - e, one_ge));
        return cexp_(C + v0 * D);
    }
};

// Six CTAs per SM (80 registers, a few spilled) instead of the compiler's five
// (94 registers): the FP64 pipe is half idle at five, and the sixth CTA's
// warps fill it (65536 options: 7.5 -> 6.6 ms end to end; eight CTAs measured
// the same, seven slower).
__global__ void __launch_bounds__(128, 6)
    heston_cf_kernel(const CfOption* __restrict__ opts, int32_t n, double* __restrict__ out) {
    __shared__ double s1s[128], s2s[128];
    const int32_t i = blockIdx.x;
    if (i >= n) return;
    const CfOption o = opts[i];
    if (o.mode != 0) {
        if (threadIdx.x == 0) out[i] = o.const_price;
        return;
    }
    HestonCf cf;
    cf.kappa = o.kappa;
    cf.sigma2 = o.sigma * o.sigma;
    cf.inv_sigma2 = 1.0 / cf.sigma2;
    cf.theta_k_s2 = o.kappa * o.theta * cf.inv_sigma2;
    cf.rho_sigma = o.rho * o.sigma;
    cf.v0 = o.v0;
    cf.t = o.t;
    cf.drift = log(o.spot) + (o.r - o.q) * o.t;
    const double lk = log(o.strike);
    const Cx phi_mi = cf(cx(0.0, -1.0));
    const double phi_abs = hypot(phi_mi.re, phi_mi.im);
    const double inv_phi_abs2 = 1.0 / (phi_mi.re * phi_mi.re + phi_mi.im * phi_mi.im);
    const double a = 1e-8, width = (o.limit - a) / static_cast<double>(o.panels);
    double s1 = 0.0, s2 = 0.0;
    // 64-bit node counter: panels * 64 and the strided index can pass INT32_MAX
    const int64_t nodes = static_cast<int64_t>(o.panels) * 64;
    for (int64_t k = threadIdx.x; k < nodes; k += blockDim.x) {
        const int32_t p = static_cast<int32_t>(k >> 6), j = static_cast<int32_t>((k >> 1) & 31),
                      side = static_cast<int32_t>(k & 1);
        const double pa = a + static_cast<double>(p) * width;
        const double pb = pa + width;
        const double mid = 0.5 * (pa + pb), half = 0.5 * (pb - pa);
        const double u = side == 0 ? mid - half * c_gl_x[j] : mid + half * c_gl_x[j];
        const double wi = c_gl_w[j];
        const double inv_u = 1.0 / u;
        double sn, cs;
        sincos(u * lk, &sn, &cs);
        const Cx c2 = cf(cx(u, 0.0));
        s2 += half * wi * ((cs * c2.im - sn * c2.re) * inv_u);
        if (phi_abs >= 1e-14) {
            const Cx c1 = cf(cx(u, -1.0));
            const double n1_re = cs * c1.re + sn * c1.im;
            const double n1_im = cs * c1.im - sn * c1.re;
            const double d_re = n1_im * inv_u, d_im = -n1_re * inv_u;
            s1 += half * wi * ((d_re * phi_mi.re + d_im * phi_mi.im) * inv_phi_abs2);
        }
    }
    s1s[threadIdx.x] = s1;
    s2s[threadIdx.x] = s2;
    __syncthreads();
    for (int off = 64; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            s1s[threadIdx.x] += s1s[threadIdx.x + off];
            s2s[threadIdx.x] += s2s[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double kPi = 3.1415926535897932384626433832795;
        double p2 = 0.5 + s2s[0] / kPi;
        double p1 = 0.5 + s1s[0] / kPi;
        p2 = fmin(1.0, fmax(0.0, p2));
        p1 = fmin(1.0, fmax(0.0, p1));
        double price;
        if (!(phi_abs >= 1e-14) || !isfinite(p1) || !isfinite(p2)) {
            price = __longlong_as_double(0x7FF8000000000000ll);
        } else {
            const double call = o.spot * exp(-o.q * o.t) * p1 - o.strike * exp(-o.r * o.t) * p2;
            price = o.option_type == 0 ? call : call - o.spot * exp(-o.q * o.t) + o.strike * exp(-o.r * o.t);
        }
        out[i] = price;
    }
}


// ---------------------------------------------------------------------------
// COS expansion.  Complex arithmetic in the reference's expression order
// (std::complex products and real-complex mixes), so the terms agree with the
// reference's to rounding.
// ---------------------------------------------------------------------------
__device__ __forceinline__ Cx cmul(Cx a, Cx b) {
    return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
// real - complex as std::complex does it: (x - re, 0 - im)
__device__ __forceinline__ Cx rsub(double x, Cx a) { return cx(x - a.re, 0.0 - a.im); }
__device__ __forceinline__ Cx scale(Cx a, double s) { return cx(a.re * s, a.im * s); }

struct HestonLogCf {
    double spot_log, r, q, v0, kappa, theta, sigma, rho;
    // charfn_concepts.h:57-77: phi(u, t) of log S_t
    __device__ __noinline__ Cx operator()(Cx u, double t) const {
        const Cx iu = cmul(cx(0.0, 1.0), u);
        const Cx rs_iu = scale(iu, rho * sigma);
        const Cx a = rsub(kappa, rs_iu);
        const Cx b = scale(iu + cmul(u, u), sigma * sigma);
        const Cx d = csqrt_(cmul(a, a) + b);
        const Cx amd = a - d;
        const Cx g = amd / (a + d);
        const Cx edt = cexp_(scale(cx(-d.re, -d.im), t));
        const Cx lg = clog_(rsub(1.0, cmul(g, edt)) / rsub(1.0, g));
        const Cx C = scale(scale(amd, t) - scale(lg, 2.0), kappa * theta / (sigma * sigma));
        const Cx D = cmul(cx(amd.re / (sigma * sigma), amd.im / (sigma * sigma)), rsub(1.0, edt)) /
                     rsub(1.0, cmul(g, edt));
        return cexp_(scale(iu, spot_log) + scale(scale(iu, r - q), t) + C + scale(D, v0));
    }
};

__global__ void __launch_bounds__(128)
    heston_cos_kernel(const CfOption* __restrict__ opts, int32_t n, double* __restrict__ out) {
    __shared__ double ss[128];
    const int32_t i = blockIdx.x;
    if (i >= n) return;
    const CfOption o = opts[i];
    if (o.mode != 0) {
        if (threadIdx.x == 0) out[i] = o.const_price;
        return;
    }
    const double kPi = 3.1415926535897932384626433832795;
    const double a = o.limit, b = o.hi;
    const double lk = log(o.strike);
    const double cm = lk < a ? a : lk;   // std::min(std::max(log K, a), b)
    const double c = b < cm ? b : cm;
    const double dd = b;
    const bool summed = c < dd;
    double s = 0.0;
    if (summed) {
        HestonLogCf phi;
        phi.spot_log = log(o.spot);
        phi.r = o.r;
        phi.q = o.q;
        phi.v0 = o.v0;
        phi.kappa = o.kappa;
        phi.theta = o.theta;
        phi.sigma = o.sigma;
        phi.rho = o.rho;
        const double interval = b - a;
        const double inv = 1.0 / interval;
        const double exp_d = exp(dd), exp_c = exp(c);
        for (int64_t k = threadIdx.x; k < o.panels; k += blockDim.x) {  // 64-bit: no wrap
            const double u = static_cast<double>(k) * kPi * inv;
            double chi, psi;
            if (k == 0) {
                chi = exp_d - exp_c;
                psi = dd - c;
            } else {
                double sd, cd, sc, cc;
                sincos(u * (dd - a), &sd, &cd);
                sincos(u * (c - a), &sc, &cc);
                chi = ((cd * exp_d - cc * exp_c) + u * (sd * exp_d - sc * exp_c)) / (1.0 + u * u);
                psi = (sd - sc) / u;
            }
            const double u_k = 2.0 * inv * (chi - o.strike * psi);
            const Cx f = phi(cx(u, 0.0), o.t);
            // Re(phi * exp(-i u a)) = Re(phi * (cos ua, -sin ua))
            double sa, ca;
            sincos(u * a, &sa, &ca);
            const double f_k = f.re * ca - f.im * (-sa);
            const double weight = (k == 0) ? 0.5 : 1.0;
            s += weight * f_k * u_k;
        }
    }
    ss[threadIdx.x] = s;
    __syncthreads();
    for (int off = 64; off > 0; off >>= 1) {
        if (threadIdx.x < off) ss[threadIdx.x] += ss[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double call = summed ? exp(-o.r * o.t) * ss[0] : 0.0;
        call = (0.0 < call) ? call : 0.0;  // std::max(0.0, call): NaN -> 0
        out[i] = o.option_type == 0 ? call
                                    : call - o.spot * exp(-o.q * o.t) + o.strike * exp(-o.r * o.t);
    }
}

// 64-point Gauss-Legendre nodes (the 32 positive ones) and weights.
void gl64(double* x, double* w) {
    const int n = 64;
    for (int i = 0; i < 32; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = pk;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[31 - i] = z;
        w[31 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

bool finite_(double x) { return std::isfinite(x); }

double intrinsic_(double s, double k, int32_t ot) {
    const double d = ot == 0 ? s - k : k - s;
    return (0.0 < d) ? d : 0.0;
}

constexpr int kMaxDev = 64;
std::mutex g_cf_mu;
bool g_cf_ready[kMaxDev] = {};

}  // namespace

CfOption pack_cf_option(double spot, double strike, double t, double r, double q, double v0,
                        double kappa, double theta, double sigma, double rho, int32_t ot,
                        int32_t steps, double limit) {
    CfOption o;
    std::memset(&o, 0, sizeof o);
    const double nan = std::numeric_limits<double>::quiet_NaN();
    o.mode = 1;
    o.const_price = nan;
    // heston.cpp:10-24
    if (!(ot == 0 || ot == 1)) return o;
    if (!finite_(spot) || !finite_(strike) || !finite_(t) || !finite_(r) || !finite_(q) ||
        !finite_(v0) || !finite_(kappa) || !finite_(theta) || !finite_(sigma) || !finite_(rho))
        return o;
    if (spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0 || kappa <= 0.0 || theta < 0.0 ||
        sigma <= 0.0 || rho <= -1.0 || rho >= 1.0)
        return o;
    if (t <= 1e-12) {
        o.const_price = intrinsic_(spot, strike, ot);
        return o;
    }
    if (steps < 16 || limit <= 1e-6) return o;
    o.mode = 0;
    o.spot = spot;
    o.strike = strike;
    o.t = t;
    o.r = r;
    o.q = q;
    o.v0 = v0;
    o.kappa = kappa;
    o.theta = theta;
    o.sigma = sigma;
    o.rho = rho;
    o.limit = limit;
    o.option_type = ot;
    const int64_t panels = (static_cast<int64_t>(steps) + 63) / 64;  // no int32 overflow
    o.panels = static_cast<int32_t>(panels > 1 ? panels : 1);
    return o;
}

CfOption pack_cos_option(double spot, double strike, double t, double r, double q, double v0,
                         double kappa, double theta, double sigma, double rho, int32_t ot,
                         int32_t n_terms, double width) {
    CfOption o;
    std::memset(&o, 0, sizeof o);
    o.method = kCfMethodCos;
    o.mode = 1;
    o.const_price = std::numeric_limits<double>::quiet_NaN();
    // cos_method.cpp:38-48 (no range checks on kappa, theta, sigma, rho)
    if (!(ot == 0 || ot == 1)) return o;
    if (!finite_(spot) || !finite_(strike) || !finite_(t) || !finite_(r) || !finite_(q) ||
        !finite_(v0) || !finite_(kappa) || !finite_(theta) || !finite_(sigma) || !finite_(rho) ||
        !finite_(width))
        return o;
    if (spot <= 0.0 || strike <= 0.0 || t < 0.0 || v0 < 0.0) return o;
    if (t <= 1e-12) {
        o.const_price = intrinsic_(spot, strike, ot);
        return o;
    }
    if (n_terms < 8 || width <= 0.0) return o;
    // cos_method.cpp:50-55: truncation interval from max(v0, theta)
    const double eff_var = (v0 < theta) ? theta : v0;
    const double c1 = std::log(spot) + (r - q - 0.5 * eff_var) * t;
    const double c2 = eff_var * t;
    const double half = width * std::sqrt((c2 < 0.0) ? 0.0 : c2);
    const double a = c1 - half, b = c1 + half;
    if (!(b > a + 1e-12)) return o;  // cos_method.h:22
    o.mode = 0;
    o.spot = spot;
    o.strike = strike;
    o.t = t;
    o.r = r;
    o.q = q;
    o.v0 = v0;
    o.kappa = kappa;
    o.theta = theta;
    o.sigma = sigma;
    o.rho = rho;
    o.limit = a;
    o.hi = b;
    o.option_type = ot;
    o.panels = n_terms;
    return o;
}

cudaError_t launch_heston_cos(const CfOption* d_opts, int32_t n, double* d_out, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (cudaError_t e = injected_fault(kFaultLaunch)) return e;
    heston_cos_kernel<<<n, 128, 0, st>>>(d_opts, n, d_out);
    return cudaGetLastError();
}

cudaError_t launch_heston_cf(const CfOption* d_opts, int32_t n, double* d_out, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    {
        std::lock_guard<std::mutex> lk(g_cf_mu);
        if (!g_cf_ready[dev]) {
            double x[32], w[32];
            gl64(x, w);
            if ((e = cudaMemcpyToSymbol(c_gl_x, x, sizeof x)) != cudaSuccess) return e;
            if ((e = cudaMemcpyToSymbol(c_gl_w, w, sizeof w)) != cudaSuccess) return e;
            g_cf_ready[dev] = true;
        }
    }
    if (n <= 0) return cudaSuccess;
    if ((e = injected_fault(kFaultLaunch)) != cudaSuccess) return e;
    heston_cf_kernel<<<n, 128, 0, st>>>(d_opts, n, d_out);
    return cudaGetLastError();
}

namespace {

// Per-thread, per-device staging for the host-buffer entry points.
struct CfScratch {
    DevBuf d_opts, d_out;
    PinnedBuf h_opts, h_out;
    cudaStream_t st = nullptr;
    ~CfScratch() {
        d_opts.release();
        d_out.release();
        h_opts.release();
        h_out.release();
        if (st) cudaStreamDestroy(st);
    }
};

}  // namespace

cudaError_t heston_cf_price_host(const CfOption* h_opts, int32_t n, double* out) {
    NvtxRange range("qk.heston_cf");
    if (n <= 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    thread_local std::map<int, std::unique_ptr<CfScratch>> scratch;
    auto& sp = scratch[dev];
    if (!sp) sp.reset(new CfScratch());
    CfScratch& s = *sp;
    if (!s.st && (e = cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking)) != cudaSuccess) {
        s.st = nullptr;
        return e;
    }
    const size_t ob = sizeof(CfOption) * static_cast<size_t>(n);
    const size_t pb = sizeof(double) * static_cast<size_t>(n);
    if ((e = s.d_opts.ensure(ob)) != cudaSuccess) return e;
    if ((e = s.d_out.ensure(pb)) != cudaSuccess) return e;
    if ((e = s.h_opts.ensure(ob)) != cudaSuccess) return e;
    if ((e = s.h_out.ensure(pb)) != cudaSuccess) return e;
    std::memcpy(s.h_opts.p, h_opts, ob);
    if ((e = cudaMemcpyAsync(s.d_opts.p, s.h_opts.p, ob, cudaMemcpyHostToDevice, s.st)) != cudaSuccess)
        return e;
    e = h_opts[0].method == kCfMethodCos
            ? launch_heston_cos(static_cast<const CfOption*>(s.d_opts.p), n,
                                static_cast<double*>(s.d_out.p), s.st)
            : launch_heston_cf(static_cast<const CfOption*>(s.d_opts.p), n,
                               static_cast<double*>(s.d_out.p), s.st);
    if (e != cudaSuccess) return e;
    if ((e = injected_fault(kFaultCopy)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(s.h_out.p, s.d_out.p, pb, cudaMemcpyDeviceToHost, s.st)) != cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(s.st)) != cudaSuccess) return e;
    std::memcpy(out, s.h_out.p, pb);
    return cudaSuccess;
}

}  // namespace qkb
