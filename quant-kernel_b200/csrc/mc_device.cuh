// mc_device.cuh -- device building blocks of the Monte Carlo kernels.
//
// * Philox4x32-10 counter-based generator + Box-Muller, in registers.
// * Double-double (hi, lo) accumulators for compensated FP64 sums.
// * FP32 PTX approximations used on the hot path (MUFU unit).
//
// All kernels are compiled with --fmad=false: every fused multiply-add below
// is written explicitly, so a path's FP32 arithmetic is the same whatever the
// unrolling or launch shape, and results do not depend on the tile config.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "mc_types.h"

namespace qkb {

// ---------------------------------------------------------------------------
// FP32 approximations on the special-function unit (PTX ISA, sm_100a).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float ptx_lg2(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_sqrt(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_sin(float x) {
    float y;
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_cos(float x) {
    float y;
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// max that propagates NaN: the reference floors with std::max(s, 1e-12),
// which keeps a NaN s; fmaxf would replace it.
__device__ __forceinline__ float ptx_max_nan(float a, float b) {
    float y;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(y) : "f"(a), "f"(b));
    return y;
}
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Packed FP32 pairs (sm_100 f32x2 FMA / multiply / add: one instruction for
// both lanes, each lane rounded exactly as its scalar form), used where two
// units of a thread take the same operation: same bits as the scalar code,
// fewer issued instructions.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11).  Counter (c0, c1, 0, c3), key = seed.
// ---------------------------------------------------------------------------
struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                            uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint32_t lo0 = c0 * 0xD2511F53u;
        const uint32_t hi0 = __umulhi(c0, 0xD2511F53u);
        const uint32_t lo1 = c2 * 0xCD9E8D57u;
        const uint32_t hi1 = __umulhi(c2, 0xCD9E8D57u);
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return U4{c0, c1, c2, c3};
}

// Uniforms without an integer-to-float conversion: OR-ing k <= 23 bits b into
// the mantissa of 1.0f gives y = 1 + b 2^-k exactly in [1, 2), and y minus
// (1 - 2^-24) is exact (Sterbenz), so it equals (b + 1/2) 2^-23 bit for bit
// while staying off the conversion pipe.
__device__ __forceinline__ float unit_from_bits(uint32_t b23) {  // (b + 1/2) 2^-23
    return __uint_as_float(0x3F800000u | b23) - 0x1.fffffep-1f;   // y - (1 - 2^-24)
}

// FP64 Box-Muller from one Philox call (the terminal models, which the
// reference evaluates in FP64 end to end):  52-bit words
//   ub = x << 20 | y >> 12,  gb = z << 20 | w >> 12,
//   u = (ub + 1/2) 2^-52 in (0,1),  g = (gb + 1/2) 2^-51 - 1 in (-1,1),
//   za = sqrt(-2 ln u) cos(pi g),  zb = sqrt(-2 ln u) sin(pi g).
// Both are formed without an integer-to-double conversion: OR-ing the 52 bits
// into the mantissa of 1.0 (of 2.0) gives y = 1 + ub 2^-52 (y = 2 + gb 2^-51)
// exactly, and y - (1 - 2^-53) (y - (3 - 2^-52)) is exact (Sterbenz).
__device__ __forceinline__ void box_muller_f64(U4 x, double& za, double& zb) {
    const unsigned long long ub = ((unsigned long long)x.x << 20) | (x.y >> 12);
    const unsigned long long gb = ((unsigned long long)x.z << 20) | (x.w >> 12);
    const double u = __longlong_as_double((long long)(0x3FF0000000000000ull | ub)) -
                     0x1.fffffffffffffp-1;
    const double g = __longlong_as_double((long long)(0x4000000000000000ull | gb)) -
                     (3.0 - 0x1p-52);
    const double rad = sqrt(-2.0 * log(u));
    double sn, cs;
    sincospi(g, &sn, &cs);
    za = rad * cs;
    zb = rad * sn;
}

// Four FP64 normals of quad `unit`: counter (unit, 0, 0, c3) gives normals 0
// and 1, counter (unit, 1, 0, c3) normals 2 and 3.
__device__ __forceinline__ void normals4_f64(uint32_t unit, uint32_t c3, uint32_t k0, uint32_t k1,
                                             double z[4]) {
    box_muller_f64(philox4x32_10(unit, 0u, 0u, c3, k0, k1), z[0], z[1]);
    box_muller_f64(philox4x32_10(unit, 1u, 0u, c3, k0, k1), z[2], z[3]);
}

// sqrt(2 ln 2): sqrt(-2 ln u) = kBmRadius * sqrt(-log2 u).
constexpr float kBmRadius = 1.17741002251547469101f;
constexpr double kBmRadiusD = 1.17741002251547469101;
constexpr float kBmRadius2 = 1.38629436111989061883f;  // kBmRadius^2 = 2 ln 2

// Box-Muller from a 23-bit radius word and a K-bit angle word, in parts:
//   u = (ub + 1/2) 2^-23,  g = (gb + 1/2) 2^-(K-1) - 1,
//   w = -log2 u,  c = cos(pi g),  s = sin(pi g),
// so that the normals are kBmRadius sqrt(w) c and kBmRadius sqrt(w) s.  With
// y = 1 + gb 2^-K (gb OR-ed into the mantissa of 1.0f), pi g =
// 2 pi y - pi (3 - 2^-K): one FMA from y to the angle.
template <int K>
__device__ __forceinline__ void box_muller_parts(uint32_t ub, uint32_t gb, float& w, float& c,
                                                 float& s) {
    constexpr float kTwoPi = 6.28318530717958647692f;
    constexpr float kOff = (float)(3.14159265358979323846 * (3.0 - 1.0 / (double)(1u << K)));
    const float u = unit_from_bits(ub);
    const float y = __uint_as_float(0x3F800000u | (gb << (23 - K)));
    w = -ptx_lg2(u);
    const float ang = fma_rn(y, kTwoPi, -kOff);
    c = ptx_cos(ang);
    s = ptx_sin(ang);
}

// box_muller_parts for two units at once (lane 0: ub0, gb0; lane 1: ub1,
// gb1), the uniform's subtraction and the angle's FMA as packed pairs.
template <int K>
__device__ __forceinline__ void box_muller_parts2(uint32_t ub0, uint32_t gb0, uint32_t ub1,
                                                  uint32_t gb1, float2& w, float2& c, float2& s) {
    constexpr float kTwoPi = 6.28318530717958647692f;
    constexpr float kOff = (float)(3.14159265358979323846 * (3.0 - 1.0 / (double)(1u << K)));
    const float2 u = add2(f2(__uint_as_float(0x3F800000u | ub0), __uint_as_float(0x3F800000u | ub1)),
                          f2(-0x1.fffffep-1f));
    const float2 y = f2(__uint_as_float(0x3F800000u | (gb0 << (23 - K))),
                        __uint_as_float(0x3F800000u | (gb1 << (23 - K))));
    w = f2(-ptx_lg2(u.x), -ptx_lg2(u.y));
    const float2 ang = fma2(y, f2(kTwoPi), f2(-kOff));
    c = f2(ptx_cos(ang.x), ptx_cos(ang.y));
    s = f2(ptx_sin(ang.x), ptx_sin(ang.y));
}

// The normals of box_muller_parts divided by kBmRadius (the callers fold that
// factor into their step constants, which saves a multiply per pair):
//   za = sqrt(w) c,  zb = sqrt(w) s.
template <int K>
__device__ __forceinline__ void box_muller_bits(uint32_t ub, uint32_t gb, float& za, float& zb) {
    float w, c, s;
    box_muller_parts<K>(ub, gb, w, c, s);
    const float rad = ptx_sqrt(w);
    za = rad * c;
    zb = rad * s;
}

// Six normals from one Philox call: three Box-Muller pairs, each with a
// 23-bit radius (the top 23 bits of x, y, z) and an angle of 16, 16 and 18
// bits (the low and high halves of w; the low 9 bits of x and of y).  Every
// output bit of the call is used once.  pair(p) computes pair p on demand, so
// only the four words stay live across the three steps they feed.  pair()
// gives the normals divided by kBmRadius (box_muller_bits); parts() gives
// (w, c, s) of box_muller_parts, for a caller that folds sqrt(w) into a square
// root of its own (sqrt(v) sqrt(w) = sqrt(v w)).
struct Philox6 {
    U4 x;
    __device__ __forceinline__ void pair(int p, float& za, float& zb) const {
        if (p == 0)
            box_muller_bits<16>(x.x >> 9, x.w & 0xFFFFu, za, zb);
        else if (p == 1)
            box_muller_bits<16>(x.y >> 9, x.w >> 16, za, zb);
        else
            box_muller_bits<18>(x.z >> 9, (x.x & 0x1FFu) | ((x.y & 0x1FFu) << 9), za, zb);
    }
    __device__ __forceinline__ void parts(int p, float& w, float& c, float& s) const {
        if (p == 0)
            box_muller_parts<16>(x.x >> 9, x.w & 0xFFFFu, w, c, s);
        else if (p == 1)
            box_muller_parts<16>(x.y >> 9, x.w >> 16, w, c, s);
        else
            box_muller_parts<18>(x.z >> 9, (x.x & 0x1FFu) | ((x.y & 0x1FFu) << 9), w, c, s);
    }
};

// parts() of pair p for two units' calls a (lane 0) and b (lane 1).
__device__ __forceinline__ void philox6_parts2(const Philox6& a, const Philox6& b, int p, float2& w,
                                               float2& c, float2& s) {
    if (p == 0)
        box_muller_parts2<16>(a.x.x >> 9, a.x.w & 0xFFFFu, b.x.x >> 9, b.x.w & 0xFFFFu, w, c, s);
    else if (p == 1)
        box_muller_parts2<16>(a.x.y >> 9, a.x.w >> 16, b.x.y >> 9, b.x.w >> 16, w, c, s);
    else
        box_muller_parts2<18>(a.x.z >> 9, (a.x.x & 0x1FFu) | ((a.x.y & 0x1FFu) << 9), b.x.z >> 9,
                              (b.x.x & 0x1FFu) | ((b.x.y & 0x1FFu) << 9), w, c, s);
}

// pair() of pair p for two units' calls a (lane 0) and b (lane 1).
__device__ __forceinline__ void philox6_pair2(const Philox6& a, const Philox6& b, int p, float2& za,
                                              float2& zb) {
    float2 w, c, s;
    philox6_parts2(a, b, p, w, c, s);
    const float2 rad = f2(ptx_sqrt(w.x), ptx_sqrt(w.y));
    za = mul2(rad, c);
    zb = mul2(rad, s);
}

// ---------------------------------------------------------------------------
// Double-double accumulation (Knuth TwoSum).  A non-finite sum drops its error
// term so that inf stays inf instead of turning into NaN.
// ---------------------------------------------------------------------------
struct DD {
    double hi, lo;
};

__device__ __forceinline__ DD dd_add(DD a, double b) {
    const double s = __dadd_rn(a.hi, b);
    const double bb = __dsub_rn(s, a.hi);
    double err = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b, bb));
    if (!isfinite(s)) err = 0.0;
    return DD{s, __dadd_rn(a.lo, err)};
}

__device__ __forceinline__ DD dd_merge(DD a, DD b) {
    DD r = dd_add(a, b.hi);
    r.lo = __dadd_rn(r.lo, b.lo);
    return r;
}

__device__ __forceinline__ DD dd_shfl_down(DD v, int offset) {
    return DD{__shfl_down_sync(0xffffffffu, v.hi, offset), __shfl_down_sync(0xffffffffu, v.lo, offset)};
}

__device__ __forceinline__ double payoff(double s_t, double strike, int32_t option_type) {
    // option_util.h:33-38: max(0, S - K) / max(0, K - S).  fmax(NaN, 0) = 0
    // matches std::max(0.0, NaN) = 0.0.
    return option_type == 0 ? fmax(__dsub_rn(s_t, strike), 0.0) : fmax(__dsub_rn(strike, s_t), 0.0);
}

}  // namespace qkb
