// pipe_probe.cu -- measured per-SM instruction throughput of the pipes the
// Monte Carlo kernels are bound by (the denominators of their rooflines):
// the special-function unit (MUFU), the FP32 FMA pipe (scalar and packed
// f32x2), the FP64 pipe, and a MUFU : FP32 mix at the Heston step's ratio.
//
// Each thread runs CH independent dependency chains of one operation for
// kIters iterations; every CTA records its SM id and its start and end
// clock64() (a per-SM counter), the host takes, per SM, the span from the
// earliest start to the latest end of the CTAs it ran, and the rate is the
// SM's lane-operations over that span.  The grid is kCtasPerSm CTAs of
// kProbeThreads per SM, all co-resident (tiny register and no shared-memory
// use), so the spans cover concurrent work.  No input is read; each thread
// writes one float (so the chains are not optimised away) and each CTA one
// record.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "qk_diag.h"

namespace qkb {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kCtasPerSm = 4;
constexpr int CH = 8;
constexpr int kIters = 2048;
constexpr int kMaxSmId = 1024;  // bound on %smid, whose range may have gaps

struct CtaSpan {
    long long start, end;
    int smid, pad;
};

__device__ __forceinline__ int sm_id() {
    int id;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(id));
    return id;
}

template <int KIND>
__device__ __forceinline__ void step(float (&x)[CH], double (&d)[CH], float2 (&p)[CH], uint32_t (&u)[CH]) {
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        if (KIND == QK_PROBE_MUFU) asm volatile("sin.approx.ftz.f32 %0, %0;" : "+f"(x[c]));
        if (KIND == QK_PROBE_FFMA) asm volatile("fma.rn.f32 %0, %0, %0, 0f3F000000;" : "+f"(x[c]));
        if (KIND == QK_PROBE_FFMA2) p[c] = __ffma2_rn(p[c], p[c], make_float2(0.5f, 0.5f));
        if (KIND == QK_PROBE_DFMA) asm volatile("fma.rn.f64 %0, %0, %0, 0d3FE0000000000000;" : "+d"(d[c]));
        if (KIND == QK_PROBE_MIX) {
            // per chain element one MUFU op, one packed FP32 FMA and about
            // four integer operations (shift, 3-input logic, add, multiply):
            // the Heston step's mix of ~6-7 other instructions per MUFU op
            asm volatile("sqrt.approx.ftz.f32 %0, %0;" : "+f"(x[c]));
            p[c] = __ffma2_rn(p[c], make_float2(0.999f, 0.998f), make_float2(1e-3f, 2e-3f));
            u[c] = ((u[c] ^ (u[c] >> 7)) + 0x9E3779B9u) * 0xD2511F53u;
        }
    }
}

template <int KIND>
__global__ void __launch_bounds__(kProbeThreads) probe_kernel(float* __restrict__ sink, CtaSpan* __restrict__ spans) {
    float x[CH];
    double d[CH];
    float2 p[CH];
    uint32_t u[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        u[c] = threadIdx.x * 8u + (uint32_t)c;
        x[c] = 0.25f + 0.001f * (float)(threadIdx.x + c);
        d[c] = 0.25 + 0.001 * (double)(threadIdx.x + c);
        p[c] = make_float2(x[c], 0.5f * x[c]);
    }
    __syncthreads();
    const long long t0 = clock64();
    for (int i = 0; i < kIters; ++i) step<KIND>(x, d, p, u);
    __syncthreads();
    const long long t1 = clock64();
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < CH; ++c) s += x[c] + (float)d[c] + p[c].x + p[c].y + (float)(u[c] & 1u);
    sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
    if (threadIdx.x == 0) spans[blockIdx.x] = CtaSpan{t0, t1, sm_id(), 0};
}

// lane-operations of the probed kind per thread
double lane_ops_per_thread(int kind) {
    const double e = (double)CH * kIters;
    switch (kind) {
        case QK_PROBE_FFMA2: return 2.0 * e;
        case QK_PROBE_MIX: return e;  // the MUFU ops (the FMAs are the filler)
        default: return e;
    }
}

}  // namespace
}  // namespace qkb

extern "C" int32_t qk_b200_pipe_probe(int32_t device, int32_t kind, double* lane_ops_per_sm_clock) {
    using namespace qkb;
    if (lane_ops_per_sm_clock == nullptr) return QK_PROBE_ERR;
    *lane_ops_per_sm_clock = 0.0;
    if (kind < QK_PROBE_MUFU || kind > QK_PROBE_MIX) return QK_PROBE_ERR;
    if (cudaSetDevice(device) != cudaSuccess) return QK_PROBE_ERR;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
        return QK_PROBE_ERR;
    const int grid = sms * kCtasPerSm;
    float* sink = nullptr;
    CtaSpan* spans = nullptr;
    if (cudaMalloc(&sink, sizeof(float) * (size_t)grid * kProbeThreads) != cudaSuccess) return QK_PROBE_ERR;
    if (cudaMalloc(&spans, sizeof(CtaSpan) * (size_t)grid) != cudaSuccess) {
        cudaFree(sink);
        return QK_PROBE_ERR;
    }
    std::vector<CtaSpan> h((size_t)grid);
    cudaError_t e = cudaSuccess;
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // the first run warms up
        switch (kind) {
            case QK_PROBE_MUFU: probe_kernel<QK_PROBE_MUFU><<<grid, kProbeThreads>>>(sink, spans); break;
            case QK_PROBE_FFMA: probe_kernel<QK_PROBE_FFMA><<<grid, kProbeThreads>>>(sink, spans); break;
            case QK_PROBE_FFMA2: probe_kernel<QK_PROBE_FFMA2><<<grid, kProbeThreads>>>(sink, spans); break;
            case QK_PROBE_DFMA: probe_kernel<QK_PROBE_DFMA><<<grid, kProbeThreads>>>(sink, spans); break;
            default: probe_kernel<QK_PROBE_MIX><<<grid, kProbeThreads>>>(sink, spans); break;
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(h.data(), spans, sizeof(CtaSpan) * (size_t)grid, cudaMemcpyDeviceToHost);
    cudaFree(sink);
    cudaFree(spans);
    if (e != cudaSuccess) return QK_PROBE_ERR;
    // per SM: span of its CTAs, lane-operations of its CTAs; median rate
    std::vector<long long> lo((size_t)kMaxSmId, -1), hi((size_t)kMaxSmId, -1);
    std::vector<int> ctas((size_t)kMaxSmId, 0);
    for (const CtaSpan& s : h) {
        if (s.smid < 0 || s.smid >= kMaxSmId) return QK_PROBE_ERR;
        const size_t i = (size_t)s.smid;
        lo[i] = lo[i] < 0 ? s.start : std::min(lo[i], s.start);
        hi[i] = std::max(hi[i], s.end);
        ++ctas[i];
    }
    std::vector<double> rate;
    const double per_cta = lane_ops_per_thread(kind) * kProbeThreads;
    for (int i = 0; i < kMaxSmId; ++i)
        if (ctas[(size_t)i] > 0 && hi[(size_t)i] > lo[(size_t)i])
            rate.push_back(per_cta * ctas[(size_t)i] / (double)(hi[(size_t)i] - lo[(size_t)i]));
    if (rate.empty()) return QK_PROBE_ERR;
    std::sort(rate.begin(), rate.end());
    *lane_ops_per_sm_clock = rate[rate.size() / 2];
    return 0;
}
