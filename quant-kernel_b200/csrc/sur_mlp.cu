// sur_mlp.cu -- training and inference of the Heston price surrogate.
//
// One optimiser step on a minibatch of B rows (B % 128 == 0) is 14 launches,
// captured once into a CUDA graph and replayed:
//   gather      minibatch rows (a permutation drawn per epoch) -> X, X^T, target
//   fwd1/fwd2   tcgen05 GEMM, epilogue z = acc + b, h = silu(z) -> Z, H, H^T
//   fwd3        tcgen05 GEMM, epilogue: y = silu(acc + b3) . w4 + b4,
//               dy = 2 (y - t) / B, dZ3 = dy w4 silu'(z3) -> dZ3, dZ3^T, H3^T
//   loss        db4 = sum dy, loss = mean (y - t)^2          (fixed order)
//   rowsum      db3 = sum_b dZ3^T, dw4 = H3^T . dy           (fixed order)
//   bwd2/bwd1   tcgen05 GEMM dH = dZ . W, epilogue dZ = dH silu'(z) -> dZ, dZ^T
//   dW3/dW2/dW1 tcgen05 GEMM dZ^T . H over the batch, split-K slabs
//   rowsum      db2, db1
//   adam        sum slabs (fixed order), Adam with cosine-decayed lr, write the
//               FP32 master, and the bf16 weights and transposed weights the
//               next step's GEMMs read
//   advance     step += 1
// All reductions run in a fixed order: training is deterministic.
#include "sur_mlp.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "mc_device.cuh"
#include "sur_gemm.cuh"

namespace qkb {

namespace {

constexpr int kPredChunk = 65536;

#define QK_TRY(x)                                \
    do {                                         \
        cudaError_t e_ = (x);                    \
        if (e_ != cudaSuccess) return e_;        \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    return cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(count, 1));
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// He-normal weights from the Philox/Box-Muller stream (seed, parameter index),
// zero biases, zero layer-1 padding columns, and a zero output layer: the
// untrained model is its base, and the first steps grow the residual from 0.
__global__ void init_params_kernel(float* P, uint64_t seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= SurLayout::total) return;
    double z[4];
    normals4_f64(static_cast<uint32_t>(i), 7u, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), z);
    const float z0 = static_cast<float>(z[0]);
    float v = 0.0f;
    if (i < SurLayout::b1) {
        const int col = (i - SurLayout::W1) % kSurInPad;
        v = col < kSurIn ? z0 * sqrtf(2.0f / kSurIn) : 0.0f;
    } else if ((i >= SurLayout::W2 && i < SurLayout::b2) || (i >= SurLayout::W3 && i < SurLayout::b3)) {
        v = z0 * sqrtf(2.0f / kSurHid);
    }
    P[i] = v;
}

__global__ void gather_kernel(const __nv_bfloat16* __restrict__ xall, const float* __restrict__ tall,
                              const int32_t* __restrict__ perm, const SurState* __restrict__ st,
                              __nv_bfloat16* __restrict__ xb, __nv_bfloat16* __restrict__ xtb,
                              float* __restrict__ tb) {
    const int B = st->batch;
    const int i = blockIdx.x;  // row in the batch
    const int c = threadIdx.x; // feature column, 0..63
    const int64_t b0 = static_cast<int64_t>(st->step % st->steps_per_epoch) * B;
    const int64_t src = perm[b0 + i];
    const __nv_bfloat16 v = xall[src * kSurInPad + c];
    xb[static_cast<int64_t>(i) * kSurInPad + c] = v;
    xtb[static_cast<int64_t>(c) * B + i] = v;
    if (c == 0) tb[i] = tall[src];
}

// The residual's base: the Black-Scholes call / S at the Heston model's mean
// variance over [0, T],
//   vbar = theta + (v0 - theta) (1 - exp(-kappa T)) / (kappa T)
// (the expectation of (1/T) int_0^T v_t dt), from f = (S/K, T, r, q, v0,
// kappa, theta, ...).  The host and the device evaluate the same FP64
// expression with their own exp/log/erfc; rounded to FP32 the two agree.
__host__ __device__ inline double sur_base(const double* f) {
    const double m = f[0], T = f[1], r = f[2], q = f[3], v0 = f[4], kappa = f[5], theta = f[6];
    const double x = kappa * T;
    const double w = (x > 1e-12) ? -expm1(-x) / x : 1.0;
    double vbar = theta + (v0 - theta) * w;
    if (!(vbar > 0.0)) vbar = 0.0;
    const double sd = sqrt(vbar * T);
    const double dq = exp(-q * T);
    const double dk = exp(-r * T) / m;
    if (!(sd > 1e-12)) {  // no variance left: the discounted forward payoff
        const double fwd = dq - dk;
        return fwd > 0.0 ? fwd : 0.0;
    }
    const double inv_sqrt2 = 0.70710678118654752440;
    const double d1 = (log(m) + (r - q) * T) / sd + 0.5 * sd;
    return dq * (0.5 * erfc(-d1 * inv_sqrt2)) - dk * (0.5 * erfc(-(d1 - sd) * inv_sqrt2));
}

// The normalised coordinate of feature value x in [lo, hi], as bf16 bits.
__host__ __device__ inline unsigned short sur_norm_bits(double x, double lo, double hi) {
    const double u = hi > lo ? 2.0 * (x - lo) / (hi - lo) - 1.0 : 0.0;
    return __bfloat16_as_ushort(__float2bfloat16_rn(static_cast<float>(u)));
}

// Device features: one thread per row computes its nine normalised values
// and base; the block then writes its 256 rows of 128 bytes as consecutive
// 16-byte chunks (columns 9..63 are zero).
constexpr int kFeatRows = 256;
__global__ void __launch_bounds__(kFeatRows)
features_kernel(const double* __restrict__ f, int64_t n, SurBox box, int32_t kind,
                __nv_bfloat16* __restrict__ rows, float* __restrict__ base) {
    __shared__ uint4 stage[kFeatRows][2];
    const int t = threadIdx.x;
    const int64_t row0 = static_cast<int64_t>(blockIdx.x) * kFeatRows;
    const int64_t i = row0 + t;
    unsigned short b[16] = {};
    if (i < n) {
        double x[kSurIn];
#pragma unroll
        for (int c = 0; c < kSurIn; ++c) x[c] = f[i * kSurIn + c];
#pragma unroll
        for (int c = 0; c < kSurIn; ++c) b[c] = sur_norm_bits(x[c], box.lo[c], box.hi[c]);
        if (base) base[i] = kind == kSurBaseBsmMeanVar ? static_cast<float>(sur_base(x)) : 0.0f;
    }
    uint4 c0, c1;
    c0.x = b[0] | (static_cast<uint32_t>(b[1]) << 16);
    c0.y = b[2] | (static_cast<uint32_t>(b[3]) << 16);
    c0.z = b[4] | (static_cast<uint32_t>(b[5]) << 16);
    c0.w = b[6] | (static_cast<uint32_t>(b[7]) << 16);
    c1.x = b[8];
    c1.y = c1.z = c1.w = 0u;
    stage[t][0] = c0;
    stage[t][1] = c1;
    __syncthreads();
    uint4* out = reinterpret_cast<uint4*>(rows);
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int k = 0; k < 8; ++k) {  // 256 rows x 8 chunks, 8 per thread
        const int idx = k * kFeatRows + t;
        const int r = idx >> 3, c = idx & 7;
        const int64_t row = row0 + r;
        if (row < n) out[row * 8 + c] = c < 2 ? stage[r][c] : zero;
    }
}

// out[r] = sum_j X[r][j] * (w ? w[j] : 1), one warp per row, fixed order.
__global__ void rowsum_kernel(const __nv_bfloat16* __restrict__ X, int rows, int L,
                              const float* __restrict__ w, float* __restrict__ out) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= rows) return;
    float acc = 0.0f;
    const __nv_bfloat16* x = X + static_cast<int64_t>(row) * L;
    for (int j = lane; j < L; j += 32) acc = fmaf(__bfloat162float(x[j]), w ? w[j] : 1.0f, acc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) out[row] = acc;
}

// db4 = sum dy; loss = mean (y - t)^2, written to loss_hist[step].
__global__ void loss_kernel(const float* __restrict__ y, const float* __restrict__ t,
                            const float* __restrict__ dy, const SurState* __restrict__ st,
                            float* __restrict__ db4, float* __restrict__ loss_hist, int loss_cap) {
    __shared__ float s1[256], s2[256];
    const int B = st->batch;
    float a = 0.0f, b = 0.0f;
    for (int i = threadIdx.x; i < B; i += 256) {
        a += dy[i];
        const float d = y[i] - t[i];
        b = fmaf(d, d, b);
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            s1[threadIdx.x] += s1[threadIdx.x + off];
            s2[threadIdx.x] += s2[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *db4 = s1[0];
        const int k = st->step;
        if (k >= 0 && k < loss_cap) loss_hist[k] = s2[0] / static_cast<float>(B);
    }
}

struct AdamSeg {
    int off, n;               // range in the flat layout
    const float* g;           // gradient (or split-K slabs); null: no gradient
    int splits;
    int64_t split_stride;
    __nv_bfloat16* wb;        // bf16 copy, same layout (optional)
    __nv_bfloat16* wtb;       // bf16 transpose (optional)
    int rows, cols;
};

struct AdamArgs {
    AdamSeg seg[8];
    int nseg;
    int total;
    float* P;
    float* M;
    float* V;
    float* G;
    int update;
    const SurState* st;
};

__global__ void adam_kernel(const AdamArgs a) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.total) return;
    int s = 0;
    while (s + 1 < a.nseg && idx >= a.seg[s + 1].off) ++s;
    const AdamSeg& sg = a.seg[s];
    const int local = idx - sg.off;
    if (local >= sg.n) return;
    float p = a.P[idx];
    if (sg.g != nullptr) {
        float g = 0.0f;
        for (int k = 0; k < sg.splits; ++k) g += sg.g[k * sg.split_stride + local];
        a.G[idx] = g;
        if (a.update) {
            const SurState& st = *a.st;
            const int t = st.step + 1;
            const float span = static_cast<float>(max(st.total_steps - st.step_begin, 1));
            const float prog = fminf(static_cast<float>(st.step - st.step_begin) / span, 1.0f);
            const float lr = st.lr0 * 0.5f * (1.0f + cosf(3.14159265358979f * prog));
            const float m = st.beta1 * a.M[idx] + (1.0f - st.beta1) * g;
            const float v = st.beta2 * a.V[idx] + (1.0f - st.beta2) * g * g;
            a.M[idx] = m;
            a.V[idx] = v;
            const float mh = m / (1.0f - powf(st.beta1, static_cast<float>(t)));
            const float vh = v / (1.0f - powf(st.beta2, static_cast<float>(t)));
            p -= lr * mh / (sqrtf(vh) + st.eps);
            a.P[idx] = p;
        }
    }
    const __nv_bfloat16 pb = __float2bfloat16_rn(p);
    if (sg.wb) sg.wb[local] = pb;
    if (sg.wtb) {
        const int r = local / sg.cols, c = local % sg.cols;
        sg.wtb[static_cast<int64_t>(c) * sg.rows + r] = pb;
    }
}

__global__ void advance_kernel(SurState* st) { st->step += 1; }

bool tmap(CUtensorMap* m, const void* base, int64_t rows, int64_t cols, int box_rows) {
    return make_tmap_bf16(m, base, static_cast<uint64_t>(rows), static_cast<uint64_t>(cols),
                          static_cast<uint32_t>(box_rows));
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (dev >= 0 && prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

// ----------------------------------------------------------------------------
SurModel::~SurModel() {
    if (device_ < 0) return;
    DeviceGuard g(device_);
    if (step_graph_) cudaGraphExecDestroy(step_graph_);
    float* fl[] = {P_, M_, V_, G_, Tall_, Tb_, y_, dy_, dW1p_, dW2p_, dW3p_, db1_, db2_, db3_, dw4_, db4_, loss_hist_, Py_, Pbase_};
    for (float* p : fl)
        if (p) cudaFree(p);
    __nv_bfloat16* bl[] = {W1b_, W2b_, W3b_, W2Tb_, W3Tb_, Xall_, Xb_, XTb_, Z1_, H1_, H1T_, Z2_, H2_, H2T_,
                           dZ3_, dZ3T_, H3T_, dZ2_, dZ2T_, dZ1_, dZ1T_, PX_, PH1_, PH2_};
    for (__nv_bfloat16* p : bl)
        if (p) cudaFree(p);
    if (perm_) cudaFree(perm_);
    if (state_) cudaFree(state_);
    for (cudaEvent_t& e : ev_)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t& a : aux_)
        if (a) cudaStreamDestroy(a);
    if (stream_) cudaStreamDestroy(stream_);
}

cudaError_t SurModel::init(uint64_t seed, const SurBox& box) {
    QK_TRY(cudaGetDevice(&device_));
    box_ = box;
    QK_TRY(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (cudaStream_t& a : aux_) QK_TRY(cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking));
    for (cudaEvent_t& e : ev_) QK_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    QK_TRY(dalloc(&P_, SurLayout::total));
    QK_TRY(dalloc(&M_, SurLayout::total));
    QK_TRY(dalloc(&V_, SurLayout::total));
    QK_TRY(dalloc(&G_, SurLayout::total));
    QK_TRY(dalloc(&W1b_, kSurHid * kSurInPad));
    QK_TRY(dalloc(&W2b_, kSurHid * kSurHid));
    QK_TRY(dalloc(&W3b_, kSurHid * kSurHid));
    QK_TRY(dalloc(&W2Tb_, kSurHid * kSurHid));
    QK_TRY(dalloc(&W3Tb_, kSurHid * kSurHid));
    QK_TRY(dalloc(&state_, 1));
    SurState s{};
    s.beta1 = 0.9f;
    s.beta2 = 0.999f;
    s.eps = 1e-8f;
    s.lr0 = 1e-3f;
    s.steps_per_epoch = 1;
    s.total_steps = 1;
    QK_TRY(cudaMemcpyAsync(state_, &s, sizeof s, cudaMemcpyHostToDevice, stream_));
    init_params_kernel<<<(SurLayout::total + 255) / 256, 256, 0, stream_>>>(P_, seed);
    QK_TRY(cudaGetLastError());
    QK_TRY(cudaMemsetAsync(M_, 0, sizeof(float) * SurLayout::total, stream_));
    QK_TRY(cudaMemsetAsync(V_, 0, sizeof(float) * SurLayout::total, stream_));
    QK_TRY(refresh_bf16(stream_));
    return cudaStreamSynchronize(stream_);
}

void SurModel::normalise(const double* f, int64_t n, __nv_bfloat16* out) const {
    for (int64_t i = 0; i < n; ++i) {
        __nv_bfloat16* row = out + i * kSurInPad;
        for (int c = 0; c < kSurInPad; ++c) row[c] = __float2bfloat16_rn(0.0f);
        for (int c = 0; c < kSurIn; ++c)
            row[c] = __ushort_as_bfloat16(sur_norm_bits(f[i * kSurIn + c], box_.lo[c], box_.hi[c]));
    }
}

void SurModel::base_host(const double* f, int64_t n, float* out) const {
    for (int64_t i = 0; i < n; ++i)
        out[i] = base_kind_ == kSurBaseBsmMeanVar ? static_cast<float>(sur_base(f + i * kSurIn)) : 0.0f;
}

cudaError_t SurModel::features_device(const double* f, int64_t n, __nv_bfloat16* rows, float* base,
                                      cudaStream_t st) {
    DeviceGuard g(device_);
    if (n <= 0 || (reinterpret_cast<uintptr_t>(rows) & 15u) != 0 ||
        (reinterpret_cast<uintptr_t>(f) & 7u) != 0 || (reinterpret_cast<uintptr_t>(base) & 3u) != 0)
        return cudaErrorInvalidValue;
    const int64_t blocks = (n + kFeatRows - 1) / kFeatRows;
    if (blocks > 0x7fffffff) return cudaErrorInvalidValue;
    features_kernel<<<static_cast<unsigned>(blocks), kFeatRows, 0, st ? st : stream_>>>(
        f, n, box_, base_kind_, rows, base);
    return cudaGetLastError();
}

bool SurModel::in_box(const double* f) const {
    for (int c = 0; c < kSurIn; ++c) {
        if (!(f[c] >= box_.lo[c] && f[c] <= box_.hi[c])) return false;
    }
    return true;
}

cudaError_t SurModel::refresh_bf16(cudaStream_t st) {
    AdamArgs a{};
    const int hid2 = kSurHid * kSurHid;
    a.seg[0] = AdamSeg{SurLayout::W1, kSurHid * kSurInPad, nullptr, 0, 0, W1b_, nullptr, kSurHid, kSurInPad};
    a.seg[1] = AdamSeg{SurLayout::W2, hid2, nullptr, 0, 0, W2b_, W2Tb_, kSurHid, kSurHid};
    a.seg[2] = AdamSeg{SurLayout::W3, hid2, nullptr, 0, 0, W3b_, W3Tb_, kSurHid, kSurHid};
    a.nseg = 3;
    a.total = SurLayout::b3;
    a.P = P_;
    a.M = M_;
    a.V = V_;
    a.G = G_;
    a.update = 0;
    a.st = state_;
    // segments must be ordered and contiguous for the lookup: W1 | b1 gap | W2 ...
    // (indices in gaps find the previous segment and return at local >= n)
    adam_kernel<<<(a.total + 255) / 256, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t SurModel::set_dataset(const double* features, const double* target, int64_t n) {
    DeviceGuard g(device_);
    if (step_graph_) {
        cudaGraphExecDestroy(step_graph_);
        step_graph_ = nullptr;
    }
    std::vector<__nv_bfloat16> rows(static_cast<size_t>(n) * kSurInPad);
    normalise(features, n, rows.data());
    // the network learns target - base
    std::vector<float> t(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        const double b = base_kind_ == kSurBaseBsmMeanVar ? sur_base(features + i * kSurIn) : 0.0;
        t[i] = static_cast<float>(target[i] - b);
    }
    QK_TRY(dalloc(&Xall_, static_cast<size_t>(n) * kSurInPad));
    QK_TRY(dalloc(&Tall_, static_cast<size_t>(n)));
    QK_TRY(dalloc(&perm_, static_cast<size_t>(n)));
    QK_TRY(cudaMemcpy(Xall_, rows.data(), rows.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    QK_TRY(cudaMemcpy(Tall_, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<int32_t> id(static_cast<size_t>(n));
    std::iota(id.begin(), id.end(), 0);
    QK_TRY(cudaMemcpy(perm_, id.data(), id.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    n_data_ = n;
    return cudaSuccess;
}

cudaError_t SurModel::ensure_batch_buffers(int B) {
    if (B == batch_) return cudaSuccess;
    if (step_graph_) {
        cudaGraphExecDestroy(step_graph_);
        step_graph_ = nullptr;
    }
    const size_t BH = static_cast<size_t>(B) * kSurHid;
    const int S = B / 128;
    QK_TRY(dalloc(&Xb_, static_cast<size_t>(B) * kSurInPad));
    QK_TRY(dalloc(&XTb_, static_cast<size_t>(B) * kSurInPad));
    QK_TRY(dalloc(&Tb_, B));
    __nv_bfloat16** act[] = {&Z1_, &H1_, &H1T_, &Z2_, &H2_, &H2T_, &dZ3_, &dZ3T_, &H3T_, &dZ2_, &dZ2T_, &dZ1_, &dZ1T_};
    for (auto p : act) QK_TRY(dalloc(p, BH));
    QK_TRY(dalloc(&y_, B));
    QK_TRY(dalloc(&dy_, B));
    QK_TRY(dalloc(&dW1p_, static_cast<size_t>(S) * kSurHid * kSurInPad));
    QK_TRY(dalloc(&dW2p_, static_cast<size_t>(S) * kSurHid * kSurHid));
    QK_TRY(dalloc(&dW3p_, static_cast<size_t>(S) * kSurHid * kSurHid));
    float** vec[] = {&db1_, &db2_, &db3_, &dw4_};
    for (auto p : vec) QK_TRY(dalloc(p, kSurHid));
    QK_TRY(dalloc(&db4_, 4));
    batch_ = B;
    return cudaSuccess;
}

cudaError_t SurModel::run_step(cudaStream_t st, bool update) {
    const int B = batch_;
    const int S = B / 128;
    CUtensorMap tXb, tW1, tH1, tW2, tH2, tW3, tdZ3, tW3T, tdZ3T, tH2T, tdZ2, tW2T, tdZ2T, tH1T, tdZ1T, tXTb;
    bool ok = tmap(&tXb, Xb_, B, kSurInPad, 128) && tmap(&tW1, W1b_, kSurHid, kSurInPad, 128) &&
              tmap(&tH1, H1_, B, kSurHid, 128) && tmap(&tW2, W2b_, kSurHid, kSurHid, 128) &&
              tmap(&tH2, H2_, B, kSurHid, 128) && tmap(&tW3, W3b_, kSurHid, kSurHid, 256) &&
              tmap(&tdZ3, dZ3_, B, kSurHid, 128) && tmap(&tW3T, W3Tb_, kSurHid, kSurHid, 128) &&
              tmap(&tdZ3T, dZ3T_, kSurHid, B, 128) && tmap(&tH2T, H2T_, kSurHid, B, 128) &&
              tmap(&tdZ2, dZ2_, B, kSurHid, 128) && tmap(&tW2T, W2Tb_, kSurHid, kSurHid, 128) &&
              tmap(&tdZ2T, dZ2T_, kSurHid, B, 128) && tmap(&tH1T, H1T_, kSurHid, B, 128) &&
              tmap(&tdZ1T, dZ1T_, kSurHid, B, 128) && tmap(&tXTb, XTb_, kSurInPad, B, 64);
    if (!ok) return cudaErrorInvalidValue;
    int* err = &state_->err;

    gather_kernel<<<B, kSurInPad, 0, st>>>(Xall_, Tall_, perm_, state_, Xb_, XTb_, Tb_);
    QK_TRY(cudaGetLastError());

    GemmArgs g{};
    g.err = err;
    // layer 1 forward
    g.M = B; g.N = kSurHid; g.K = kSurInPad; g.k_per_split = kSurInPad;
    g.bias = P_ + SurLayout::b1; g.z_out = Z1_; g.h_out = H1_; g.t_out = H1T_; g.ldt = B;
    QK_TRY(launch_umma_gemm(kEpiFwd, 128, tXb, tW1, g, 1, st));
    // layer 2 forward
    g.K = kSurHid; g.k_per_split = kSurHid;
    g.bias = P_ + SurLayout::b2; g.z_out = Z2_; g.h_out = H2_; g.t_out = H2T_;
    QK_TRY(launch_umma_gemm(kEpiFwd, 128, tH1, tW2, g, 1, st));
    // layer 3 forward + head + loss gradient
    GemmArgs l{};
    l.err = err;
    l.M = B; l.N = kSurHid; l.K = kSurHid; l.k_per_split = kSurHid;
    l.bias = P_ + SurLayout::b3; l.w4 = P_ + SurLayout::w4; l.b4 = P_ + SurLayout::b4;
    l.target = Tb_; l.y_out = y_; l.dy_out = dy_; l.loss_scale = 2.0f / static_cast<float>(B);
    l.d_out = dZ3_; l.dt_out = dZ3T_; l.t_out = H3T_; l.ldt = B;
    QK_TRY(launch_umma_gemm(kEpiLast, 256, tH2, tW3, l, 1, st));
    // Side branch 1 (aux_[0]): the loss, db3, dw4 and the dW3 GEMM read only
    // what layer 3's epilogue wrote; they run beside the backward chain.
    QK_TRY(cudaEventRecord(ev_[0], st));
    QK_TRY(cudaStreamWaitEvent(aux_[0], ev_[0], 0));
    loss_kernel<<<1, 256, 0, aux_[0]>>>(y_, Tb_, dy_, state_, db4_, loss_hist_, loss_cap_);
    rowsum_kernel<<<kSurHid / 8, 256, 0, aux_[0]>>>(dZ3T_, kSurHid, B, nullptr, db3_);
    rowsum_kernel<<<kSurHid / 8, 256, 0, aux_[0]>>>(H3T_, kSurHid, B, dy_, dw4_);
    QK_TRY(cudaGetLastError());
    GemmArgs w{};
    w.err = err;
    w.M = kSurHid; w.N = kSurHid; w.K = B; w.k_per_split = 128; w.c_f32 = dW3p_;
    QK_TRY(launch_umma_gemm(kEpiF32, 128, tdZ3T, tH2T, w, S, aux_[0]));
    QK_TRY(cudaEventRecord(ev_[1], aux_[0]));
    // layer 3 backward to layer 2
    GemmArgs b{};
    b.err = err;
    b.M = B; b.N = kSurHid; b.K = kSurHid; b.k_per_split = kSurHid; b.ldt = B;
    b.z_in = Z2_; b.d_out = dZ2_; b.dt_out = dZ2T_;
    QK_TRY(launch_umma_gemm(kEpiBwd, 128, tdZ3, tW3T, b, 1, st));
    // Side branch 2 (aux_[1]): dW2 and db2 read layer 2's gradient
    QK_TRY(cudaEventRecord(ev_[2], st));
    QK_TRY(cudaStreamWaitEvent(aux_[1], ev_[2], 0));
    GemmArgs w2 = w;
    w2.c_f32 = dW2p_;
    QK_TRY(launch_umma_gemm(kEpiF32, 128, tdZ2T, tH1T, w2, S, aux_[1]));
    rowsum_kernel<<<kSurHid / 8, 256, 0, aux_[1]>>>(dZ2T_, kSurHid, B, nullptr, db2_);
    QK_TRY(cudaGetLastError());
    QK_TRY(cudaEventRecord(ev_[3], aux_[1]));
    // layer 2 backward to layer 1, dW1 (N = 64 padded inputs) and db1
    b.z_in = Z1_; b.d_out = dZ1_; b.dt_out = dZ1T_;
    QK_TRY(launch_umma_gemm(kEpiBwd, 128, tdZ2, tW2T, b, 1, st));
    GemmArgs w1 = w;
    w1.N = kSurInPad; w1.c_f32 = dW1p_;
    QK_TRY(launch_umma_gemm(kEpiF32, 64, tdZ1T, tXTb, w1, S, st));
    rowsum_kernel<<<kSurHid / 8, 256, 0, st>>>(dZ1T_, kSurHid, B, nullptr, db1_);
    QK_TRY(cudaGetLastError());
    // join both branches before Adam reads every gradient
    QK_TRY(cudaStreamWaitEvent(st, ev_[1], 0));
    QK_TRY(cudaStreamWaitEvent(st, ev_[3], 0));

    AdamArgs a{};
    const int hid2 = kSurHid * kSurHid;
    a.seg[0] = AdamSeg{SurLayout::W1, kSurHid * kSurInPad, dW1p_, S, (int64_t)kSurHid * kSurInPad, W1b_, nullptr, kSurHid, kSurInPad};
    a.seg[1] = AdamSeg{SurLayout::b1, kSurHid, db1_, 1, 0, nullptr, nullptr, 1, kSurHid};
    a.seg[2] = AdamSeg{SurLayout::W2, hid2, dW2p_, S, hid2, W2b_, W2Tb_, kSurHid, kSurHid};
    a.seg[3] = AdamSeg{SurLayout::b2, kSurHid, db2_, 1, 0, nullptr, nullptr, 1, kSurHid};
    a.seg[4] = AdamSeg{SurLayout::W3, hid2, dW3p_, S, hid2, W3b_, W3Tb_, kSurHid, kSurHid};
    a.seg[5] = AdamSeg{SurLayout::b3, kSurHid, db3_, 1, 0, nullptr, nullptr, 1, kSurHid};
    a.seg[6] = AdamSeg{SurLayout::w4, kSurHid, dw4_, 1, 0, nullptr, nullptr, 1, kSurHid};
    a.seg[7] = AdamSeg{SurLayout::b4, 1, db4_, 1, 0, nullptr, nullptr, 1, 1};
    a.nseg = 8;
    a.total = SurLayout::b4 + 1;
    a.P = P_;
    a.M = M_;
    a.V = V_;
    a.G = G_;
    a.update = update ? 1 : 0;
    a.st = state_;
    adam_kernel<<<(a.total + 255) / 256, 256, 0, st>>>(a);
    QK_TRY(cudaGetLastError());
    if (update) {
        advance_kernel<<<1, 1, 0, st>>>(state_);
        QK_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}

cudaError_t SurModel::train(int epochs, int batch, float lr0, uint64_t shuffle_seed,
                            float* out_loss_last, float* out_epoch_loss) {
    DeviceGuard g(device_);
    if (batch <= 0 || batch % 128 != 0 || n_data_ < batch || epochs <= 0) return cudaErrorInvalidValue;
    QK_TRY(ensure_batch_buffers(batch));
    const int spe = static_cast<int>(n_data_ / batch);
    const int total = spe * epochs;
    SurState s{};
    QK_TRY(cudaMemcpy(&s, state_, sizeof s, cudaMemcpyDeviceToHost));
    const int step0 = s.step;
    if (loss_cap_ < step0 + total) {
        QK_TRY(dalloc(&loss_hist_, static_cast<size_t>(step0 + total)));
        loss_cap_ = step0 + total;
        if (step_graph_) {
            cudaGraphExecDestroy(step_graph_);
            step_graph_ = nullptr;
        }
    }
    s.total_steps = step0 + total;
    s.step_begin = step0;
    s.steps_per_epoch = spe;
    s.batch = batch;
    s.lr0 = lr0;
    s.err = 0;
    // steps_per_epoch and batch change the gather: keep the step counter and
    // make epoch boundaries relative to it
    QK_TRY(cudaMemcpy(state_, &s, sizeof s, cudaMemcpyHostToDevice));
    if (!step_graph_) {
        cudaGraph_t graph;
        QK_TRY(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        cudaError_t le = run_step(stream_, true);
        cudaError_t ce = cudaStreamEndCapture(stream_, &graph);
        if (le != cudaSuccess) return le;
        QK_TRY(ce);
        ce = cudaGraphInstantiate(&step_graph_, graph, 0);
        cudaGraphDestroy(graph);
        QK_TRY(ce);
    }
    std::mt19937_64 rng(shuffle_seed);
    std::vector<int32_t> perm(static_cast<size_t>(n_data_));
    std::iota(perm.begin(), perm.end(), 0);
    for (int e = 0; e < epochs; ++e) {
        std::shuffle(perm.begin(), perm.end(), rng);
        // the gather reads perm[(step % spe) * batch + i]: rotate so the epoch
        // starts at the permutation's beginning whatever step0 % spe is
        const int rot = (step0 + e * spe) % spe;
        std::vector<int32_t> rotated(perm.size());
        for (int j = 0; j < spe; ++j)
            std::copy(perm.begin() + static_cast<int64_t>(j) * batch, perm.begin() + static_cast<int64_t>(j + 1) * batch,
                      rotated.begin() + static_cast<int64_t>((j + rot) % spe) * batch);
        QK_TRY(cudaStreamSynchronize(stream_));
        QK_TRY(cudaMemcpy(perm_, rotated.data(), static_cast<size_t>(spe) * batch * sizeof(int32_t),
                          cudaMemcpyHostToDevice));
        for (int j = 0; j < spe; ++j) QK_TRY(cudaGraphLaunch(step_graph_, stream_));
    }
    QK_TRY(cudaStreamSynchronize(stream_));
    std::vector<float> hist(static_cast<size_t>(total));
    QK_TRY(cudaMemcpy(hist.data(), loss_hist_ + step0, hist.size() * sizeof(float), cudaMemcpyDeviceToHost));
    if (out_loss_last) *out_loss_last = hist.back();
    if (out_epoch_loss) {
        for (int e = 0; e < epochs; ++e) {
            double acc = 0.0;
            for (int j = 0; j < spe; ++j) acc += hist[static_cast<size_t>(e) * spe + j];
            out_epoch_loss[e] = static_cast<float>(acc / spe);
        }
    }
    return cudaSuccess;
}

cudaError_t SurModel::ensure_predict_buffers(int64_t rows) {
    if (rows <= pred_rows_) return cudaSuccess;
    QK_TRY(dalloc(&PX_, static_cast<size_t>(rows) * kSurInPad));
    QK_TRY(dalloc(&PH1_, static_cast<size_t>(rows) * kSurHid));
    QK_TRY(dalloc(&PH2_, static_cast<size_t>(rows) * kSurHid));
    QK_TRY(dalloc(&Py_, static_cast<size_t>(rows)));
    QK_TRY(dalloc(&Pbase_, static_cast<size_t>(rows)));
    pred_rows_ = rows;
    return cudaSuccess;
}

cudaError_t SurModel::predict_device(const __nv_bfloat16* x, const float* base, int64_t n, float* y,
                                     cudaStream_t st, bool layered) {
    DeviceGuard g(device_);
    if (base_kind_ != kSurBaseNone && base == nullptr) return cudaErrorInvalidValue;
    if (!layered) {
        if (sm_count_ <= 0)
            QK_TRY(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device_));
        CUtensorMap tx, tw1, tw2, tw3;
        if (!(make_tmap_bf16_k16(&tx, x, static_cast<uint64_t>(n), kSurInPad, 128) &&
              make_tmap_bf16_k16(&tw1, W1b_, kSurHid, kSurInPad, 256) &&
              tmap(&tw2, W2b_, kSurHid, kSurHid, 256) && tmap(&tw3, W3b_, kSurHid, kSurHid, 256)))
            return cudaErrorInvalidValue;
        InferArgs ia{};
        ia.n = n;
        ia.b1 = P_ + SurLayout::b1;
        ia.b2 = P_ + SurLayout::b2;
        ia.b3 = P_ + SurLayout::b3;
        ia.w4 = P_ + SurLayout::w4;
        ia.b4 = P_ + SurLayout::b4;
        ia.base = base_kind_ != kSurBaseNone ? base : nullptr;
        ia.y = y;
        ia.err = &state_->err;
        return launch_mlp_infer(tx, tw1, tw2, tw3, ia, sm_count_, st);
    }
    QK_TRY(ensure_predict_buffers(std::min<int64_t>(n, kPredChunk)));
    for (int64_t off = 0; off < n; off += kPredChunk) {
        const int64_t m = std::min<int64_t>(kPredChunk, n - off);
        CUtensorMap tx, tw1, th1, tw2, th2, tw3;
        bool ok = tmap(&tx, x + off * kSurInPad, m, kSurInPad, 128) && tmap(&tw1, W1b_, kSurHid, kSurInPad, 128) &&
                  tmap(&th1, PH1_, m, kSurHid, 128) && tmap(&tw2, W2b_, kSurHid, kSurHid, 128) &&
                  tmap(&th2, PH2_, m, kSurHid, 128) && tmap(&tw3, W3b_, kSurHid, kSurHid, 256);
        if (!ok) return cudaErrorInvalidValue;
        GemmArgs f{};
        f.err = &state_->err;
        f.M = static_cast<int>(m); f.N = kSurHid; f.K = kSurInPad; f.k_per_split = kSurInPad;
        f.bias = P_ + SurLayout::b1; f.h_out = PH1_;
        QK_TRY(launch_umma_gemm(kEpiFwd, 128, tx, tw1, f, 1, st));
        f.K = kSurHid; f.k_per_split = kSurHid; f.bias = P_ + SurLayout::b2; f.h_out = PH2_;
        QK_TRY(launch_umma_gemm(kEpiFwd, 128, th1, tw2, f, 1, st));
        GemmArgs l{};
        l.err = &state_->err;
        l.M = static_cast<int>(m); l.N = kSurHid; l.K = kSurHid; l.k_per_split = kSurHid;
        l.bias = P_ + SurLayout::b3; l.w4 = P_ + SurLayout::w4; l.b4 = P_ + SurLayout::b4;
        l.y_out = y + off;
        l.base = base_kind_ != kSurBaseNone ? base + off : nullptr;
        QK_TRY(launch_umma_gemm(kEpiLast, 256, th2, tw3, l, 1, st));
    }
    return cudaSuccess;
}

cudaError_t SurModel::predict(const double* features, int64_t n, double* out) {
    DeviceGuard g(device_);
    const int64_t chunk = std::min<int64_t>(n, kPredChunk);
    QK_TRY(ensure_predict_buffers(chunk));
    std::vector<__nv_bfloat16> rows(static_cast<size_t>(chunk) * kSurInPad);
    std::vector<float> y(static_cast<size_t>(chunk)), b(static_cast<size_t>(chunk));
    __nv_bfloat16* xin = PX_;  // the chunk's inputs; predict_device uses PH1_/PH2_
    cudaError_t e = cudaSuccess;
    for (int64_t off = 0; off < n && e == cudaSuccess; off += chunk) {
        const int64_t m = std::min<int64_t>(chunk, n - off);
        normalise(features + off * kSurIn, m, rows.data());
        base_host(features + off * kSurIn, m, b.data());
        e = cudaMemcpyAsync(xin, rows.data(), static_cast<size_t>(m) * kSurInPad * sizeof(__nv_bfloat16),
                            cudaMemcpyHostToDevice, stream_);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(Pbase_, b.data(), static_cast<size_t>(m) * sizeof(float), cudaMemcpyHostToDevice,
                                stream_);
        if (e == cudaSuccess) e = predict_device(xin, Pbase_, m, Py_, stream_);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(y.data(), Py_, static_cast<size_t>(m) * sizeof(float), cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
        for (int64_t i = 0; i < m && e == cudaSuccess; ++i) out[off + i] = y[i];
    }
    return e;
}

cudaError_t SurModel::gradients(const double* features, const double* target, int n, double* grads,
                                double* loss) {
    DeviceGuard g(device_);
    if (n <= 0 || n % 128 != 0) return cudaErrorInvalidValue;
    QK_TRY(set_dataset(features, target, n));
    QK_TRY(ensure_batch_buffers(n));
    SurState s{};
    QK_TRY(cudaMemcpy(&s, state_, sizeof s, cudaMemcpyDeviceToHost));
    if (loss_cap_ < s.step + 1) {
        QK_TRY(dalloc(&loss_hist_, static_cast<size_t>(s.step + 1)));
        loss_cap_ = s.step + 1;
    }
    s.batch = n;
    s.steps_per_epoch = 1;
    QK_TRY(cudaMemcpy(state_, &s, sizeof s, cudaMemcpyHostToDevice));
    QK_TRY(run_step(stream_, false));
    QK_TRY(cudaStreamSynchronize(stream_));
    std::vector<float> G(SurLayout::total);
    QK_TRY(cudaMemcpy(G.data(), G_, G.size() * sizeof(float), cudaMemcpyDeviceToHost));
    float l = 0.0f;
    QK_TRY(cudaMemcpy(&l, loss_hist_ + s.step, sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    int k = 0;
    for (int r = 0; r < kSurHid; ++r)
        for (int c = 0; c < kSurIn; ++c) grads[k++] = G[SurLayout::W1 + r * kSurInPad + c];
    for (int i = SurLayout::b1; i <= SurLayout::b4; ++i) grads[k++] = G[i];
    return cudaSuccess;
}

cudaError_t SurModel::parameters(double* out) const {
    std::vector<float> P(SurLayout::total);
    QK_TRY(cudaMemcpy(P.data(), P_, P.size() * sizeof(float), cudaMemcpyDeviceToHost));
    int k = 0;
    for (int r = 0; r < kSurHid; ++r)
        for (int c = 0; c < kSurIn; ++c) out[k++] = P[SurLayout::W1 + r * kSurInPad + c];
    for (int i = SurLayout::b1; i <= SurLayout::b4; ++i) out[k++] = P[i];
    return cudaSuccess;
}

cudaError_t SurModel::set_parameters(const double* in) {
    DeviceGuard g(device_);
    std::vector<float> P(SurLayout::total, 0.0f);
    int k = 0;
    for (int r = 0; r < kSurHid; ++r)
        for (int c = 0; c < kSurIn; ++c) P[SurLayout::W1 + r * kSurInPad + c] = static_cast<float>(in[k++]);
    for (int i = SurLayout::b1; i <= SurLayout::b4; ++i) P[i] = static_cast<float>(in[k++]);
    QK_TRY(cudaMemcpy(P_, P.data(), P.size() * sizeof(float), cudaMemcpyHostToDevice));
    QK_TRY(refresh_bf16(stream_));
    return cudaStreamSynchronize(stream_);
}

int SurModel::steps_done() const {
    SurState s{};
    if (cudaMemcpy(&s, state_, sizeof s, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return s.step;
}

int SurModel::device_error() {
    SurState s{};
    if (cudaMemcpy(&s, state_, sizeof s, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return s.err;
}

// Checkpoint: "QKSURv02", layout size, base kind, the box, the state, P, M, V
// (FP32).  "QKSURv01" files (no base kind: a network without a base) load too.
cudaError_t SurModel::save(const char* path) {
    DeviceGuard g(device_);
    SurState s{};
    QK_TRY(cudaMemcpy(&s, state_, sizeof s, cudaMemcpyDeviceToHost));
    std::vector<float> buf(static_cast<size_t>(SurLayout::total) * 3);
    QK_TRY(cudaMemcpy(buf.data(), P_, SurLayout::total * sizeof(float), cudaMemcpyDeviceToHost));
    QK_TRY(cudaMemcpy(buf.data() + SurLayout::total, M_, SurLayout::total * sizeof(float), cudaMemcpyDeviceToHost));
    QK_TRY(cudaMemcpy(buf.data() + 2 * SurLayout::total, V_, SurLayout::total * sizeof(float), cudaMemcpyDeviceToHost));
    FILE* f = std::fopen(path, "wb");
    if (!f) return cudaErrorInvalidValue;
    const char magic[8] = {'Q', 'K', 'S', 'U', 'R', 'v', '0', '2'};
    const int32_t total = SurLayout::total;
    bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&total, sizeof total, 1, f) == 1 &&
              std::fwrite(&base_kind_, sizeof base_kind_, 1, f) == 1 &&
              std::fwrite(&box_, sizeof box_, 1, f) == 1 && std::fwrite(&s, sizeof s, 1, f) == 1 &&
              std::fwrite(buf.data(), sizeof(float), buf.size(), f) == buf.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t SurModel::load(const char* path) {
    DeviceGuard g(device_);
    FILE* f = std::fopen(path, "rb");
    if (!f) return cudaErrorInvalidValue;
    char magic[8];
    int32_t total = 0, kind = kSurBaseNone;
    SurBox box{};
    SurState s{};
    std::vector<float> buf(static_cast<size_t>(SurLayout::total) * 3);
    bool ok = std::fread(magic, 1, 8, f) == 8;
    const bool v2 = ok && std::memcmp(magic, "QKSURv02", 8) == 0;
    ok = ok && (v2 || std::memcmp(magic, "QKSURv01", 8) == 0) &&
         std::fread(&total, sizeof total, 1, f) == 1 && total == SurLayout::total &&
         (!v2 || std::fread(&kind, sizeof kind, 1, f) == 1) &&
         (kind == kSurBaseNone || kind == kSurBaseBsmMeanVar) &&
         std::fread(&box, sizeof box, 1, f) == 1 && std::fread(&s, sizeof s, 1, f) == 1 &&
         std::fread(buf.data(), sizeof(float), buf.size(), f) == buf.size();
    std::fclose(f);
    if (!ok) return cudaErrorInvalidValue;
    box_ = box;
    base_kind_ = kind;
    s.err = 0;
    QK_TRY(cudaMemcpy(state_, &s, sizeof s, cudaMemcpyHostToDevice));
    QK_TRY(cudaMemcpy(P_, buf.data(), SurLayout::total * sizeof(float), cudaMemcpyHostToDevice));
    QK_TRY(cudaMemcpy(M_, buf.data() + SurLayout::total, SurLayout::total * sizeof(float), cudaMemcpyHostToDevice));
    QK_TRY(cudaMemcpy(V_, buf.data() + 2 * SurLayout::total, SurLayout::total * sizeof(float), cudaMemcpyHostToDevice));
    QK_TRY(refresh_bf16(stream_));
    return cudaStreamSynchronize(stream_);
}

}  // namespace qkb
