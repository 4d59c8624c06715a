// sur_gemm.cu -- tcgen05 / TMEM / TMA BF16 GEMM with fused MLP epilogues.
// See sur_gemm.cuh for the structure.
#include "sur_gemm.cuh"

#include <cudaTypedefs.h>

#include <mutex>

namespace qkb {

namespace {

constexpr int kStages = 4;
constexpr int kBM = 128;
constexpr int kBK = 64;                       // 64 bf16 = 128 B = one swizzle row
constexpr uint32_t kSpinLimit = 1u << 25;     // bounded mbarrier polls (seconds)
constexpr uint32_t kABytes = kBM * kBK * 2;   // 16 KiB
constexpr int kSurHidden = 256;               // hidden width of the surrogate MLP

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false after kSpinLimit polls (each poll may suspend briefly).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 B apart (SBO), leading offset unused for swizzled K-major (1),
// descriptor version 1 (sm_100), layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
           (static_cast<uint64_t>(1024 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
           (static_cast<uint64_t>(2) << 61);
}

// The same for 32-byte rows (K = 16 bf16): 32-byte swizzle, 8-row groups 256
// B apart, layout type 6 (SWIZZLE_32B).
__device__ __forceinline__ uint64_t desc_sw32(uint32_t addr) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
           (static_cast<uint64_t>(256 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
           (static_cast<uint64_t>(6) << 61);
}

// Instruction descriptor, kind::f16: D fp32, A and B bf16, both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24.
template <int BN>
__device__ __forceinline__ constexpr uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(BN >> 3) << 17) |
           (static_cast<uint32_t>(kBM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// sigmoid(z) = (1 + tanh(z / 2)) / 2 with the MUFU tanh (one special-function
// op; |error| ~ 2^-11, below the bf16 rounding every activation gets next).
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigmoidf_(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }

// SiLU straight from the accumulator: hz = z / 2 = fma(acc, 1/2, bias / 2) is
// exact (halving commutes with the rounding of acc + bias), so tanh(hz) is the
// sigmoid's tanh(z / 2), and silu(z) = z sigma(z) = hz + hz tanh(hz): two FMAs
// around one MUFU op.  Returns silu; hz and t = tanh(hz) for the caller.
__device__ __forceinline__ float silu_from_acc(float acc, float half_bias, float& hz, float& t) {
    hz = fmaf(acc, 0.5f, half_bias);
    t = tanh_approx(hz);
    return fmaf(hz, t, hz);
}

// silu_from_acc on two adjacent columns, the two FMAs as packed f32x2
// operations (each lane rounded as the scalar fmaf: the same bits).
__device__ __forceinline__ float2 silu2_from_acc(float2 acc, float2 half_bias) {
    const float2 hz = __ffma2_rn(acc, make_float2(0.5f, 0.5f), half_bias);
    const float2 t = make_float2(tanh_approx(hz.x), tanh_approx(hz.y));
    return __ffma2_rn(hz, t, hz);
}

// 32 bf16 values to 64 contiguous bytes.
__device__ __forceinline__ void store_bf16x32(__nv_bfloat16* dst, const float (&v)[32]) {
    uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        __nv_bfloat162 p[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) p[j] = __floats2bfloat162_rn(v[q * 8 + 2 * j], v[q * 8 + 2 * j + 1]);
        d[q] = *reinterpret_cast<uint4*>(p);
    }
}

__device__ __forceinline__ void load_bf16x32(const __nv_bfloat16* src, float (&v)[32]) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint4 u = s[q];
        const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float2 f = __bfloat1622float2(p[j]);
            v[q * 8 + 2 * j] = f.x;
            v[q * 8 + 2 * j + 1] = f.y;
        }
    }
}

// Eight epilogue warps: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its tile
// rows) and the column half w / 4 of the tile (chunks of 32 columns
// [c_lo, c_hi)); every element's arithmetic is the same as with one warp per
// lane quarter, so the split changes no bits.
template <int BN, int EPI>
__device__ __forceinline__ void epilogue(const GemmArgs& a, uint32_t tmem, int m0, int n0,
                                         float (*part_s)[kBM]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = warp & 3, half = warp >> 2;
    const int row = m0 + q * 32 + lane;
    const bool live = row < a.M;
    const uint32_t tbase = tmem + (static_cast<uint32_t>(q * 32) << 16);
    constexpr int kChunks = BN / 32;
    const int c_lo = half * (kChunks / 2), c_hi = c_lo + kChunks / 2;
    float v[32];
    if (EPI == kEpiF32) {
#pragma unroll 1
        for (int c = c_lo; c < c_hi; ++c) {
            tmem_ld32(tbase + c * 32, v);
            if (live) {
                float4* dst = reinterpret_cast<float4*>(
                    a.c_f32 + (static_cast<size_t>(blockIdx.z) * a.M + row) * a.N + n0 + c * 32);
#pragma unroll
                for (int q = 0; q < 8; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        }
    } else if (EPI == kEpiFwd) {
#pragma unroll 1
        for (int c = c_lo; c < c_hi; ++c) {
            tmem_ld32(tbase + c * 32, v);
            const int col0 = n0 + c * 32;
            float z[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                float hz, t;
                v[j] = silu_from_acc(v[j], 0.5f * __ldg(a.bias + col0 + j), hz, t);
                z[j] = 2.0f * hz;  // exact: the pre-activation acc + bias
            }
            if (live) {
                if (a.z_out) store_bf16x32(a.z_out + static_cast<size_t>(row) * a.N + col0, z);
                if (a.h_out) store_bf16x32(a.h_out + static_cast<size_t>(row) * a.N + col0, v);
                if (a.t_out) {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        a.t_out[static_cast<size_t>(col0 + j) * a.ldt + row] = __float2bfloat16_rn(v[j]);
                }
            }
        }
    } else if (EPI == kEpiBwd) {
#pragma unroll 1
        for (int c = c_lo; c < c_hi; ++c) {
            tmem_ld32(tbase + c * 32, v);
            const int col0 = n0 + c * 32;
            if (live) {
                float z[32];
                load_bf16x32(a.z_in + static_cast<size_t>(row) * a.N + col0, z);
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const float s = sigmoidf_(z[j]);
                    v[j] = v[j] * s * (1.0f + z[j] * (1.0f - s));
                }
                store_bf16x32(a.d_out + static_cast<size_t>(row) * a.N + col0, v);
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    a.dt_out[static_cast<size_t>(col0 + j) * a.ldt + row] = __float2bfloat16_rn(v[j]);
            }
        }
    } else {  // kEpiLast: BN == N (the whole hidden row is in this CTA)
        // head dot product as four partial sums, group g over the columns
        // 64 kb + 16 g + j (kb = 0..3, j = 0..15, in that order), combined in
        // order -- the summation of the fused inference kernel, whose warp g
        // owns those columns.  This warp's half takes groups 2 half, 2 half + 1.
        float p0 = 0.0f, p1 = 0.0f;
#pragma unroll 1
        for (int kb = 0; kb < 4; ++kb) {
            const int col0 = kb * 64 + half * 32;  // groups 2 half (16 cols), 2 half + 1 (16)
            tmem_ld32(tbase + col0, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                float hz, t;
                const float h = silu_from_acc(v[j], 0.5f * __ldg(a.bias + col0 + j), hz, t);
                p0 = fmaf(h, __ldg(a.w4 + col0 + j), p0);
            }
#pragma unroll
            for (int j = 16; j < 32; ++j) {
                float hz, t;
                const float h = silu_from_acc(v[j], 0.5f * __ldg(a.bias + col0 + j), hz, t);
                p1 = fmaf(h, __ldg(a.w4 + col0 + j), p1);
            }
        }
        part_s[2 * half][q * 32 + lane] = p0;
        part_s[2 * half + 1][q * 32 + lane] = p1;
        __syncthreads();  // all eight warps run the epilogue
        const int r = q * 32 + lane;
        float y = ((part_s[0][r] + part_s[1][r]) + part_s[2][r]) + part_s[3][r];
        y += __ldg(a.b4);
        if (live && half == 0) a.y_out[row] = a.base ? y + __ldg(a.base + row) : y;
        if (a.target != nullptr) {
            const float dy = live ? a.loss_scale * (y - a.target[row]) : 0.0f;
            if (live && half == 0) a.dy_out[row] = dy;
#pragma unroll 1
            for (int c = c_lo; c < c_hi; ++c) {
                tmem_ld32(tbase + c * 32, v);
                const int col0 = c * 32;
                float h[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    float hz, t;
                    h[j] = silu_from_acc(v[j], 0.5f * __ldg(a.bias + col0 + j), hz, t);
                    const float z = 2.0f * hz, s = fmaf(0.5f, t, 0.5f);
                    v[j] = dy * __ldg(a.w4 + col0 + j) * s * (1.0f + z * (1.0f - s));
                }
                if (live) {
                    store_bf16x32(a.d_out + static_cast<size_t>(row) * a.N + col0, v);
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        a.dt_out[static_cast<size_t>(col0 + j) * a.ldt + row] = __float2bfloat16_rn(v[j]);
                        a.t_out[static_cast<size_t>(col0 + j) * a.ldt + row] = __float2bfloat16_rn(h[j]);
                    }
                }
            }
        }
    }
}

constexpr int kGemmThreads = 256;  // warp 0: TMA, warp 1: MMA; all 8 warps: epilogue

template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                     const GemmArgs a) {
    constexpr uint32_t kBBytes = BN * kBK * 2;
    constexpr uint32_t kStage = kABytes + kBBytes;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                               ~static_cast<uintptr_t>(1023));
    __shared__ __align__(8) uint64_t full_bar[kStages];
    __shared__ __align__(8) uint64_t empty_bar[kStages];
    __shared__ __align__(8) uint64_t acc_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    __shared__ float part_s[4][kBM];  // head partial sums (kEpiLast)

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    const int kb0 = blockIdx.z * (a.k_per_split / kBK);
    int krem = a.K - blockIdx.z * a.k_per_split;
    if (krem > a.k_per_split) krem = a.k_per_split;
    const int nkb = krem > 0 ? krem / kBK : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        mbar_init(smem_u32(&acc_bar), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(static_cast<uint32_t>(BN))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;

    int last_round[kStages];
#pragma unroll
    for (int s = 0; s < kStages; ++s) last_round[s] = -1;

    if (warp == 0 && lane == 0) {
        // TMA producer
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % kStages;
            const int round = kb / kStages;
            if (round > 0 && !mbar_wait(smem_u32(&empty_bar[s]), (round - 1) & 1)) {
                abort_flag = 1;
                atomicExch(a.err, 1);
                break;
            }
            if (abort_flag) break;
            const uint32_t sa = smem_u32(smem + s * kStage);
            mbar_expect_tx(smem_u32(&full_bar[s]), kStage);
            const int kx = (kb0 + kb) * kBK;
            tma_load_2d(sa, &ta, kx, m0, smem_u32(&full_bar[s]));
            tma_load_2d(sa + kABytes, &tb, kx, n0, smem_u32(&full_bar[s]));
            last_round[s] = round;
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        constexpr uint32_t idesc = idesc_bf16<BN>();
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % kStages;
            if (!mbar_wait(smem_u32(&full_bar[s]), (kb / kStages) & 1)) {
                abort_flag = 1;
                atomicExch(a.err, 2);
                break;
            }
            if (abort_flag) break;
            fence_after();
            const uint32_t sa = smem_u32(smem + s * kStage);
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk)
                umma_bf16(tmem, desc_sw128(sa + kk * 32), desc_sw128(sa + kABytes + kk * 32), idesc,
                          (kb | kk) != 0 ? 1u : 0u);
            umma_commit(smem_u32(&empty_bar[s]));
        }
        umma_commit(smem_u32(&acc_bar));  // arrives once every issued MMA has completed
    }
    __syncwarp();

    // Epilogue: accumulator ready (bounded wait), then TMEM -> registers -> global.
    const bool acc_ok = mbar_wait(smem_u32(&acc_bar), 0);
    __syncwarp();
    fence_after();
    if (!acc_ok) {
        if (threadIdx.x == 0) atomicExch(a.err, 3);
        abort_flag = 1;
    }
    __syncthreads();
    if (!abort_flag && nkb > 0) epilogue<BN, EPI>(a, tmem, m0, n0, part_s);

    // Teardown: the producer drains its own loads (bounded), then TMEM is freed.
    if (warp == 0 && lane == 0 && abort_flag) {
        for (int s = 0; s < kStages; ++s)
            if (last_round[s] >= 0) mbar_wait(smem_u32(&full_bar[s]), last_round[s] & 1);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(static_cast<uint32_t>(BN))
                     : "memory");
    }
}


// ----------------------------------------------------------------------------
// Fused MLP inference.  One persistent CTA per SM walks its 128-row tiles two
// at a time, ping-pong: tile slot s (0, 1) owns TMEM accumulator s (256 fp32
// columns) and a 64 KiB shared buffer that holds the slot's input rows, then
// layer 1's and layer 2's activations.  While the epilogue warps work on one
// slot's layer, the tensor core computes the other slot's, so neither waits
// for the other's tail.  Four warp roles:
//   warp 16 (one lane)  weight producer: W1's first 16 columns once (8 KiB,
//                       resident), then the 32 KiB k-blocks of W2 and W3 in
//                       the order the MMA issuer takes them (per tile pair:
//                       W2[0..3] for A, for B, W3[0..3] for A, for B) through
//                       a 2-slot ring;
//   warp 17 (one lane)  MMA issuer: per tile pair, layer by layer, tile A's
//                       then tile B's: layer 1 (one K = 16 MMA: the 9
//                       features and their zero padding; the rows' columns
//                       16..63 are zeros too and would add exact zeros) once
//                       the slot's input rows have landed and its previous
//                       tile's head has read the accumulator, layers 2 and 3
//                       once the epilogue has written the slot's previous
//                       layer;
//   warp 18 (one lane)  input loader: a slot's next input rows (their first
//                       16 columns, 32-byte swizzled: 4 KiB) once the MMAs
//                       of its previous tile's layer 3 (the last reader of
//                       the slot's buffer) have completed;
//   warps 0-15          epilogue, in the MMA issuer's order: warp w reads TMEM
//                       lanes 32 (w % 4) .. + 31 (its tile rows) and, in each
//                       64-column block kb, columns 64 kb + 16 (w / 4) .. + 15;
//                       bias + SiLU, BF16 into the slot's buffer in the
//                       128-byte-swizzled K-major layout the next layer's MMA
//                       reads as its A operand; the head sums partial chains
//                       and writes the prices.
// Every hand-off is an mbarrier with a bounded wait (no CTA-wide barrier
// inside the loop), so a timeout anywhere ends every role with an error code.
// Barriers per slot: xfull (input rows landed), accfull (a layer's MMAs
// complete: three phases per tile), hdone (all 16 epilogue warps finished a
// layer of the slot: three phases per tile), pready (the head's partial sums,
// one phase per tile).  Hazards, each closed by the chain: an accumulator is
// rewritten only after hdone reports the epilogue read it; a buffer is
// rewritten by the epilogue only after accfull reports that the MMAs which
// read it completed, and by the input loader only after the slot's layer-3
// accfull; the head's partial sums are double-buffered by slot.
// The arithmetic and summation order are those of the layer-by-layer GEMMs
// (kEpiFwd, kEpiLast), so the results are the same bits.
// ----------------------------------------------------------------------------
constexpr int kIWSlots = 2;
constexpr uint32_t kWBlock = 256 * kBK * 2;        // 32 KiB: 256 rows x 64 bf16
constexpr uint32_t kHBytes = 4 * kABytes;          // 64 KiB: 128 rows x 256 bf16
constexpr int kTileSlots = 2;
// Layer 1 reads only K = 16 (the 9 features and their zero padding): input
// rows of 32 bytes, and W1's first 16 columns held resident for the launch.
constexpr uint32_t kXBytes = kBM * 16 * 2;         // 4 KiB: 128 rows x 16 bf16
constexpr uint32_t kW1Bytes = 256 * 16 * 2;        // 8 KiB: 256 rows x 16 bf16
constexpr size_t kInferSmem = kTileSlots * kHBytes + kIWSlots * kWBlock + kW1Bytes + 1024;
constexpr int kInferEpiWarps = 16;                 // 4 per TMEM lane quarter
constexpr int kInferThreads = (kInferEpiWarps + 3) * 32;
constexpr int kProducerWarp = kInferEpiWarps, kMmaWarp = kInferEpiWarps + 1,
              kXWarp = kInferEpiWarps + 2;

// 16 consecutive fp32 columns of this thread's TMEM lane (no wait).
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// 16 activations (columns col0 .. col0 + 15 of tile row r, col0 % 16 == 0)
// into the layout a 128-byte-swizzle TMA load would produce: k-block
// col / 64, row r at 128 r, 16-byte chunk c at (c ^ (r & 7)) * 16.
__device__ __forceinline__ void store_h16_sw128(uint8_t* hbuf, int r, int col0, const float (&v)[16]) {
    uint8_t* row = hbuf + (col0 >> 6) * kABytes + r * 128;
    const int c0 = (col0 & 63) >> 3;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        __nv_bfloat162 p[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) p[j] = __floats2bfloat162_rn(v[q * 8 + 2 * j], v[q * 8 + 2 * j + 1]);
        *reinterpret_cast<uint4*>(row + (((c0 + q) ^ (r & 7)) << 4)) = *reinterpret_cast<uint4*>(p);
    }
}

__global__ void __launch_bounds__(kInferThreads, 1)
    mlp_infer_kernel(const __grid_constant__ CUtensorMap tx, const __grid_constant__ CUtensorMap tw1,
                     const __grid_constant__ CUtensorMap tw2, const __grid_constant__ CUtensorMap tw3,
                     const InferArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                               ~static_cast<uintptr_t>(1023));
    uint8_t* hbufs = smem;  // [kTileSlots][kHBytes]: a slot's input rows, then its activations
    uint8_t* wbuf = smem + kTileSlots * kHBytes;
    uint8_t* w1s = wbuf + kIWSlots * kWBlock;  // W1 [256][16], resident
    __shared__ __align__(8) uint64_t w1full;
    __shared__ __align__(8) uint64_t xfull[kTileSlots], slotfree[kTileSlots], accfull[kTileSlots];
    __shared__ __align__(8) uint64_t hdone[kTileSlots], pready[kTileSlots];
    __shared__ __align__(8) uint64_t wfull[kIWSlots], wempty[kIWSlots], drain;
    __shared__ __align__(16) float sb1[kSurHidden], sb2[kSurHidden], sb3[kSurHidden], sw4[kSurHidden];
    __shared__ float part[kTileSlots][4][kBM];  // head partial sums per slot and column group
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t n_tiles = (a.n + kBM - 1) / kBM;
    // this CTA's tiles i = 0, 1, ...: tile blockIdx.x + i gridDim.x, slot i % 2,
    // the slot's use u = i / 2; tiles 2p and 2p + 1 form pair p
    const int64_t my_tiles =
        blockIdx.x < n_tiles ? (n_tiles - 1 - static_cast<int64_t>(blockIdx.x)) / gridDim.x + 1 : 0;

    if (tid < kSurHidden) {
        sb1[tid] = 0.5f * a.b1[tid];  // halved biases for silu_from_acc (exact)
        sb2[tid] = 0.5f * a.b2[tid];
        sb3[tid] = 0.5f * a.b3[tid];
        sw4[tid] = a.w4[tid];
    }
    if (tid == 0) {
        for (int s = 0; s < kTileSlots; ++s) {
            mbar_init(smem_u32(&xfull[s]), 1);
            mbar_init(smem_u32(&slotfree[s]), 1);
            mbar_init(smem_u32(&accfull[s]), 1);
            mbar_init(smem_u32(&hdone[s]), kInferEpiWarps);
            mbar_init(smem_u32(&pready[s]), kInferEpiWarps);
        }
        for (int s = 0; s < kIWSlots; ++s) {
            mbar_init(smem_u32(&wfull[s]), 1);
            mbar_init(smem_u32(&wempty[s]), 1);
        }
        mbar_init(smem_u32(&drain), 1);
        mbar_init(smem_u32(&w1full), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {  // one accumulator of 256 fp32 columns per tile slot
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    auto fail = [&](int code) {
        abort_flag = 1;
        atomicExch(a.err, code);
    };

    // bookkeeping for the teardown drain
    int last_round[kIWSlots] = {-1, -1};
    int64_t x_last[kTileSlots] = {-1, -1};
    bool w1_issued = false;

    if (warp == kProducerWarp) {
        if (lane == 0) {
            uint32_t wl = 0;
            auto load_w = [&](const CUtensorMap* m, int kx) -> bool {
                const uint32_t s = wl % kIWSlots, round = wl / kIWSlots;
                if (round > 0 && !mbar_wait(smem_u32(&wempty[s]), (round - 1) & 1)) return false;
                mbar_expect_tx(smem_u32(&wfull[s]), kWBlock);
                tma_load_2d(smem_u32(wbuf + s * kWBlock), m, kx, 0, smem_u32(&wfull[s]));
                last_round[s] = static_cast<int>(round);
                ++wl;
                return true;
            };
            if (my_tiles > 0) {  // W1's first 16 columns, once
                mbar_expect_tx(smem_u32(&w1full), kW1Bytes);
                tma_load_2d(smem_u32(w1s), &tw1, 0, 0, smem_u32(&w1full));
                w1_issued = true;
            }
            for (int64_t i0 = 0; i0 < my_tiles; i0 += 2) {
                if (abort_flag) break;
                const int nt = (my_tiles - i0) >= 2 ? 2 : 1;
                // the MMA issuer's order: layers 2 and 3 for tile A, then tile B
                bool ok = true;
                for (int k = 0; ok && k < nt; ++k)
                    for (int kb = 0; ok && kb < 4; ++kb) ok = load_w(&tw2, kb * kBK);
                for (int k = 0; ok && k < nt; ++k)
                    for (int kb = 0; ok && kb < 4; ++kb) ok = load_w(&tw3, kb * kBK);
                if (!ok) {
                    fail(22);
                    break;
                }
            }
        }
    } else if (warp == kXWarp) {
        if (lane == 0) {
            for (int64_t i = 0; i < my_tiles; ++i) {
                if (abort_flag) break;
                const int s = static_cast<int>(i & 1);
                const int64_t u = i >> 1;
                // the slot's previous tile's layer-3 MMAs, the last readers of
                // its buffer, have completed (one slotfree phase per tile)
                if (u > 0 && !mbar_wait(smem_u32(&slotfree[s]), static_cast<uint32_t>((u - 1) & 1))) {
                    fail(21);
                    break;
                }
                mbar_expect_tx(smem_u32(&xfull[s]), kXBytes);
                const int64_t t = blockIdx.x + i * gridDim.x;
                tma_load_2d(smem_u32(hbufs + s * kHBytes), &tx, 0, static_cast<int>(t * kBM),
                            smem_u32(&xfull[s]));
                x_last[s] = u;
            }
        }
    } else if (warp == kMmaWarp) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16<256>();
            uint32_t wc = 0;
            // one k-block of W from the ring into accumulator acc
            auto mma_kblock = [&](uint32_t acc, uint32_t sa, bool first) -> bool {
                const uint32_t s = wc % kIWSlots;
                if (!mbar_wait(smem_u32(&wfull[s]), (wc / kIWSlots) & 1)) return false;
                fence_after();
                const uint32_t sb = smem_u32(wbuf + s * kWBlock);
#pragma unroll
                for (int kk = 0; kk < kBK / 16; ++kk)
                    umma_bf16(acc, desc_sw128(sa + kk * 32), desc_sw128(sb + kk * 32), idesc,
                              (first && kk == 0) ? 0u : 1u);
                umma_commit(smem_u32(&wempty[s]));
                ++wc;
                return true;
            };
            bool ok = my_tiles == 0 || mbar_wait(smem_u32(&w1full), 0u);
            if (!ok) fail(25);
            const uint64_t dw1 = desc_sw32(smem_u32(w1s));
            for (int64_t i0 = 0; ok && i0 < my_tiles; i0 += 2) {
                if (abort_flag) break;
                const int nt = (my_tiles - i0) >= 2 ? 2 : 1;
                const int64_t u = i0 >> 1;
                for (int l = 0; ok && l < 3; ++l) {
                    for (int s = 0; ok && s < nt; ++s) {
                        const uint32_t acc = tmem + s * 256;
                        const uint8_t* hb = hbufs + s * kHBytes;
                        if (l == 0) {
                            // the slot's input rows, and its previous tile's
                            // head done reading the accumulator
                            ok = mbar_wait(smem_u32(&xfull[s]), static_cast<uint32_t>(u & 1));
                            if (ok && u > 0)
                                ok = mbar_wait(smem_u32(&hdone[s]), static_cast<uint32_t>((3 * u - 1) & 1));
                            fence_after();
                            // K = 16: the input rows and the resident W1 slice
                            if (ok) umma_bf16(acc, desc_sw32(smem_u32(hb)), dw1, idesc, 0u);
                        } else {
                            // layer l's activations written (and its
                            // accumulator read) by every epilogue warp
                            ok = mbar_wait(smem_u32(&hdone[s]), static_cast<uint32_t>((3 * u + l - 1) & 1));
                            fence_after();
                            for (int kb = 0; ok && kb < 4; ++kb)
                                ok = mma_kblock(acc, smem_u32(hb + kb * kABytes), kb == 0);
                        }
                        if (!ok) break;
                        umma_commit(smem_u32(&accfull[s]));
                        if (l == 2) umma_commit(smem_u32(&slotfree[s]));
                    }
                }
                if (!ok) fail(24);
            }
        }
    } else {
        // epilogue warps; lane 0 polls each barrier and broadcasts the
        // outcome, so a warp's lanes always take the same path; then every
        // lane observes the completed phase itself (its own acquire: the
        // phase cannot advance again before this warp's next arrival)
        auto warp_wait = [&](uint32_t bar, uint32_t parity) -> bool {
            bool done = false;
            if (lane == 0) done = mbar_wait(bar, parity);
            done = __shfl_sync(0xFFFFFFFFu, done ? 1 : 0, 0) != 0;
            if (done) done = __all_sync(0xFFFFFFFFu, mbar_try(bar, parity)) != 0;
            return done;
        };
        const int q = warp & 3, g = warp >> 2;
        const int r = q * 32 + lane;
        const uint32_t lane_off = static_cast<uint32_t>(q * 32) << 16;
        const float b4 = __ldg(a.b4);
        bool ok = true;
        for (int64_t i0 = 0; ok && i0 < my_tiles; i0 += 2) {
            const int nt = (my_tiles - i0) >= 2 ? 2 : 1;
            const int64_t u = i0 >> 1;
            for (int l = 0; ok && l < 3; ++l) {
                for (int s = 0; ok && s < nt; ++s) {
                    const uint32_t acc = tmem + s * 256 + lane_off;
                    ok = warp_wait(smem_u32(&accfull[s]), static_cast<uint32_t>((3 * u + l) & 1));
                    fence_after();
                    if (!ok) {
                        if (lane == 0) fail(26);
                        break;
                    }
                    if (l < 2) {
                        const float* bias = l == 0 ? sb1 : sb2;
                        uint8_t* hbuf = hbufs + s * kHBytes;
#pragma unroll
                        for (int kb = 0; kb < 4; ++kb) {
                            const int col0 = kb * 64 + g * 16;
                            uint32_t uu[16];
                            tmem_ld16_async(acc + col0, uu);
                            tmem_wait_ld();
                            float v[16];
#pragma unroll
                            for (int j = 0; j < 16; j += 2) {
                                const float2 h = silu2_from_acc(
                                    make_float2(__uint_as_float(uu[j]), __uint_as_float(uu[j + 1])),
                                    *reinterpret_cast<const float2*>(bias + col0 + j));
                                v[j] = h.x;
                                v[j + 1] = h.y;
                            }
                            store_h16_sw128(hbuf, r, col0, v);
                        }
                        // the shared stores to the tensor core's (async) proxy,
                        // the TMEM reads before the hand-off
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(smem_u32(&hdone[s]));
                    } else {
                        // head: this warp's chain over columns 64 kb + 16 g + j
                        float p = 0.0f;
#pragma unroll
                        for (int kb = 0; kb < 4; ++kb) {
                            const int col0 = kb * 64 + g * 16;
                            uint32_t uu[16];
                            tmem_ld16_async(acc + col0, uu);
                            tmem_wait_ld();
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                float hz, t;
                                const float h = silu_from_acc(__uint_as_float(uu[j]), sb3[col0 + j], hz, t);
                                p = fmaf(h, sw4[col0 + j], p);
                            }
                        }
                        // the accumulator is read: the slot's next tile may
                        // start its layer 1
                        fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(smem_u32(&hdone[s]));
                        part[s][g][r] = p;
                        __syncwarp();
                        if (lane == 0) mbar_arrive(smem_u32(&pready[s]));
                        if (g == 0) {
                            ok = warp_wait(smem_u32(&pready[s]), static_cast<uint32_t>(u & 1));
                            if (!ok) {
                                if (lane == 0) fail(27);
                                break;
                            }
                            const float y =
                                (((part[s][0][r] + part[s][1][r]) + part[s][2][r]) + part[s][3][r]) + b4;
                            const int64_t row = (blockIdx.x + (i0 + s) * gridDim.x) * kBM + r;
                            if (row < a.n) a.y[row] = a.base ? y + __ldg(a.base + row) : y;
                        }
                    }
                }
            }
        }
    }

    // Teardown.  After an abort: the producer and the input loader wait
    // (bounded) for the loads they issued, the MMA issuer for its MMAs (a
    // commit on `drain`), then the accumulators are freed.
    fence_before();
    __syncthreads();
    if (abort_flag) {
        if (warp == kProducerWarp && lane == 0) {
            for (int s = 0; s < kIWSlots; ++s)
                if (last_round[s] >= 0) mbar_wait(smem_u32(&wfull[s]), last_round[s] & 1);
            if (w1_issued) mbar_wait(smem_u32(&w1full), 0u);
        } else if (warp == kXWarp && lane == 0) {
            for (int s = 0; s < kTileSlots; ++s)
                if (x_last[s] >= 0) mbar_wait(smem_u32(&xfull[s]), static_cast<uint32_t>(x_last[s] & 1));
        } else if (warp == kMmaWarp && lane == 0) {
            umma_commit(smem_u32(&drain));
            mbar_wait(smem_u32(&drain), 0);
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u)
                     : "memory");
    }
}

template <int BN, int EPI>
cudaError_t launch_t(const CUtensorMap& ta, const CUtensorMap& tb, const GemmArgs& a, int splits,
                     cudaStream_t st) {
    constexpr size_t smem = kStages * (kABytes + BN * kBK * 2) + 1024;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(umma_gemm_kernel<BN, EPI>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    if (attr_err != cudaSuccess) return attr_err;
    dim3 grid((a.M + kBM - 1) / kBM, a.N / BN, splits);
    umma_gemm_kernel<BN, EPI><<<grid, kGemmThreads, smem, st>>>(ta, tb, a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_mlp_infer(const CUtensorMap& tx, const CUtensorMap& tw1, const CUtensorMap& tw2,
                             const CUtensorMap& tw3, const InferArgs& a, int ctas, cudaStream_t st) {
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(kInferSmem));
    });
    if (attr_err != cudaSuccess) return attr_err;
    if (a.n <= 0) return cudaSuccess;
    const int64_t tiles = (a.n + kBM - 1) / kBM;
    const int grid = static_cast<int>(tiles < ctas ? tiles : ctas);
    mlp_infer_kernel<<<grid, kInferThreads, kInferSmem, st>>>(tx, tw1, tw2, tw3, a);
    return cudaGetLastError();
}

bool make_tmap_bf16(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols,
                    uint32_t box_rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!encode) return false;
    // Host-side checks of the TMA rules: 16-byte aligned base, row stride a
    // multiple of 16 bytes, a 64-element (128-byte) inner box.
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (cols * 2) % 16 != 0 || cols < 64) return false;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {cols * 2};
    const cuuint32_t box[2] = {64, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool make_tmap_bf16_k16(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols,
                        uint32_t box_rows) {
    if (!make_tmap_bf16(map, base, rows, cols, box_rows)) return false;  // also loads the encoder
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!encode || box_rows == 0 || box_rows > 256) return false;
    // 16 bf16 = 32 bytes: the inner box equals the 32-byte swizzle span
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {cols * 2};
    const cuuint32_t box[2] = {16, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_umma_gemm(int epi, int bn, const CUtensorMap& ta, const CUtensorMap& tb,
                             const GemmArgs& a, int splits, cudaStream_t st) {
    if (a.K % kBK != 0 || a.k_per_split % kBK != 0 || a.N % bn != 0 || splits < 1)
        return cudaErrorInvalidValue;
    switch (bn) {
        case 64:
            if (epi == kEpiF32) return launch_t<64, kEpiF32>(ta, tb, a, splits, st);
            break;
        case 128:
            if (epi == kEpiF32) return launch_t<128, kEpiF32>(ta, tb, a, splits, st);
            if (epi == kEpiFwd) return launch_t<128, kEpiFwd>(ta, tb, a, splits, st);
            if (epi == kEpiBwd) return launch_t<128, kEpiBwd>(ta, tb, a, splits, st);
            break;
        case 256:
            if (epi == kEpiF32) return launch_t<256, kEpiF32>(ta, tb, a, splits, st);
            if (epi == kEpiFwd) return launch_t<256, kEpiFwd>(ta, tb, a, splits, st);
            if (epi == kEpiLast) return launch_t<256, kEpiLast>(ta, tb, a, splits, st);
            if (epi == kEpiBwd) return launch_t<256, kEpiBwd>(ta, tb, a, splits, st);
            break;
        default:
            break;
    }
    return cudaErrorInvalidValue;
}

}  // namespace qkb
