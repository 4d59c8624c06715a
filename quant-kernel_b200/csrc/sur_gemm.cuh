// sur_gemm.cuh -- BF16 tensor-core GEMM for the surrogate MLP (sm_100a).
//
//   C[M x N] = A[M x K] . B[N x K]^T      A, B bf16 row-major (K contiguous)
//
// One CTA computes a 128 x BN tile over a K range (split-K over blockIdx.z):
//   * warp 0 / lane 0 loads 128x64 A and BNx64 B tiles with TMA
//     (cp.async.bulk.tensor, 128-byte swizzle) into a 4-stage ring, each stage
//     guarded by "full" and "empty" mbarriers;
//   * warp 1 / lane 0 issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32,
//     M = 128, N = BN, K = 16 per instruction) from shared-memory descriptors
//     into a TMEM accumulator, and frees a stage with tcgen05.commit;
//   * all four warps then read the accumulator with tcgen05.ld (warp w owns
//     TMEM lanes 32w..32w+31 = tile rows) and run the fused epilogue.
// Every mbarrier wait is bounded: on timeout the kernel records an error code
// in *err, drains what it issued (again bounded), frees its TMEM and returns.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace qkb {

enum : int {
    kEpiF32 = 0,    // C fp32 (split-K partial slab per blockIdx.z)
    kEpiFwd = 1,    // z = acc + bias; h = silu(z): write Z, H (bf16) and H^T
    kEpiLast = 2,   // layer 3 + head: y = silu(acc + b3) . w4 + b4; training: dZ3, dZ3^T, H3^T
    kEpiBwd = 3,    // dz = acc * silu'(z_in): write dZ and dZ^T
};

struct GemmArgs {
    int M, N, K;             // problem size (K range split over gridDim.z)
    int k_per_split;         // multiple of 64
    // epilogue operands (bf16 outputs are row-major [M][N]; "t" outputs [N][ldt])
    float* c_f32;            // kEpiF32: [gridDim.z][M][N]
    const float* bias;       // [N]
    __nv_bfloat16* z_out;
    __nv_bfloat16* h_out;
    __nv_bfloat16* t_out;    // transposed output, row stride ldt
    int ldt;
    const __nv_bfloat16* z_in;   // kEpiBwd: pre-activation [M][N]
    __nv_bfloat16* d_out;        // kEpiLast (training) / kEpiBwd: dZ [M][N]
    __nv_bfloat16* dt_out;       // dZ^T [N][ldt]
    const float* w4;             // head weights [N]
    const float* b4;             // head bias [1]
    const float* target;         // [M] (training) or null (inference)
    float* y_out;                // [M]
    const float* base;           // [M] added to y_out (inference), or null
    float* dy_out;               // [M] dL/dy (training)
    float loss_scale;            // dL/dy = loss_scale * (y - target)
    int* err;                    // error word (0 = ok)
};

// Fused MLP inference: y[i] = w4 . silu(W3 silu(W2 silu(W1 x_i + b1) + b2) + b3) + b4
// (+ base[i] when base is not null) for normalised bf16 rows x [n][64] (see
// sur_gemm.cu, mlp_infer_kernel).
struct InferArgs {
    int64_t n;               // rows
    const float* b1;         // [256]
    const float* b2;
    const float* b3;
    const float* w4;
    const float* b4;         // [1]
    const float* base;       // [n] added to the network's output, or null
    float* y;                // [n]
    int* err;                // error word (0 = ok)
};
// tx: x [n][64] and tw1: W1 [256][64] read through their first 16 columns
// (make_tmap_bf16_k16: the 9 features and their zero padding; boxes 16 x 128
// and 16 x 256, 32-byte swizzle); tw2, tw3: [256][256] (boxes 64 x 256).
// ctas: persistent grid size (one CTA per SM).
cudaError_t launch_mlp_infer(const CUtensorMap& tx, const CUtensorMap& tw1, const CUtensorMap& tw2,
                             const CUtensorMap& tw3, const InferArgs& a, int ctas, cudaStream_t st);

// Host side: tensor maps over bf16 row-major [rows][cols] (cols contiguous).
bool make_tmap_bf16(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols,
                    uint32_t box_rows);
// The same over columns 0..15 only (a 16 x box_rows box, 32-byte swizzle).
bool make_tmap_bf16_k16(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols,
                        uint32_t box_rows);
cudaError_t launch_umma_gemm(int epi, int bn, const CUtensorMap& ta, const CUtensorMap& tb,
                             const GemmArgs& a, int splits, cudaStream_t st);

}  // namespace qkb
