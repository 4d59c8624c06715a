// sur_api.cpp -- extern "C" entry points of the Heston surrogate.
#include "../../include/qk_api.h"

#include <cuda_runtime.h>

#include "qk_error.h"
#include "sur_gemm.cuh"

extern "C" {

int32_t qk_sur_gemm_bf16(const void* a, const void* b, float* c, int32_t m, int32_t n, int32_t k,
                         int32_t splits, void* stream) {
    if (!a) return qkb::fail_null("a");
    if (!b) return qkb::fail_null("b");
    if (!c) return qkb::fail_null("c");
    if (m <= 0 || n <= 0 || k <= 0 || splits <= 0 || k % 64 != 0 || n % 64 != 0 ||
        k % (64 * splits) != 0)
        return qkb::fail_size(m <= 0 ? m : (n <= 0 ? n : k));
    CUtensorMap ta, tb;
    const int bn = (n % 128 == 0) ? 128 : 64;
    if (!qkb::make_tmap_bf16(&ta, a, (uint64_t)m, (uint64_t)k, 128) ||
        !qkb::make_tmap_bf16(&tb, b, (uint64_t)n, (uint64_t)k, (uint32_t)bn))
        return qkb::fail_cuda(cudaErrorInvalidValue, "qk_sur_gemm_bf16 (tensor map)");
    qkb::GemmArgs g = {};
    g.M = m;
    g.N = n;
    g.K = k;
    g.k_per_split = k / splits;
    g.c_f32 = c;
    static int* err_word[64] = {};  // one device error word per GPU
    int dev = 0;
    cudaError_t de = cudaGetDevice(&dev);
    if (de != cudaSuccess || dev < 0 || dev >= 64) return qkb::fail_cuda(de, "qk_sur_gemm_bf16");
    if (!err_word[dev]) {
        cudaError_t e = cudaMalloc(&err_word[dev], sizeof(int));
        if (e != cudaSuccess) return qkb::fail_cuda(e, "qk_sur_gemm_bf16");
        cudaMemset(err_word[dev], 0, sizeof(int));
    }
    g.err = err_word[dev];
    cudaError_t e = qkb::launch_umma_gemm(qkb::kEpiF32, bn, ta, tb, g, splits,
                                          static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? QK_OK : qkb::fail_cuda(e, "qk_sur_gemm_bf16");
}

}  // extern "C"
