// qk_error.h -- the thread-local error message behind qk_get_last_error().
//
// Restates yluoc/Quant-Kernel cpp/src/qk_api.cpp:19-37: a 256-byte
// thread-local buffer, "null pointer: <param>", "bad batch size: <n>"; CUDA
// failures (no reference counterpart) read "cuda error: <name> (<text>) in <call>".
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace qkb {

const char* last_error();
void clear_error();
void set_error_fmt(const char* fmt, ...);
int32_t fail_null(const char* name);   // QK_ERR_NULL_PTR
int32_t fail_size(int64_t n);          // QK_ERR_BAD_SIZE
int32_t fail_cuda(cudaError_t e, const char* where);  // QK_ERR_RUNTIME_INIT

}  // namespace qkb
