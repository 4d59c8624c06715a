// qk_error.cpp -- thread-local error message (see qk_error.h).
#include "qk_error.h"

#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/qk_abi.h"
#include "qk_fault.h"

namespace qkb {

namespace {
thread_local char tl_error_msg[256] = "";
}

const char* last_error() { return tl_error_msg; }

void clear_error() { tl_error_msg[0] = '\0'; }

void set_error_fmt(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(tl_error_msg, sizeof tl_error_msg, fmt, ap);
    va_end(ap);
}

int32_t fail_null(const char* name) {
    set_error_fmt("null pointer: %s", name);
    return QK_ERR_NULL_PTR;
}

int32_t fail_size(int64_t n) {
    set_error_fmt("bad batch size: %lld", static_cast<long long>(n));
    return QK_ERR_BAD_SIZE;
}

int32_t fail_cuda(cudaError_t e, const char* where) {
    set_error_fmt("cuda error: %s (%s) in %s%s", cudaGetErrorName(e), cudaGetErrorString(e), where,
                  take_injected_flag() ? " [injected]" : "");
    return QK_ERR_RUNTIME_INIT;
}

}  // namespace qkb
