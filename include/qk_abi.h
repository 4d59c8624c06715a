/*
 * qk_abi.h -- ABI constants of the B200 Monte Carlo pricing library.
 *
 * Same values as yluoc/Quant-Kernel cpp/include/quantkernel/qk_abi.h:10-31
 * (return codes, option-type constants, QKPluginAPI layout), so callers of
 * the reference's batch MC calls keep their error handling unchanged.  The
 * minor version is 13: every 2.12 MC entry point is kept with its exact
 * signature and the additions are new names only.
 */
#ifndef QK_ABI_H
#define QK_ABI_H

#ifdef __cplusplus
#include <cstdint>
#else
#include <stdint.h>
#endif

#define QK_ABI_MAJOR 2
#define QK_ABI_MINOR 13

/* Return codes (qk_abi.h:15-20 of the reference). */
#define QK_OK                 0
#define QK_ERR_NULL_PTR      -1
#define QK_ERR_BAD_SIZE      -2
#define QK_ERR_ABI_MISMATCH  -3
#define QK_ERR_RUNTIME_INIT  -4  /* here: a CUDA call failed (no device, launch error, ...) */
#define QK_ERR_INVALID_INPUT -5

/* Option type constants (qk_abi.h:23-24 of the reference). */
#define QK_CALL 0
#define QK_PUT  1

typedef struct QKPluginAPI {
    int32_t     abi_major;
    int32_t     abi_minor;
    const char* plugin_name;
} QKPluginAPI;

#endif /* QK_ABI_H */
