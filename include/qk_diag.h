/*
 * qk_diag.h -- diagnostics of the B200 Monte Carlo pricing library.  No
 * counterpart in the reference (which has no GPU code): these measure the
 * hardware the kernels run on, for the rooflines the benchmark reports.
 */
#ifndef QK_DIAG_H
#define QK_DIAG_H

#include "qk_api.h" /* QK_EXPORT */

#ifdef __cplusplus
extern "C" {
#endif

/* What qk_b200_pipe_probe measures. */
#define QK_PROBE_MUFU  0 /* special-function unit: sin.approx, lane-ops per SM per clock */
#define QK_PROBE_FFMA  1 /* FP32 FMA, lane-FMAs per SM per clock */
#define QK_PROBE_FFMA2 2 /* packed f32x2 FMA, lane-FMAs per SM per clock */
#define QK_PROBE_DFMA  3 /* FP64 FMA, lane-FMAs per SM per clock */
#define QK_PROBE_MIX   4 /* MUFU ops per SM per clock when each comes with one packed
                          * FP32 FMA and ~4 integer operations (the Heston step's mix) */
#define QK_PROBE_ERR  -1

/*
 * Throughput of one pipe on `device`, in lane-operations per SM per SM clock:
 * every SM runs four 256-thread CTAs of independent dependency chains, and
 * each SM's rate is its lane-operations over the span of its CTAs' clock64()
 * stamps; the median over SMs is returned in *lane_ops_per_sm_clock.  Takes
 * a few milliseconds; allocates two small device buffers for the call.
 * Returns 0, or QK_PROBE_ERR (bad argument, or a CUDA call failed).
 */
QK_EXPORT int32_t qk_b200_pipe_probe(int32_t device, int32_t kind, double* lane_ops_per_sm_clock);

#ifdef __cplusplus
}
#endif

#endif /* QK_DIAG_H */
