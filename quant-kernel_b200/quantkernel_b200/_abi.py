"""ABI constants of libqk_b200.so (values of yluoc/Quant-Kernel python/quantkernel/_abi.py,
minor version 13 for the additive Monte Carlo calls)."""

ABI_MAJOR = 2
ABI_MINOR = 13

QK_OK = 0
QK_ERR_NULL_PTR = -1
QK_ERR_BAD_SIZE = -2
QK_ERR_ABI_MISMATCH = -3
QK_ERR_RUNTIME_INIT = -4
QK_ERR_INVALID_INPUT = -5

QK_CALL = 0
QK_PUT = 1

# Model codes of the mixed-model batch and of plans (include/qk_api.h).
QK_MC_STANDARD = 0
QK_MC_ANTITHETIC = 1
QK_MC_EULER = 2
QK_MC_MILSTEIN = 3
QK_MC_LOCAL_VOL = 4
QK_MC_TERMINAL_PLAIN = 5
QK_MC_HESTON = 6
QK_MC_HESTON_LR_DELTA = 7
QK_MC_CONTROL_VARIATES = 8
QK_MC_IMPORTANCE_SAMPLING = 9  # shift read from v0 in mixed batches and plans
QK_MC_STRATIFIED = 10
QK_MC_QMC_SOBOL = 11
QK_MC_QMC_HALTON = 12

QK_PLAN_PERSISTENT = 0x1
QK_PLAN_GRAPH = 0x2
QK_PLAN_NO_ANTITHETIC = 0x4
QK_PLAN_TIMING = 0x8
QK_PLAN_AUTOTUNE = 0x10
QK_PLAN_FAMILY_GRIDS = 0x20
QK_PLAN_STEP_UNROLL2 = 0x40

QK_DIST_ID_BYTES = 128  # communicator id of the sharded calls (qk_dist_unique_id)
