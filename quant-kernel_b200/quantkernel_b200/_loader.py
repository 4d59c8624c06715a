"""Finds libqk_b200.so, binds its C ABI and verifies the ABI version.

Mirrors yluoc/Quant-Kernel python/quantkernel/_loader.py:91-363 (search path,
eager binding, ABI negotiation) for the Monte Carlo subset this library
exports.  The search order is ``QK_B200_LIB_PATH``, then this package's
directory.  There is no fallback: a missing library raises ``OSError``.
"""

import ctypes as ct
import os
from pathlib import Path

from ._abi import ABI_MAJOR, ABI_MINOR, QK_OK

D = ct.c_double
I32 = ct.c_int32
I64 = ct.c_int64
U64 = ct.c_uint64
PD = ct.POINTER(ct.c_double)
PI32 = ct.POINTER(ct.c_int32)
PI64 = ct.POINTER(ct.c_int64)
PU64 = ct.POINTER(ct.c_uint64)
VP = ct.c_void_p

LIB_NAME = "libqk_b200.so"


class QKPluginAPI(ct.Structure):
    _fields_ = [
        ("abi_major", I32),
        ("abi_minor", I32),
        ("plugin_name", ct.c_char_p),
    ]


_term_scalar = [D, D, D, D, D, D, I32, I32, U64]
_term_batch = [PD, PD, PD, PD, PD, PD, PI32, PI32, PU64, I32, PD]
_step_scalar = [D, D, D, D, D, D, I32, I32, I32, U64]
_step_batch = [PD, PD, PD, PD, PD, PD, PI32, PI32, PI32, PU64, I32, PD]
_hes_scalar = [D, D, D, D, D, D, D, D, D, D, I32, I32, I32, U64]
_hes_batch = [PD] * 10 + [PI32, PI32, PI32, PU64, I32, PD]
_mixed_arrays = [PI32] + [PD] * 11 + [PI32, PI32, PI32, PU64, I32]
_is_scalar = [D, D, D, D, D, D, I32, I32, D, U64]
_is_batch = [PD] * 6 + [PI32, PI32, PD, PU64, I32, PD]
_qmc_scalar = [D, D, D, D, D, D, I32, I32]
_qmc_batch = [PD] * 6 + [PI32, PI32, I32, PD]

FUNCTION_SIGNATURES = [
    ("qk_abi_version", None, [ct.POINTER(I32), ct.POINTER(I32)]),
    ("qk_plugin_get_api", I32, [I32, I32, ct.POINTER(ct.POINTER(QKPluginAPI))]),
    ("qk_get_last_error", ct.c_char_p, []),
    ("qk_clear_last_error", None, []),
    ("qk_set_device", I32, [I32]),
    ("qk_get_device", I32, [PI32]),
    ("qk_mcm_standard_monte_carlo_price", D, _term_scalar),
    ("qk_mcm_standard_monte_carlo_price_batch", I32, _term_batch),
    ("qk_mcm_standard_monte_carlo_price_se_batch", I32, _term_batch + [PD]),
    ("qk_mcm_antithetic_variates_price", D, _term_scalar),
    ("qk_mcm_antithetic_variates_price_batch", I32, _term_batch),
    ("qk_mcm_antithetic_variates_price_se_batch", I32, _term_batch + [PD]),
    ("qk_mcm_euler_maruyama_price", D, _step_scalar),
    ("qk_mcm_euler_maruyama_price_batch", I32, _step_batch),
    ("qk_mcm_euler_maruyama_price_se_batch", I32, _step_batch + [PD]),
    ("qk_mcm_milstein_price", D, _step_scalar),
    ("qk_mcm_milstein_price_batch", I32, _step_batch),
    ("qk_mcm_milstein_price_se_batch", I32, _step_batch + [PD]),
    ("qk_mcm_local_vol_monte_carlo_price", D, _step_scalar),
    ("qk_mcm_local_vol_monte_carlo_price_batch", I32, _step_batch),
    ("qk_mcm_local_vol_monte_carlo_price_se_batch", I32, _step_batch + [PD]),
    ("qk_mcm_heston_monte_carlo_price", D, _hes_scalar),
    ("qk_mcm_heston_monte_carlo_price_batch", I32, _hes_batch),
    ("qk_mcm_heston_monte_carlo_price_se_batch", I32, _hes_batch + [PD]),
    ("qk_mcm_heston_monte_carlo_price_batch_noalloc", I32, _hes_batch + [PD]),
    ("qk_mcm_heston_lr_delta", D, _hes_scalar + [D]),
    ("qk_mcm_heston_lr_delta_batch", I32, [PD] * 10 + [PI32, PI32, PI32, PU64, PD, I32, PD]),
    ("qk_mcm_heston_lr_delta_se_batch", I32, [PD] * 10 + [PI32, PI32, PI32, PU64, PD, I32, PD, PD]),
    ("qk_mcm_control_variates_price", D, _term_scalar),
    ("qk_mcm_control_variates_price_batch", I32, _term_batch),
    ("qk_mcm_control_variates_price_se_batch", I32, _term_batch + [PD]),
    ("qk_mcm_importance_sampling_price", D, _is_scalar),
    ("qk_mcm_importance_sampling_price_batch", I32, _is_batch),
    ("qk_mcm_importance_sampling_price_se_batch", I32, _is_batch + [PD]),
    ("qk_mcm_stratified_sampling_price", D, _term_scalar),
    ("qk_mcm_stratified_sampling_price_batch", I32, _term_batch),
    ("qk_mcm_stratified_sampling_price_se_batch", I32, _term_batch + [PD]),
    ("qk_mcm_quasi_monte_carlo_sobol_price", D, _qmc_scalar),
    ("qk_mcm_quasi_monte_carlo_sobol_price_batch", I32, _qmc_batch),
    ("qk_mcm_quasi_monte_carlo_sobol_price_se_batch", I32, _qmc_batch + [PD]),
    ("qk_mcm_quasi_monte_carlo_halton_price", D, _qmc_scalar),
    ("qk_mcm_quasi_monte_carlo_halton_price_batch", I32, _qmc_batch),
    ("qk_mcm_quasi_monte_carlo_halton_price_se_batch", I32, _qmc_batch + [PD]),
    ("qk_cf_heston_price_cf", D, [D] * 10 + [I32, I32, D]),
    ("qk_ftm_cos_fang_oosterlee_heston_price", D, [D] * 10 + [I32, I32, D]),
    ("qk_ftm_cos_fang_oosterlee_heston_price_batch", I32, [PD] * 10 + [PI32, PI32, PD, I32, PD]),
    ("qk_cf_heston_price_cf_batch", I32, [PD] * 10 + [PI32, PI32, PD, I32, PD]),
    ("qk_mcm_mixed_price_batch", I32, _mixed_arrays + [PD, PD]),
    ("qk_mcm_plan_create", I32, _mixed_arrays + [I32, ct.POINTER(VP)]),
    ("qk_mcm_plan_execute", I32, [VP, VP]),
    ("qk_mcm_plan_results", I32, [VP, PD, PD]),
    ("qk_mcm_plan_device_results", I32, [VP, ct.POINTER(VP), ct.POINTER(VP)]),
    ("qk_mcm_plan_stats", I32, [VP, PD, PI32, PI64]),
    ("qk_mcm_plan_config", I32, [VP, PI32, PI32, PI32]),
    ("qk_mcm_plan_step_unroll", I32, [VP, PI32]),
    ("qk_mcm_plan_destroy", I32, [VP]),
    ("qk_dist_unique_id", I32, [VP]),
    ("qk_dist_create", I32, [VP, I32, I32, ct.POINTER(VP)]),
    ("qk_dist_info", I32, [VP, PI32, PI32, PI32]),
    ("qk_dist_abort", I32, [VP]),
    ("qk_dist_destroy", I32, [VP]),
    ("qk_dist_partition", I32, [PD, I64, I32, PI64]),
    ("qk_b200_pipe_probe", I32, [I32, I32, PD]),
    ("qk_mcm_plan_execute_sharded", I32, [VP, VP, VP]),
    ("qk_mcm_plan_shard_bounds", I32, [VP, I32, PI64]),
    ("qk_mcm_plan_execute_tiles", I32, [VP, I64, I64, VP]),
    ("qk_mcm_plan_device_partials", I32, [VP, ct.POINTER(VP), PI64, PI32]),
    ("qk_mcm_plan_finalize", I32, [VP, VP]),
    ("qk_mcm_mixed_price_batch_sharded", I32, [VP] + _mixed_arrays + [PD, PD]),
    ("qk_sur_gemm_bf16", I32, [VP, VP, VP, I32, I32, I32, I32, VP]),
    ("qk_sur_heston_create", I32, [PD, PD, U64, ct.POINTER(VP)]),
    ("qk_sur_heston_destroy", I32, [VP]),
    ("qk_sur_heston_set_dataset", I32, [VP, PD, PD, I64]),
    ("qk_sur_heston_train", I32, [VP, I32, I32, D, U64, PD]),
    ("qk_sur_heston_predict", I32, [VP, PD, I64, PD]),
    ("qk_sur_heston_predict_device", I32, [VP, VP, VP, I64, VP, VP]),
    ("qk_sur_heston_predict_device_layered", I32, [VP, VP, VP, I64, VP, VP]),
    ("qk_sur_heston_features", I32, [VP, PD, I64, VP, VP]),
    ("qk_sur_heston_features_device", I32, [VP, VP, I64, VP, VP, VP]),
    ("qk_sur_heston_gradients", I32, [VP, PD, PD, I32, PD, PD]),
    ("qk_sur_heston_parameters", I32, [VP, PD]),
    ("qk_sur_heston_set_parameters", I32, [VP, PD]),
    ("qk_sur_heston_save", I32, [VP, ct.c_char_p]),
    ("qk_sur_heston_load", I32, [VP, ct.c_char_p]),
    ("qk_sur_heston_price_batch", I32, [VP] + [PD] * 10 + [PI32, I32, I32, I32, U64, PD, PI32]),
]


def search_dirs() -> list[Path]:
    dirs: list[Path] = []
    env = os.environ.get("QK_B200_LIB_PATH")
    if env:
        dirs.append(Path(env))
    dirs.append(Path(__file__).resolve().parent)
    return dirs


def find_library() -> Path:
    for d in search_dirs():
        cand = d / LIB_NAME
        if cand.exists():
            return cand
    raise OSError(
        f"Cannot find {LIB_NAME}. Searched: {[str(d) for d in search_dirs()]}. "
        "Build it with `make -C quant-kernel_b200/csrc` (or __graft_entry__.build()), "
        "or set QK_B200_LIB_PATH."
    )


def configure(lib: ct.CDLL) -> None:
    for name, restype, argtypes in FUNCTION_SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes


def verify_abi(lib: ct.CDLL) -> None:
    major = ct.c_int32(-1)
    minor = ct.c_int32(-1)
    lib.qk_abi_version(ct.byref(major), ct.byref(minor))
    if major.value != ABI_MAJOR:
        raise RuntimeError(f"ABI major version mismatch: library={major.value}, expected={ABI_MAJOR}")
    if minor.value < ABI_MINOR:
        raise RuntimeError(f"ABI minor version too old: library={minor.value}, expected>={ABI_MINOR}")
    api = ct.POINTER(QKPluginAPI)()
    rc = lib.qk_plugin_get_api(ABI_MAJOR, ABI_MINOR, ct.byref(api))
    if rc != QK_OK or not api:
        raise RuntimeError(f"qk_plugin_get_api failed: rc={rc}")
    if api.contents.abi_major != ABI_MAJOR or api.contents.abi_minor < ABI_MINOR:
        raise RuntimeError("plugin API version mismatch")


_LIB = None


def load_library() -> ct.CDLL:
    """Load libqk_b200.so once per process, bind every symbol and check the ABI."""
    global _LIB
    if _LIB is None:
        lib = ct.CDLL(str(find_library()))
        configure(lib)
        verify_abi(lib)
        _LIB = lib
    return _LIB
