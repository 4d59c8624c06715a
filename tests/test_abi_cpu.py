"""C-ABI boundary checks that need no GPU: the library loads, exports every
symbol include/qk_api.h declares, negotiates its ABI, and reports argument
errors exactly as the reference does (cpp/tests/test_error_handling.cpp:5-108,
python/tests/test_abi_version.py).  No call here reaches a kernel: the null
and size checks return before any CUDA call."""

import ctypes as ct
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "qk_api.h"
HEADERS = sorted((ROOT / "include").glob("*.h"))


def _declared_functions():
    text = "".join(h.read_text() for h in HEADERS)
    return sorted(set(re.findall(r"QK_EXPORT\s+[\w\s\*]+?\b(qk_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(qk):
    names = _declared_functions()
    assert len(names) >= 28
    for name in names:
        assert hasattr(qk._lib, name), f"{name} declared in include/ but not exported"


def test_loader_binds_every_declared_symbol():
    from quantkernel_b200._loader import FUNCTION_SIGNATURES

    bound = {name for name, _, _ in FUNCTION_SIGNATURES}
    assert set(_declared_functions()) == bound


def test_drop_in_signatures_match_reference_subset():
    """Every reference MC batch/scalar entry on the hot path is declared here."""
    text = HEADER.read_text()
    for name in [
        "qk_mcm_control_variates_price", "qk_mcm_control_variates_price_batch",
        "qk_mcm_importance_sampling_price", "qk_mcm_importance_sampling_price_batch",
        "qk_mcm_stratified_sampling_price", "qk_mcm_stratified_sampling_price_batch",
        "qk_mcm_quasi_monte_carlo_sobol_price", "qk_mcm_quasi_monte_carlo_sobol_price_batch",
        "qk_mcm_quasi_monte_carlo_halton_price", "qk_mcm_quasi_monte_carlo_halton_price_batch",
        "qk_cf_heston_price_cf", "qk_cf_heston_price_cf_batch",
        "qk_ftm_cos_fang_oosterlee_heston_price", "qk_ftm_cos_fang_oosterlee_heston_price_batch",
        "qk_mcm_standard_monte_carlo_price", "qk_mcm_standard_monte_carlo_price_batch",
        "qk_mcm_antithetic_variates_price", "qk_mcm_antithetic_variates_price_batch",
        "qk_mcm_euler_maruyama_price", "qk_mcm_euler_maruyama_price_batch",
        "qk_mcm_milstein_price", "qk_mcm_milstein_price_batch",
        "qk_mcm_heston_monte_carlo_price", "qk_mcm_heston_monte_carlo_price_batch",
        "qk_mcm_local_vol_monte_carlo_price", "qk_mcm_local_vol_monte_carlo_price_batch",
        "qk_abi_version", "qk_plugin_get_api", "qk_get_last_error", "qk_clear_last_error",
    ]:
        assert re.search(rf"\b{name}\s*\(", text), name


def test_abi_version_and_plugin_negotiation(qk):
    from quantkernel_b200 import ABI_MAJOR, ABI_MINOR

    assert qk.abi_version() == (2, 13)
    major, minor, name = qk.plugin_get_api()
    assert (major, minor) == (ABI_MAJOR, ABI_MINOR) and name
    # host asks for a newer minor or a different major -> QK_ERR_ABI_MISMATCH
    from quantkernel_b200._loader import QKPluginAPI

    out = ct.POINTER(QKPluginAPI)()
    assert qk._lib.qk_plugin_get_api(3, 0, ct.byref(out)) == -3 and not out
    assert qk._lib.qk_plugin_get_api(2, 99, ct.byref(out)) == -3
    assert qk._lib.qk_plugin_get_api(2, 12, ct.byref(out)) == 0 and out
    assert qk._lib.qk_plugin_get_api(2, 12, None) == -1


PD = ct.POINTER(ct.c_double)


def _arrays(n=1):
    d = np.full(n, 1.0)
    i = np.ones(n, np.int32)
    u = np.ones(n, np.uint64)
    return d, i, u


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(ct.POINTER({np.float64: ct.c_double, np.int32: ct.c_int32,
                                        np.uint64: ct.c_uint64}[a.dtype.type]))


# name -> (argument names in declaration order, kind of each)
BATCHES = {
    "qk_mcm_standard_monte_carlo_price_batch": "spot strike t vol r q option_type paths seed",
    "qk_mcm_antithetic_variates_price_batch": "spot strike t vol r q option_type paths seed",
    "qk_mcm_euler_maruyama_price_batch": "spot strike t vol r q option_type paths steps seed",
    "qk_mcm_milstein_price_batch": "spot strike t vol r q option_type paths steps seed",
    "qk_mcm_local_vol_monte_carlo_price_batch": "spot strike t vol r q option_type paths steps seed",
    "qk_mcm_heston_monte_carlo_price_batch":
        "spot strike t r q v0 kappa theta sigma rho option_type paths steps seed",
    "qk_cf_heston_price_cf_batch":
        "spot strike t r q v0 kappa theta sigma rho option_type integration_steps "
        "integration_limit",
    "qk_ftm_cos_fang_oosterlee_heston_price_batch":
        "spot strike t r q v0 kappa theta sigma rho option_type n_terms truncation_width",
    "qk_mcm_control_variates_price_batch": "spot strike t vol r q option_type paths seed",
    "qk_mcm_stratified_sampling_price_batch": "spot strike t vol r q option_type paths seed",
    "qk_mcm_importance_sampling_price_batch":
        "spot strike t vol r q option_type paths shift seed",
    "qk_mcm_quasi_monte_carlo_sobol_price_batch": "spot strike t vol r q option_type paths",
    "qk_mcm_quasi_monte_carlo_halton_price_batch": "spot strike t vol r q option_type paths",
}
MC_BATCHES = sorted(k for k in BATCHES if k.startswith("qk_mcm_"))
INT_ARGS = {"option_type", "paths", "steps", "integration_steps", "n_terms"}


def _call(qk, fn, names, null=None, n=1, out=True, se=None):
    d, i, u = _arrays(max(n, 1))
    args = []
    for nm in names.split():
        if nm == null:
            args.append(None)
        elif nm in INT_ARGS:
            args.append(_p(i))
        elif nm == "seed":
            args.append(_p(u))
        else:
            args.append(_p(d))
    outa = np.empty(max(n, 1))
    args += [n, _p(outa) if out else None]
    if se is not None:
        args.append(_p(np.empty(max(n, 1))) if se else None)
    return getattr(qk._lib, fn)(*args)


@pytest.mark.parametrize("fn", sorted(BATCHES))
def test_null_pointer_identifies_first_null_parameter(qk, fn):
    names = BATCHES[fn]
    for nm in names.split():
        qk.clear_last_error()
        assert _call(qk, fn, names, null=nm) == -1
        msg = qk.get_last_error()
        assert msg == f"null pointer: {nm}", (fn, nm, msg)
    qk.clear_last_error()
    assert _call(qk, fn, names, out=False) == -1
    assert qk.get_last_error() == "null pointer: out_prices"
    # null is checked before size (qk_api.cpp:1149-1151)
    assert _call(qk, fn, names, null="spot", n=0) == -1


@pytest.mark.parametrize("fn", sorted(BATCHES))
@pytest.mark.parametrize("n", [0, -3])
def test_bad_size(qk, fn, n):
    qk.clear_last_error()
    assert _call(qk, fn, BATCHES[fn], n=n) == -2
    assert qk.get_last_error() == f"bad batch size: {n}"


@pytest.mark.parametrize("fn", MC_BATCHES)
def test_se_batch_checks_out_stderr(qk, fn):
    se_fn = fn.replace("_price_batch", "_price_se_batch")
    qk.clear_last_error()
    assert _call(qk, se_fn, BATCHES[fn], se=False) == -1
    assert qk.get_last_error() == "null pointer: out_stderr"
    assert _call(qk, se_fn, BATCHES[fn], n=0, se=True) == -2


def test_clear_error_works(qk):
    _call(qk, "qk_mcm_heston_monte_carlo_price_batch", BATCHES["qk_mcm_heston_monte_carlo_price_batch"], n=-1)
    assert qk.get_last_error() != ""
    qk.clear_last_error()
    assert qk.get_last_error() == ""


def test_python_errors_map_like_reference(qk):
    from quantkernel_b200 import QKBadSizeError

    with pytest.raises(QKBadSizeError):
        qk.heston_monte_carlo_price_batch(*([[]] * 14))
    with pytest.raises(ValueError, match="length mismatch"):
        qk.euler_maruyama_price_batch([100, 100], [100], [1], [0.2], [0.05], [0], [0], [10], [10], [1])
    with pytest.raises(ValueError, match="1D"):
        qk.standard_monte_carlo_price_batch([[100]], [100], [1], [0.2], [0.05], [0], [0], [10], [1])


@pytest.mark.parametrize("call", [
    lambda qk: qk.control_variates_price_batch([100, 100], [100], [1], [0.2], [0.05], [0], [0],
                                               [10], [1]),
    lambda qk: qk.stratified_sampling_price_batch([100], [100], [1], [0.2], [0.05], [0], [0],
                                                  [10, 10], [1]),
    lambda qk: qk.importance_sampling_price_batch([100], [100], [1], [0.2], [0.05], [0], [0], [10],
                                                  [0.1, 0.2], [1]),
    lambda qk: qk.quasi_monte_carlo_sobol_price_batch([100], [100, 90], [1], [0.2], [0.05], [0],
                                                      [0], [10]),
    lambda qk: qk.quasi_monte_carlo_halton_price_batch([100], [100], [1], [0.2], [0.05], [0],
                                                       [0, 1], [10]),
    lambda qk: qk.heston_price_cf_batch([100], [100], [1], [0.05], [0], [0.04], [2], [0.04], [0.3],
                                        [-0.7], [0], [1024], [120.0, 80.0]),
])
def test_ragged_inputs_rejected_before_the_library(qk, call):
    """Ragged arrays are a caller error the Python layer reports (ValueError)
    before any C call, as the reference engine does (engine.py:120-141)."""
    with pytest.raises(ValueError, match="length mismatch"):
        call(qk)


@pytest.mark.parametrize("fn,nargs", [("control_variates_price_batch", 9),
                                      ("importance_sampling_price_batch", 10),
                                      ("stratified_sampling_price_batch", 9),
                                      ("quasi_monte_carlo_sobol_price_batch", 8),
                                      ("quasi_monte_carlo_halton_price_batch", 8),
                                      ("heston_price_cf_batch", 13)])
def test_empty_batches_are_bad_size(qk, fn, nargs):
    from quantkernel_b200 import QKBadSizeError

    with pytest.raises(QKBadSizeError):
        getattr(qk, fn)(*([[]] * nargs))


def test_mixed_batch_requires_arrays_its_models_use(qk):
    n = 2
    model = np.array([2, 6], np.int32)
    d = np.ones(n)
    i = np.ones(n, np.int32)
    u = np.ones(n, np.uint64)
    out = np.empty(n)
    base = [_p(model), _p(d), _p(d), _p(d), _p(d), _p(d), _p(d)]
    # v0 missing while a Heston option is present
    rc = qk._lib.qk_mcm_mixed_price_batch(*base, None, _p(d), _p(d), _p(d), _p(d), _p(i), _p(i),
                                          _p(i), _p(u), n, _p(out), None)
    assert rc == -1 and qk.get_last_error() == "null pointer: v0"
    rc = qk._lib.qk_mcm_mixed_price_batch(*base, _p(d), _p(d), _p(d), _p(d), _p(d), _p(i), _p(i),
                                          _p(i), _p(u), 0, _p(out), None)
    assert rc == -2
    # importance sampling reads its shift from v0; the QMC models need no seed
    # but the mixed call checks it for every batch
    model2 = np.array([11, 9], np.int32)
    base2 = [_p(model2)] + base[1:]
    rc = qk._lib.qk_mcm_mixed_price_batch(*base2, None, None, None, None, None, _p(i), _p(i),
                                          None, _p(u), n, _p(out), None)
    assert rc == -1 and qk.get_last_error() == "null pointer: v0"


def test_no_gpu_means_runtime_error_not_cpu_fallback(qk):
    """Without a usable GPU a valid batch fails loudly (QK_ERR_RUNTIME_INIT)."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    qk.clear_last_error()
    rc = _call(qk, "qk_mcm_heston_monte_carlo_price_batch",
               BATCHES["qk_mcm_heston_monte_carlo_price_batch"])
    assert rc == -4
    assert qk.get_last_error().startswith("cuda error")
    p = qk._lib.qk_mcm_heston_monte_carlo_price(100, 100, 1, 0.05, 0, 0.04, 2, 0.04, 0.3, -0.7,
                                                0, 100, 10, 1)
    assert np.isnan(p)
    qk.clear_last_error()
    rc = _call(qk, "qk_cf_heston_price_cf_batch", BATCHES["qk_cf_heston_price_cf_batch"])
    assert rc == -4 and qk.get_last_error().startswith("cuda error")
    assert np.isnan(qk._lib.qk_cf_heston_price_cf(100, 100, 1, 0.03, 0, 0.04, 2, 0.04, 0.3, -0.7,
                                                   0, 1024, 120.0))
