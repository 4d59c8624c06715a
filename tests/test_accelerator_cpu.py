"""QuantAccelerator routing (host logic; no kernel runs here).

The reference's accelerator tests (python/tests/test_accelerator.py) check
strategy selection, unknown methods, empty batches and that backend='gpu'
never silently falls back to the CPU; the same properties hold here, with
the GPU library as the only backend.
"""

import numpy as np
import pytest

from quantkernel_b200 import QK_CALL, QKRuntimeError, QuantAccelerator

MC_METHODS = [
    "standard_monte_carlo_price", "antithetic_variates_price", "euler_maruyama_price",
    "milstein_price", "local_vol_monte_carlo_price", "heston_monte_carlo_price",
    "heston_lr_delta", "importance_sampling_price", "control_variates_price",
    "stratified_sampling_price", "quasi_monte_carlo_sobol_price",
    "quasi_monte_carlo_halton_price",
]


def test_native_batch_for_every_supported_method(qk):
    accel = QuantAccelerator(qk=qk, backend="gpu")
    for m in MC_METHODS + ["heston_price_cf", "cos_method_fang_oosterlee_heston_price"]:
        assert accel.suggest_strategy(m, 1) == "native_batch"
        assert accel.suggest_strategy(m, 100000) == "native_batch"
        assert hasattr(qk, accel._NATIVE_BATCH_METHODS[m])


def test_unsupported_and_unknown_methods(qk):
    accel = QuantAccelerator(qk=qk)
    with pytest.raises(RuntimeError, match="not supported"):
        accel.suggest_strategy("crr_price", 10)
    with pytest.raises(AttributeError):
        accel.price_batch("nope", [{"x": 1.0}])
    with pytest.raises(AttributeError):
        accel.price_many([("nope", {"x": 1.0})])


def test_cpu_backend_refused(qk):
    with pytest.raises(RuntimeError, match="GPU only"):
        QuantAccelerator(qk=qk, backend="cpu")
    with pytest.raises(ValueError):
        QuantAccelerator(qk=qk, backend="tpu")


def test_empty_batches(qk):
    accel = QuantAccelerator(qk=qk)
    out = accel.price_batch("heston_monte_carlo_price", [])
    assert out.shape == (0,) and out.dtype == np.float64
    p, se = accel.price_many([], with_stderr=True)
    assert p.shape == (0,) and se.shape == (0,)


def test_job_columns_take_scalar_defaults(qk):
    accel = QuantAccelerator(qk=qk)
    jobs = [{"spot": 100.0, "strike": 100.0, "t": 1.0, "vol": 0.2, "r": 0.03, "q": 0.0,
             "option_type": QK_CALL, "paths": 1000}]
    cols = accel._columns("standard_monte_carlo_price", jobs)
    assert cols["seed"] == [42]
    cf = accel._columns("heston_price_cf", [{"spot": 100.0}])
    assert cf["integration_steps"] == [1024] and cf["integration_limit"] == [120.0]
    cos = accel._columns("cos_method_fang_oosterlee_heston_price", [{"spot": 100.0}])
    assert cos["n_terms"] == [256] and cos["truncation_width"] == [10.0]


def test_no_gpu_raises_instead_of_cpu_result(qk):
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    accel = QuantAccelerator(qk=qk)
    assert not accel.gpu_available
    job = {"spot": 100.0, "strike": 100.0, "t": 1.0, "vol": 0.2, "r": 0.03, "q": 0.0,
           "option_type": QK_CALL, "paths": 1000, "seed": 1}
    with pytest.raises(QKRuntimeError):
        accel.price_batch("standard_monte_carlo_price", [job])
    with pytest.raises(QKRuntimeError):
        accel.price_many([("standard_monte_carlo_price", job)])
