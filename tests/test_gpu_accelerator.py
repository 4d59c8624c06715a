"""QuantAccelerator on the GPU: each routed batch equals the direct batch call
bit for bit, and a heterogeneous request list priced in one mixed launch
equals the per-method batches."""

import numpy as np
import pytest

from quantkernel_b200 import QK_CALL, QK_PUT, QuantAccelerator

pytestmark = pytest.mark.gpu

FOURIER = ("heston_price_cf", "cos_method_fang_oosterlee_heston_price")


def _jobs(method, n, rng):
    out = []
    for i in range(n):
        j = dict(spot=float(rng.uniform(90, 110)), strike=float(rng.uniform(90, 110)),
                 t=float(rng.uniform(0.25, 1.5)), r=float(rng.uniform(0.0, 0.05)),
                 q=float(rng.uniform(0.0, 0.02)), option_type=QK_CALL if i % 2 == 0 else QK_PUT)
        heston = method in ("heston_monte_carlo_price", "heston_lr_delta", "heston_price_cf",
                            "cos_method_fang_oosterlee_heston_price")
        if heston:
            j.update(v0=float(rng.uniform(0.02, 0.08)), kappa=float(rng.uniform(1, 3)),
                     theta=float(rng.uniform(0.02, 0.08)), sigma=float(rng.uniform(0.2, 0.6)),
                     rho=float(rng.uniform(-0.8, -0.2)))
        else:
            j["vol"] = float(rng.uniform(0.15, 0.4))
        if method not in FOURIER:
            j["paths"] = int(rng.integers(2000, 20000))
            if method not in ("quasi_monte_carlo_sobol_price", "quasi_monte_carlo_halton_price"):
                j["seed"] = int(rng.integers(0, 2**40))
        if method in ("euler_maruyama_price", "milstein_price", "local_vol_monte_carlo_price",
                      "heston_monte_carlo_price", "heston_lr_delta"):
            j["steps"] = int(rng.integers(8, 64))
        if method == "importance_sampling_price":
            j["shift"] = float(rng.uniform(0.0, 0.5))
        if method == "heston_lr_delta":
            j["weight_clip"] = 6.0
        out.append(j)
    return out


METHODS = list(QuantAccelerator._NATIVE_BATCH_METHODS)


@pytest.mark.parametrize("method", METHODS)
def test_price_batch_equals_direct_batch(qk, method):
    accel = QuantAccelerator(qk=qk, backend="gpu")
    assert accel.gpu_available
    jobs = _jobs(method, 9, np.random.default_rng(sum(map(ord, method))))
    got = accel.price_batch(method, jobs)
    cols = accel._columns(method, jobs)
    want = getattr(qk, accel._NATIVE_BATCH_METHODS[method])(**cols)
    assert np.array_equal(got, want)
    # and the scalar call for the first job
    assert getattr(qk, method)(**jobs[0]) == got[0]


def test_price_many_mixed_launch_equals_per_method_batches(qk):
    accel = QuantAccelerator(qk=qk)
    rng = np.random.default_rng(7)
    requests = []
    for method in METHODS:
        for job in _jobs(method, 5, rng):
            requests.append((method, job))
    order = rng.permutation(len(requests))
    requests = [requests[i] for i in order]
    prices, se = accel.price_many(requests, with_stderr=True)
    for method in METHODS:
        idx = [i for i, (m, _) in enumerate(requests) if m == method]
        want = accel.price_batch(method, [requests[i][1] for i in idx])
        # double-double sums make results independent of the launch shape up to
        # the final rounding; the control-variate moments are plain FP64
        np.testing.assert_allclose(prices[idx], want, rtol=1e-13, atol=0, err_msg=method)
        if method in FOURIER:
            assert np.all(np.isnan(se[idx]))
        else:
            assert np.all(se[idx] >= 0), method
