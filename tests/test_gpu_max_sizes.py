"""Index arithmetic at the ABI's limits: path counts up to INT32_MAX (the
reference's `int32_t paths`), a million options in one batch, and the
4096-tile-per-option cap."""

import math

import numpy as np
import pytest

from quantkernel_b200 import workloads

pytestmark = pytest.mark.gpu

MAX_PATHS = 2**31 - 1


def _one(**kw):
    base = dict(spot=100.0, strike=105.0, t=1.0, vol=0.2, r=0.03, q=0.01, option_type=0)
    base.update(kw)
    return {k: np.array([v]) if not isinstance(v, np.ndarray) else v for k, v in base.items()}


def test_terminal_at_int32_max_paths(qk, oracle):
    """2^31 - 1 paths: antithetic (1.07e9 normals) and plain (2.1e9 normals,
    unit indices up to 2^29) both price to the closed form within 5 SE."""
    cf = oracle.bsm(100.0, 105.0, 1.0, 0.2, 0.03, 0.01, 0)
    a = _one(paths=np.array([MAX_PATHS], np.int32), seed=np.array([3], np.uint64))
    p, se = qk.standard_monte_carlo_price_se_batch(**a)
    assert se[0] > 0 and abs(p[0] - cf) < 5 * se[0] + 1e-4, (p, se, cf)
    model = np.array([5], np.int32)  # independent paths
    plan = qk.plan(model=model, **a)
    plan.execute()
    p5, se5 = plan.results()
    plan.close()
    assert abs(p5[0] - cf) < 5 * se5[0] + 1e-4, (p5, se5, cf)


def test_qmc_and_stratified_at_int32_max_paths(qk, oracle):
    cf = oracle.bsm(100.0, 105.0, 1.0, 0.2, 0.03, 0.01, 0)
    a = _one(paths=np.array([MAX_PATHS], np.int32))
    for fn in (qk.quasi_monte_carlo_sobol_price_batch, qk.quasi_monte_carlo_halton_price_batch):
        p = fn(**a)
        assert abs(p[0] - cf) < 1e-5, (fn.__name__, p, cf)
    s = qk.stratified_sampling_price_batch(**a, seed=np.array([9], np.uint64))
    assert abs(s[0] - cf) < 1e-5, (s, cf)


def test_million_option_batch(qk, oracle):
    """1e6 options of 64 paths each: tile offsets past 2^20, option search over
    1e6 records; every price matches the same option priced alone."""
    n = 1_000_000
    b = workloads.bsm_terminal(n, paths=64, seed=17)
    p = qk.standard_monte_carlo_price_batch(**b)
    assert np.all(np.isfinite(p))
    for i in (0, 1, 777_777, n - 1):
        one = qk.standard_monte_carlo_price(*(b[k][i].item() for k in ("spot", "strike", "t", "vol",
                                                                        "r", "q", "option_type",
                                                                        "paths", "seed")))
        assert one == p[i], i


def test_tile_cap_for_long_options(qk):
    """An option with more units than 4096 tiles' worth gets several units per
    thread (unit_iters > 1); the result equals the scalar call and the closed
    form within 5 SE."""
    h = workloads.heston(2, paths=1 << 24, steps=8, seed=5)
    p, se = qk.heston_monte_carlo_price_se_batch(**h)
    assert np.all(se > 0) and np.all(np.isfinite(p))
    one = qk.heston_monte_carlo_price(*(h[k][1].item() for k in ("spot", "strike", "t", "r", "q",
                                                                  "v0", "kappa", "theta", "sigma",
                                                                  "rho", "option_type", "paths",
                                                                  "steps", "seed")))
    assert one == p[1]
    assert math.isfinite(one)


def test_step_counts_past_the_cap_are_invalid(qk):
    """Step counts within 64 of INT32_MAX (over 2.1e9 steps per path) would
    wrap the kernels' int32 step-block index; they price as invalid input
    (NaN), like a non-positive count, without launching a simulation."""
    for steps in (MAX_PATHS, MAX_PATHS - 63):
        a = _one(paths=np.array([1000], np.int32), steps=np.array([steps], np.int32),
                 seed=np.array([1], np.uint64))
        p, se = qk.euler_maruyama_price_se_batch(**a)
        assert np.isnan(p[0]) and np.isnan(se[0])
        h = dict(spot=np.array([100.0]), strike=np.array([100.0]), t=np.array([1.0]),
                 r=np.array([0.03]), q=np.array([0.0]), v0=np.array([0.04]),
                 kappa=np.array([2.0]), theta=np.array([0.04]), sigma=np.array([0.3]),
                 rho=np.array([-0.7]), option_type=np.array([0], np.int32),
                 paths=np.array([1000], np.int32), steps=np.array([steps], np.int32),
                 seed=np.array([1], np.uint64))
        p, se = qk.heston_monte_carlo_price_se_batch(**h)
        assert np.isnan(p[0]) and np.isnan(se[0])
