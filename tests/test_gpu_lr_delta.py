"""Heston likelihood-ratio delta on the GPU: the reference's own tests
(python/tests/test_heston_lr_delta.py: finite-difference bump, seed
determinism, batch == scalar, bounds) with their cases and tolerances, and
statistical parity with the reference's CPU estimator (through the oracle)."""

import math

import numpy as np
import pytest
from scipy import stats

from quantkernel_b200 import QK_CALL, QK_PUT, workloads

pytestmark = pytest.mark.gpu

_HESTON = dict(strike=100.0, t=1.0, r=0.05, q=0.02, v0=0.04, kappa=2.0, theta=0.04, sigma=0.3,
               rho=-0.7, paths=40000, steps=80, seed=42, weight_clip=6.0)
_PRICE_KEYS = ("strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho", "paths", "steps", "seed")


@pytest.mark.parametrize("ot", [QK_CALL, QK_PUT])
def test_delta_matches_finite_difference_bump(qk, ot):
    spot, eps = 100.0, 0.5
    lr = qk.heston_lr_delta(spot=spot, option_type=ot, **_HESTON)
    pk = {k: _HESTON[k] for k in _PRICE_KEYS}
    up = qk.heston_monte_carlo_price(spot=spot + eps, option_type=ot, **pk)
    dn = qk.heston_monte_carlo_price(spot=spot - eps, option_type=ot, **pk)
    fd = (up - dn) / (2 * eps)
    assert math.isfinite(lr) and math.isfinite(fd)
    assert abs(lr - fd) < 0.15, (lr, fd)


def test_seed_determinism_and_sensitivity(qk):
    p = dict(spot=100.0, option_type=QK_CALL, **{**_HESTON, "seed": 777})
    assert qk.heston_lr_delta(**p) == qk.heston_lr_delta(**p)
    base = dict(spot=100.0, option_type=QK_CALL, **{k: v for k, v in _HESTON.items() if k != "seed"})
    assert qk.heston_lr_delta(**base, seed=42) != qk.heston_lr_delta(**base, seed=999)


def test_batch_matches_scalar(qk):
    params = [dict(spot=100.0, option_type=QK_CALL, **_HESTON),
              dict(spot=110.0, option_type=QK_PUT, **{**_HESTON, "seed": 99})]
    scal = [qk.heston_lr_delta(**p) for p in params]
    bat = qk.heston_lr_delta_batch(**{k: [p[k] for p in params] for k in params[0]})
    for i, s in enumerate(scal):
        assert abs(bat[i] - s) < 1e-12


@pytest.mark.parametrize("spot", [80.0, 100.0, 120.0])
def test_delta_in_range(qk, spot):
    c = qk.heston_lr_delta(spot=spot, option_type=QK_CALL, **_HESTON)
    p = qk.heston_lr_delta(spot=spot, option_type=QK_PUT, **_HESTON)
    assert math.isfinite(c) and -0.1 <= c <= 1.1
    assert math.isfinite(p) and -1.1 <= p <= 0.1


def test_entry_checks(qk):
    base = dict(spot=100.0, option_type=QK_CALL, **_HESTON)
    assert qk.heston_lr_delta(**{**base, "t": 1e-14, "spot": 110.0}) == 1.0
    assert qk.heston_lr_delta(**{**base, "t": 1e-14, "spot": 90.0, "option_type": QK_PUT}) == -1.0
    assert qk.heston_lr_delta(**{**base, "v0": 0.0}) == 0.0
    with pytest.raises(ValueError):
        qk.heston_lr_delta(**{**base, "weight_clip": 0.0})


def test_parity_with_reference_cpu_estimator(qk, oracle):
    h = workloads.heston(24, paths=20000, steps=40, seed=13)
    h["option_type"] = (np.arange(24) & 1).astype(np.int32)
    clip = np.full(24, 6.0)
    d, se = qk.heston_lr_delta_se_batch(**h, weight_clip=clip)
    ref = [oracle.price(7, h["spot"][i], h["strike"][i], h["t"][i], 6.0, h["r"][i], h["q"][i],
                        int(h["option_type"][i]), int(h["paths"][i]), int(h["steps"][i]),
                        int(h["seed"][i]), h["v0"][i], h["kappa"][i], h["theta"][i],
                        h["sigma"][i], h["rho"][i]) for i in range(24)]
    cp = np.array([x[0] for x in ref])
    cse = np.array([x[1] for x in ref])
    z = (d - cp) / np.hypot(se, cse)
    allowed = int(stats.binom.ppf(0.999, 24, 0.0027))
    print(f"LR delta GPU vs reference CPU: max|z| {np.abs(z).max():.2f}, mean z {z.mean():+.3f}")
    assert int((np.abs(z) > 3).sum()) <= allowed and np.abs(z).max() < 5
