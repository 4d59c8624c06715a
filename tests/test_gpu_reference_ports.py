"""The reference's own Monte Carlo tests, ported to the GPU library with their
cases and tolerances unchanged:

  cpp/tests/test_monte_carlo.cpp:5-46          positivity, near BSM, batch == scalar
  python/tests/test_monte_carlo_api.py:28-125  BSM consistency, Heston vs CF,
                                               Heston batch == scalar, determinism,
                                               antithetic odd/even path counts
  python/tests/test_heston_mc_invariants.py    bounds, monotonicity, vol-of-vol,
                                               finiteness, t -> 0, extreme rho
  python/tests/test_local_vol_monte_carlo.py   LV vs Euler, vs BSM, bounds,
                                               monotonicity, determinism, batch == scalar
  python/tests/test_batch_api.py:83-96,247-268,336-356  batch == scalar (1e-12)

The golden-seed values of test_monte_carlo.cpp:57-73 pin the mt19937 stream,
which a GPU counter-based generator does not reproduce; they pin the CPU
oracle instead (tests/test_oracle_golden.py).
"""

import math

import numpy as np
import pytest

from quantkernel_b200 import QK_CALL, QK_PUT

pytestmark = pytest.mark.gpu


# ---------------------------------------------------------------- test_monte_carlo.cpp
def test_standard_mc_positive_and_near_bsm(qk, oracle):
    price = qk.standard_monte_carlo_price(100.0, 100.0, 1.0, 0.2, 0.05, 0.0, QK_CALL, 100000, 42)
    assert price > 0.0
    bsm = oracle.bsm(100.0, 100.0, 1.0, 0.2, 0.05, 0.0, QK_CALL)
    mc = qk.standard_monte_carlo_price(100.0, 100.0, 1.0, 0.2, 0.05, 0.0, QK_CALL, 500000, 42)
    assert abs(mc - bsm) < 0.5


def test_euler_milstein_positive(qk):
    assert qk.euler_maruyama_price(100.0, 100.0, 1.0, 0.2, 0.05, 0.0, QK_CALL, 10000, 100, 42) > 0
    assert qk.milstein_price(100.0, 100.0, 1.0, 0.2, 0.05, 0.0, QK_PUT, 10000, 100, 42) > 0


def test_standard_mc_batch_matches_scalar(qk):
    spot = [100, 105, 95, 110]
    strike = [100, 100, 100, 100]
    t = [1.0, 1.0, 1.0, 0.5]
    vol = [0.2, 0.2, 0.3, 0.2]
    r = [0.05] * 4
    q = [0.0, 0.0, 0.0, 0.02]
    ot = [QK_CALL, QK_PUT, QK_CALL, QK_PUT]
    paths = [10000] * 4
    seed = [42, 43, 44, 45]
    out = qk.standard_monte_carlo_price_batch(spot, strike, t, vol, r, q, ot, paths, seed)
    for i in range(4):
        s = qk.standard_monte_carlo_price(spot[i], strike[i], t[i], vol[i], r[i], q[i], ot[i],
                                          paths[i], seed[i])
        assert abs(out[i] - s) < 1e-12


# ---------------------------------------------------------------- test_monte_carlo_api.py
def test_monte_carlo_prices_are_consistent_with_bsm(qk, oracle):
    common = dict(spot=100.0, strike=100.0, t=1.0, vol=0.2, r=0.03, q=0.01, option_type=QK_CALL)
    bsm = oracle.bsm(**common)
    mc = qk.standard_monte_carlo_price(**common, paths=60000, seed=11)
    anti = qk.antithetic_variates_price(**common, paths=60000, seed=11)
    assert abs(mc - bsm) < 0.8
    assert abs(anti - bsm) < 0.6


def test_heston_monte_carlo_price_is_finite_and_close_to_cf(qk, oracle):
    hp = dict(spot=100.0, strike=100.0, t=1.0, r=0.05, q=0.02, v0=0.04, kappa=2.0, theta=0.04,
              sigma=0.3, rho=-0.7, option_type=QK_CALL)
    mc = qk.heston_monte_carlo_price(**hp, paths=50000, steps=100, seed=42)
    cf = oracle.heston_cf(**hp)
    assert math.isfinite(mc) and mc > 0.0
    assert abs(mc - cf) < 1.5


def test_heston_monte_carlo_price_batch_matches_scalar(qk):
    params = [
        dict(spot=100.0, strike=100.0, t=1.0, r=0.05, q=0.02, v0=0.04, kappa=2.0, theta=0.04,
             sigma=0.3, rho=-0.7, option_type=QK_CALL, paths=5000, steps=50, seed=42),
        dict(spot=110.0, strike=100.0, t=0.5, r=0.03, q=0.01, v0=0.09, kappa=1.5, theta=0.06,
             sigma=0.4, rho=-0.5, option_type=QK_PUT, paths=5000, steps=50, seed=99),
    ]
    scalars = [qk.heston_monte_carlo_price(**p) for p in params]
    batch = qk.heston_monte_carlo_price_batch(**{k: [p[k] for p in params] for k in params[0]})
    for i, s in enumerate(scalars):
        assert abs(batch[i] - s) < 1e-12


def test_heston_monte_carlo_deterministic_seed(qk):
    common = dict(spot=100.0, strike=100.0, t=1.0, r=0.05, q=0.02, v0=0.04, kappa=2.0,
                  theta=0.04, sigma=0.3, rho=-0.7, option_type=QK_CALL, paths=10000, steps=50,
                  seed=777)
    assert qk.heston_monte_carlo_price(**common) == qk.heston_monte_carlo_price(**common)


def test_antithetic_uses_all_requested_paths(qk):
    common = dict(spot=100.0, strike=100.0, t=1.0, vol=0.2, r=0.03, q=0.01, option_type=QK_CALL,
                  seed=123)
    even = qk.antithetic_variates_price(**common, paths=2)
    odd = qk.antithetic_variates_price(**common, paths=3)
    assert abs(odd - even) > 1e-12


# ---------------------------------------------------------------- test_heston_mc_invariants.py
_BASE = dict(strike=100.0, t=1.0, r=0.05, q=0.02, v0=0.04, kappa=2.0, theta=0.04, sigma=0.3,
             rho=-0.7, paths=20000, steps=80, seed=314)


@pytest.mark.parametrize("spot", [80.0, 100.0, 120.0])
def test_heston_call_put_bounded(qk, spot):
    c = qk.heston_monte_carlo_price(spot=spot, option_type=QK_CALL, **_BASE)
    assert 0.0 <= c <= spot
    upper = _BASE["strike"] * math.exp(-_BASE["r"] * _BASE["t"])
    p = qk.heston_monte_carlo_price(spot=spot, option_type=QK_PUT, **_BASE)
    assert 0.0 <= p <= upper


def test_heston_monotone_in_spot(qk):
    spots = [80.0, 90.0, 100.0, 110.0, 120.0]
    calls = [qk.heston_monte_carlo_price(spot=s, option_type=QK_CALL, **_BASE) for s in spots]
    puts = [qk.heston_monte_carlo_price(spot=s, option_type=QK_PUT, **_BASE) for s in spots]
    for i in range(len(spots) - 1):
        assert calls[i + 1] >= calls[i] - 0.5
        assert puts[i + 1] <= puts[i] + 0.5


@pytest.mark.parametrize("ot", [QK_CALL, QK_PUT])
def test_heston_nondecreasing_in_vol_of_vol(qk, ot):
    base = dict(_BASE, spot=100.0, option_type=ot)
    lo = qk.heston_monte_carlo_price(**{**base, "sigma": 0.2})
    hi = qk.heston_monte_carlo_price(**{**base, "sigma": 0.5})
    assert hi >= lo - 0.5


@pytest.mark.parametrize("spot", [50.0, 100.0, 200.0])
@pytest.mark.parametrize("ot", [QK_CALL, QK_PUT])
def test_heston_finite(qk, spot, ot):
    assert math.isfinite(qk.heston_monte_carlo_price(spot=spot, option_type=ot, **_BASE))


def test_heston_extremes(qk):
    itm = qk.heston_monte_carlo_price(spot=300.0, option_type=QK_CALL, **_BASE)
    assert math.isfinite(itm) and itm > 0.0
    otm = qk.heston_monte_carlo_price(spot=300.0, option_type=QK_PUT, **_BASE)
    assert math.isfinite(otm) and otm >= 0.0
    call = qk.heston_monte_carlo_price(spot=110.0, option_type=QK_CALL, **{**_BASE, "t": 1e-14})
    assert math.isfinite(call) and abs(call - 10.0) < 0.01


@pytest.mark.parametrize("rho", [-0.99, 0.0, 0.99])
def test_heston_extreme_correlation(qk, rho):
    p = qk.heston_monte_carlo_price(spot=100.0, option_type=QK_CALL, **{**_BASE, "rho": rho})
    assert math.isfinite(p) and p > 0.0


# ---------------------------------------------------------------- test_local_vol_monte_carlo.py
_LV = dict(spot=100.0, strike=100.0, t=1.0, vol=0.2, r=0.03, q=0.01, option_type=QK_CALL,
           paths=20000, steps=64, seed=42)


@pytest.mark.parametrize("ot", [QK_CALL, QK_PUT])
def test_local_vol_matches_euler(qk, ot):
    p = {**_LV, "option_type": ot}
    lv = qk.local_vol_monte_carlo_price(**p)
    em = qk.euler_maruyama_price(**p)
    assert math.isfinite(lv) and math.isfinite(em)
    assert abs(lv - em) < 0.5


def test_local_vol_consistent_with_bsm(qk, oracle):
    bsm = oracle.bsm(100.0, 100.0, 1.0, 0.2, 0.03, 0.01, QK_CALL)
    lv = qk.local_vol_monte_carlo_price(**{**_LV, "paths": 50000})
    assert abs(lv - bsm) < 1.0


@pytest.mark.parametrize("spot", [80.0, 100.0, 120.0])
def test_local_vol_bounded(qk, spot):
    assert 0.0 <= qk.local_vol_monte_carlo_price(**{**_LV, "spot": spot}) <= spot
    upper = _LV["strike"] * math.exp(-_LV["r"] * _LV["t"])
    assert 0.0 <= qk.local_vol_monte_carlo_price(**{**_LV, "spot": spot, "option_type": QK_PUT}) <= upper


def test_local_vol_monotone_deterministic_batch(qk):
    spots = [80.0, 90.0, 100.0, 110.0, 120.0]
    c = [qk.local_vol_monte_carlo_price(**{**_LV, "spot": s}) for s in spots]
    p = [qk.local_vol_monte_carlo_price(**{**_LV, "spot": s, "option_type": QK_PUT}) for s in spots]
    for i in range(4):
        assert c[i + 1] >= c[i] - 0.5
        assert p[i + 1] <= p[i] + 0.5
    a = qk.local_vol_monte_carlo_price(**{**_LV, "seed": 777})
    assert a == qk.local_vol_monte_carlo_price(**{**_LV, "seed": 777})
    params = [_LV, {**_LV, "spot": 110.0, "option_type": QK_PUT, "seed": 99}]
    scal = [qk.local_vol_monte_carlo_price(**x) for x in params]
    bat = qk.local_vol_monte_carlo_price_batch(**{k: [x[k] for x in params] for k in params[0]})
    for i in range(2):
        assert abs(bat[i] - scal[i]) < 1e-12


# ---------------------------------------------------------------- test_batch_api.py
def _bsm_inputs(rng, n):
    return dict(spot=rng.uniform(90.0, 110.0, n), strike=rng.uniform(90.0, 110.0, n),
                t=rng.uniform(0.25, 1.0, n), vol=rng.uniform(0.15, 0.4, n),
                r=rng.uniform(0.01, 0.05, n), q=rng.uniform(0.0, 0.02, n),
                option_type=np.where((np.arange(n) & 1) == 0, QK_CALL, QK_PUT).astype(np.int32))


def test_standard_mc_batch_matches_scalar_random(qk):
    rng = np.random.default_rng(7)
    m = 16
    x = _bsm_inputs(rng, m)
    paths = np.full(m, 2048, np.int32)
    seed = np.arange(m, dtype=np.uint64) + np.uint64(12345)
    b = qk.standard_monte_carlo_price_batch(**x, paths=paths, seed=seed)
    s = [qk.standard_monte_carlo_price(*(float(x[k][i]) for k in ("spot", "strike", "t", "vol", "r", "q")),
                                       int(x["option_type"][i]), int(paths[i]), int(seed[i]))
         for i in range(m)]
    assert np.allclose(b, s, atol=1e-12, rtol=1e-12)


def test_mc_euler_milstein_batch(qk):
    rng = np.random.default_rng(300)
    n = 8
    x = _bsm_inputs(rng, n)
    paths = np.full(n, 1024, np.int32)
    steps = np.full(n, 50, np.int32)
    seed = np.arange(n, dtype=np.uint64) + np.uint64(42)
    for method in ("euler_maruyama", "milstein"):
        b = getattr(qk, f"{method}_price_batch")(**x, paths=paths, steps=steps, seed=seed)
        s = [getattr(qk, f"{method}_price")(
            *(float(x[k][i]) for k in ("spot", "strike", "t", "vol", "r", "q")),
            int(x["option_type"][i]), int(paths[i]), int(steps[i]), int(seed[i])) for i in range(n)]
        assert np.allclose(b, s, atol=1e-12, rtol=1e-12), method


def test_antithetic_batch(qk):
    rng = np.random.default_rng(304)
    n = 8
    x = _bsm_inputs(rng, n)
    paths = np.full(n, 1024, np.int32)
    seed = np.arange(n, dtype=np.uint64) + np.uint64(42)
    b = qk.antithetic_variates_price_batch(**x, paths=paths, seed=seed)
    s = [qk.antithetic_variates_price(*(float(x[k][i]) for k in ("spot", "strike", "t", "vol", "r", "q")),
                                      int(x["option_type"][i]), int(paths[i]), int(seed[i]))
         for i in range(n)]
    assert np.allclose(b, s, atol=1e-12, rtol=1e-12)


# ---------------------------------------------------------------- entry-check semantics
def test_invalid_elements_give_nan_and_batch_still_ok(qk):
    out = qk.heston_monte_carlo_price_batch(
        spot=[100.0, -1.0, 100.0, 110.0], strike=[100.0] * 4, t=[1.0, 1.0, 1.0, 1e-14],
        r=[0.05] * 4, q=[0.0] * 4, v0=[0.04, 0.04, -0.1, 0.04], kappa=[2.0] * 4, theta=[0.04] * 4,
        sigma=[0.3] * 4, rho=[-0.7] * 4, option_type=[0] * 4, paths=[1000, 1000, 1000, 1000],
        steps=[10] * 4, seed=[1, 2, 3, 4])
    assert math.isfinite(out[0]) and math.isnan(out[1]) and math.isnan(out[2])
    assert out[3] == 10.0  # t <= 1e-12: undiscounted intrinsic
    with pytest.raises(ValueError):
        qk.euler_maruyama_price(100.0, 100.0, 1.0, 0.2, 0.05, 0.0, 0, 1, 10, 1)  # paths <= 1
    zero_vol = qk.standard_monte_carlo_price(100.0, 90.0, 1.0, 0.0, 0.05, 0.0, 0, 1000, 1)
    assert abs(zero_vol - math.exp(-0.05) * (100.0 * math.exp(0.05) - 90.0)) < 1e-12
