"""Pins the FP64 MLP oracle used to check the surrogate's GPU gradients:
analytic gradients against central finite differences (CPU)."""

import numpy as np

from oracle import mlp_oracle as mo


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(scale=0.1, size=mo.N_PARAMS)
    x = rng.uniform(-1, 1, size=(16, mo.IN))
    t = rng.uniform(0, 0.3, size=16)
    loss, g = mo.loss_and_grads(p, x, t)
    assert g.shape == (mo.N_PARAMS,) and mo.N_PARAMS == 134401
    idx = rng.choice(mo.N_PARAMS, 60, replace=False)
    idx = np.concatenate([idx, [0, 2304, 2560, 68095, 134400]])  # first/last of several blocks
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (mo.loss_and_grads(p + e, x, t)[0] - mo.loss_and_grads(p - e, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-9, (i, fd, g[i])


def test_bf16_bits_roundtrip():
    v = np.array([1.0, -2.5, 0.15625], np.float32)
    bits = (v.view(np.uint32) >> 16).astype(np.uint16)
    assert np.allclose(mo.bf16_bits_to_float(bits), v)


def test_base_is_black_scholes_at_mean_variance(oracle):
    """The residual's base: Black-Scholes at vbar = theta + (v0 - theta)(1 -
    exp(-kappa T))/(kappa T); v0 = theta gives Black-Scholes at sqrt(theta)."""
    f = np.array([[100 / 95, 1.0, 0.03, 0.0, 0.04, 2.0, 0.04, 0.3, -0.7],
                  [100 / 120, 0.5, 0.01, 0.0, 0.09, 1.0, 0.01, 0.5, -0.2],
                  [100 / 80, 2.0, 0.05, 0.0, 0.01, 1e-14, 0.09, 0.5, -0.2]])
    b = mo.bsm_mean_var_base(f)
    assert abs(b[0] * 95 - oracle.bsm(100.0, 95.0, 1.0, 0.2, 0.03, 0.0, 0) * 95 / 100) < 1e-6
    vbar = 0.01 + 0.08 * (1 - np.exp(-0.5)) / 0.5
    assert abs(b[1] - oracle.bsm(100.0, 120.0, 0.5, np.sqrt(vbar), 0.01, 0.0, 0) / 100) < 1e-6
    # kappa T -> 0: the variance stays at v0
    assert abs(b[2] - oracle.bsm(100.0, 80.0, 2.0, 0.1, 0.05, 0.0, 0) / 100) < 1e-6
