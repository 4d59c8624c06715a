"""Pathwise parity: the GPU kernels against the oracle's FP64 replay of the
same Philox4x32-10 + Box-Muller stream through the reference step functions
(model_concepts.h).

Both sides see identical normals for every path.  For the stepwise models
(FP32 path state, approximate special functions) the only difference left is
FP32 rounding and the MUFU approximations, and the tolerance is written as
    |price_gpu - price_fp64| <= 5e-5 * spot + 0.02 * SE
-- a hundred times below a standard error -- so any indexing, counter,
antithetic-pairing or step-formula bug (which moves the price by O(SE))
fails; standard errors must agree to 2%.  The terminal models compute in FP64
end to end (FP64 normals and exponent), so there the bar is rounding only:
    |price_gpu - price_fp64| <= 2e-11 * spot,  standard errors to 1e-9.
"""

import math

import numpy as np
import pytest

from quantkernel_b200 import QK_PLAN_NO_ANTITHETIC

pytestmark = pytest.mark.gpu

TERMINAL = (0, 1, 5)


def _cases(model, rng):
    out = []
    shapes = [(2, 1), (3, 7), (1001, 3), (4097, 16), (20000, 50), (65537, 2)]
    if model in TERMINAL:
        shapes = [(2, 1), (3, 1), (1001, 1), (4097, 1), (65536, 1), (200001, 1)]
    for k, (paths, steps) in enumerate(shapes):
        out.append(dict(
            spot=float(rng.uniform(60, 140)), strike=float(rng.uniform(60, 140)),
            t=float(rng.uniform(0.05, 2.5)), vol=float(rng.uniform(0.05, 0.6)),
            r=float(rng.uniform(0.0, 0.06)), q=float(rng.uniform(0.0, 0.03)),
            v0=float(rng.uniform(0.01, 0.12)), kappa=float(rng.uniform(0.3, 5.0)),
            theta=float(rng.uniform(0.01, 0.1)), sigma=float(rng.uniform(0.1, 1.2)),
            rho=float(rng.uniform(-0.95, 0.3)), option_type=k & 1, paths=paths, steps=steps,
            seed=int(rng.integers(0, 2**63))))
    return out


@pytest.mark.parametrize("model,anti", [(0, True), (1, True), (5, False), (2, True), (2, False),
                                        (3, True), (3, False), (4, True), (4, False), (6, True),
                                        (6, False), (7, True), (7, False)])
def test_gpu_equals_fp64_replay_of_same_stream(qk, oracle, model, anti):
    rng = np.random.default_rng(100 + model * 2 + int(anti))
    cases = _cases(model, rng)
    if model == 7:  # the LR delta reads its weight clip from `vol`; a delta is O(1), not O(S)
        for k, c in enumerate(cases):
            c["vol"] = (0.5, 2.0, 6.0)[k % 3]
    cols = {k: np.array([c[k] for c in cases]) for k in cases[0]}
    flags = 0 if anti else QK_PLAN_NO_ANTITHETIC
    plan = qk.plan(model=np.full(len(cases), model, np.int32), flags=flags, **cols)
    plan.execute()
    price, se = plan.results()
    plan.close()
    worst = 0.0
    for i, c in enumerate(cases):
        want, want_se = oracle.philox_price(model, antithetic=anti, **c)
        scale = 1.0 if model == 7 else c["spot"]
        fp64 = model in TERMINAL
        if fp64:
            tol = 2e-11 * scale
        else:
            tol = 5e-5 * scale + 0.02 * (want_se if math.isfinite(want_se) else 0.0)
        diff = abs(price[i] - want)
        worst = max(worst, diff / tol)
        assert diff <= tol, (model, anti, c, price[i], want, se[i], want_se)
        if math.isfinite(want_se) and want_se > 0:
            se_tol = (1e-9 if fp64 else 0.02) * want_se + 1e-12
            assert abs(se[i] - want_se) <= se_tol, (c, se[i], want_se)
        elif math.isfinite(want_se):  # every payoff identical (deep out of the money)
            assert se[i] == 0.0, (c, se[i])
        else:  # fewer than two samples
            assert not math.isfinite(se[i]), (c, se[i])
    print(f"model {model} anti={anti}: worst |diff|/tol = {worst:.3f}")


def test_heston_large_and_non_finite_drift(qk, oracle):
    """The Heston kernel keeps y = log(S/spot) - j (r-q)dt as its state while
    |(r-q) t| <= 1 and log(S/spot) itself beyond, where y would outgrow FP32
    and its moving floor would lose log(1e-12/spot).  The reference accepts
    any r and q for Heston (heston_monte_carlo.cpp:18-24 checks neither), so
    both sides of that switch are held to the FP64 replay of the same stream,
    and drifts that pin every path to the 1e-12 floor, or send it to +inf, to
    the values the reference's step gives them."""
    base = dict(spot=100.0, strike=95.0, t=1.5, vol=0.0, v0=0.04, kappa=1.5, theta=0.05,
                sigma=0.6, rho=-0.6, paths=20001, steps=40, seed=77)
    keys = ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho",
            "option_type", "paths", "steps", "seed")

    def run(cases):
        cols = {k: np.array([c[k] for c in cases]) for k in keys}
        for k in ("option_type", "paths", "steps"):
            cols[k] = cols[k].astype(np.int32)
        cols["seed"] = cols["seed"].astype(np.uint64)
        return qk.heston_monte_carlo_price_se_batch(**cols)

    # |(r-q) t| = 0.9 (y state) and 1.05, 1.35, 2.25 (log-spot state)
    cases = [dict(base, r=r, q=q, option_type=ot)
             for r, q in ((0.6, 0.0), (0.7, 0.0), (0.0, 0.9), (2.0, 0.5)) for ot in (0, 1)]
    price, se = run(cases)
    for i, c in enumerate(cases):
        want, want_se = oracle.philox_price(6, antithetic=True, **c)
        tol = 5e-5 * c["spot"] + 0.02 * want_se
        assert abs(price[i] - want) <= tol, (c, price[i], want)
        assert abs(se[i] - want_se) <= 0.02 * want_se + 1e-12, (c, se[i], want_se)

    # every step's exp(-inf) (or exp of -1e4 (r-q) dt) sends S to the 1e-12 floor
    inf = math.inf
    floor_put = 95.0 - 1e-12
    cases = [dict(base, r=0.03, q=q, option_type=ot) for q in (inf, 1e4) for ot in (0, 1)]
    cases += [dict(base, r=-inf, q=0.0, option_type=ot) for ot in (0, 1)]
    cases += [dict(base, r=inf, q=0.0, option_type=ot) for ot in (0, 1)]
    price, se = run(cases)
    disc = math.exp(-0.03 * 1.5)
    for i in range(4):
        want = 0.0 if cases[i]["option_type"] == 0 else disc * floor_put
        assert abs(price[i] - want) <= 1e-12 * max(1.0, want), (cases[i], price[i], want)
        assert 0.0 <= se[i] <= 1e-9 * max(1.0, want), (cases[i], se[i])
    # r = -inf: exp(-r t) = inf times the floor payoff (inf for the put; inf * 0 for the call)
    assert math.isnan(price[4]) and price[5] == inf, price[4:6]
    # r = +inf: S = +inf at every step, exp(-r t) = 0 (0 * inf for the call; 0 for the put)
    assert math.isnan(price[6]) and price[7] == 0.0, price[6:8]
