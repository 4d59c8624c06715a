"""Statistical parity of the GPU Monte Carlo with (a) the reference's own CPU
Monte Carlo -- run through the oracle, which reproduces it bit for bit -- and
(b) the FP64 closed forms (BSM, Heston characteristic function).

A counter-based GPU generator cannot reproduce mt19937, so agreement is
statistical.  For each option z = (gpu - other) / combined SE.  With N options
a perfect estimator still exceeds |z| > 3 with probability 0.0027 each, so the
tests allow up to the 99.9% binomial quantile of that count (multiplicity) and
bound max |z|.  The observed statistics are printed.
"""

import math

import numpy as np
import pytest
from stat_check import check_z, z_scores

from quantkernel_b200 import workloads

pytestmark = pytest.mark.gpu

_z = z_scores
_check = check_z


def test_bsm_terminal_full_size_vs_closed_form_and_reference(qk, oracle):
    b = workloads.bsm_terminal()  # 64 options x 131072 paths
    for name, fn, model in (("standard", qk.standard_monte_carlo_price_se_batch, 0),
                            ("antithetic", qk.antithetic_variates_price_se_batch, 1)):
        p, se = fn(**b)
        cf = np.array([oracle.bsm(b["spot"][i], b["strike"][i], b["t"][i], b["vol"][i], b["r"][i],
                                  b["q"][i], int(b["option_type"][i])) for i in range(64)])
        _check(_z(p, cf, se), f"{name} GPU vs BSM closed form")
        cp, cse = oracle.bsm_family_batch(model, b["spot"], b["strike"], b["t"], b["vol"], b["r"],
                                          b["q"], b["option_type"], b["paths"], None, b["seed"])
        _check(_z(p, cp, np.hypot(se, cse)), f"{name} GPU vs reference CPU MC")


@pytest.mark.parametrize("model", [2, 3, 4])
def test_stepwise_vs_reference_cpu_mc(qk, oracle, model):
    rng = np.random.default_rng(40 + model)
    n = 48
    b = workloads.bsm_terminal(n, paths=20000, seed=50 + model)
    steps = rng.integers(8, 64, n).astype(np.int32)
    fn = {2: qk.euler_maruyama_price_se_batch, 3: qk.milstein_price_se_batch,
          4: qk.local_vol_monte_carlo_price_se_batch}[model]
    p, se = fn(**b, steps=steps)
    cp, cse = oracle.bsm_family_batch(model, b["spot"], b["strike"], b["t"], b["vol"], b["r"],
                                      b["q"], b["option_type"], b["paths"], steps, b["seed"])
    _check(_z(p, cp, np.hypot(se, cse)), f"model {model} GPU vs reference CPU MC")


def test_heston_vs_reference_cpu_mc(qk, oracle):
    h = workloads.heston(32, paths=32768, steps=50, seed=77)
    p, se = qk.heston_monte_carlo_price_se_batch(**h)
    cp, cse = oracle.heston_batch(**h)
    _check(_z(p, cp, np.hypot(se, cse)), "Heston GPU vs reference CPU MC (32 x 32768 x 50)")


def test_heston_full_size_vs_cf_and_reference_subset(qk, oracle):
    """The benchmark workload at full size: 1024 calls x 262144 paths x 200 steps.

    The FP64 characteristic-function price is the continuous-time Heston
    price; the reference's full-truncation Euler at 200 steps is biased away
    from it, strongly at low Feller ratio 2 kappa theta / sigma^2 (the box
    reaches 0.01).  So:
      (1) options with Feller >= 1 (small scheme bias) match the CF price
          within the multiplicity rule;
      (2) the most biased options match the reference's own CPU Monte Carlo
          at the same 200 steps -- the discretisation-free check;
      (3) their gap to the CF price shrinks when the GPU runs more steps (slowly:
          full truncation converges at a low rate when v sits at 0), so the gap
          belongs to the scheme, not to the kernel.
    Observed errors are printed."""
    h = workloads.heston()
    p, se = qk.heston_monte_carlo_price_se_batch(**h)
    assert np.all(np.isfinite(p)) and np.all(se > 0)
    n = len(p)

    def cf_of(b, i):
        return oracle.heston_cf(b["spot"][i], b["strike"][i], b["t"][i], b["r"][i], b["q"][i],
                                b["v0"][i], b["kappa"][i], b["theta"][i], b["sigma"][i],
                                b["rho"][i], 0)

    cf = np.array([cf_of(h, i) for i in range(n)])
    z = (p - cf) / se
    feller = 2 * h["kappa"] * h["theta"] / h["sigma"] ** 2
    err = np.abs(p - cf) / h["spot"]
    hi = feller >= 1.0
    print(f"|price - CF|/S: max {err.max():.2e} mean {err.mean():.2e}; Feller>=1: max "
          f"{err[hi].max():.2e}; mean SE/S {(se / h['spot']).mean():.2e}")
    for lo_f, hi_f in ((0, 0.25), (0.25, 0.5), (0.5, 1.0), (1.0, 1e9)):
        m = (feller >= lo_f) & (feller < hi_f)
        if m.any():
            print(f"  Feller [{lo_f}, {hi_f}): n={int(m.sum())} mean z vs CF {z[m].mean():+.2f}")
    _check(z[hi], "Heston GPU vs CF, Feller >= 1 (1024 x 262144 x 200)")

    order = np.argsort(feller)
    idx = np.concatenate([order[:8], order[-4:]])
    sub = {k: v[idx] for k, v in workloads.heston(paths=32768).items()}
    gp, gse = qk.heston_monte_carlo_price_se_batch(**sub)
    cp, cse = oracle.heston_batch(**sub)
    print("lowest Feller:", np.round(feller[order[:8]], 3))
    _check(_z(gp, cp, np.hypot(gse, cse)),
           "Heston GPU vs reference CPU MC, 200 steps, 8 lowest + 4 highest Feller", zmax=4.5)

    low = {k: v[order[:8]] for k, v in workloads.heston(paths=65536).items()}
    cfl = np.array([cf_of(low, i) for i in range(8)])
    g200, _ = qk.heston_monte_carlo_price_se_batch(**low)
    low800 = dict(low, steps=np.full(8, 1600, np.int32))
    g1600, s1600 = qk.heston_monte_carlo_price_se_batch(**low800)
    e200, e1600 = np.abs(g200 - cfl), np.abs(g1600 - cfl)
    print("low-Feller |GPU - CF| at 200 steps:", np.round(e200, 4), " at 1600 steps:", np.round(e1600, 4))
    # full truncation converges slowly at Feller ~0.02 (observed: -23% for 8x the steps)
    assert e1600.mean() < 0.85 * e200.mean()


def test_fixture_edge_cases_on_gpu(qk, oracle):
    """The reference fixture's deterministic edge cases reproduce exactly on the GPU."""
    import json
    from pathlib import Path

    doc = json.loads((Path(__file__).parent / "golden" / "reference_mc.json").read_text())
    checked = 0
    for case in doc["mc_cases"]:
        a = {k: (float.fromhex(v) if isinstance(v, str) else v) for k, v in case["args"].items()}
        want = float.fromhex(case["price"])
        m = case["model"]
        if "shift" in a:  # importance sampling reads its shift from v0 in plans
            a["v0"] = a.pop("shift")
        deterministic = (math.isnan(want) or a["t"] <= 1e-12 or a["paths"] <= 1 or
                         (m == 0 and a["vol"] <= 1e-12) or
                         (m == 6 and any(math.isnan(a[k]) for k in ("spot", "strike", "q", "v0"))))
        if not deterministic:
            continue
        model_arr = np.array([m], np.int32)
        plan = qk.plan(model=model_arr, **{k: np.array([v]) for k, v in a.items()})
        plan.execute()
        got, _ = plan.results()
        plan.close()
        assert (math.isnan(got[0]) and math.isnan(want)) or got[0] == want, (case, got[0], want)
        checked += 1
    assert checked >= 40


def test_full_heston_benchmark_vs_reference_cpu_mc(qk):
    """Every one of the benchmark's 1024 Heston prices (262144 paths x 200
    steps) against the reference's own CPU Monte Carlo on the same inputs
    (tests/golden/heston_full_reference.json, produced by the oracle that equals
    the reference bit for bit): z = difference / combined SE."""
    import json
    from pathlib import Path

    doc = json.loads((Path(__file__).parent / "golden" / "heston_full_reference.json").read_text())
    ref_p = np.array([float.fromhex(x) for x in doc["price"]])
    ref_se = np.array([float.fromhex(x) for x in doc["stderr"]])
    p, se = qk.heston_monte_carlo_price_se_batch(**workloads.heston())
    _check(_z(p, ref_p, np.hypot(se, ref_se)), "Heston benchmark workload GPU vs reference CPU MC")
