"""GPU Heston COS pricer against the reference's own outputs.

qk_ftm_cos_fang_oosterlee_heston_price(_batch) restates cos_method.cpp:30-58
(Fang-Oosterlee cosine expansion with the Heston log-price characteristic
function, charfn_concepts.h:54-78) in FP64 on the GPU, one CTA per option.
The terms are summed in a fixed tree instead of the reference's loop and the
elementary functions are CUDA's, so each term carries a different rounding
error.  The exponent of a term is a sum of parts that cancel, some of them
divided by sigma^2 (a - d is a difference of numbers of size |a| + |d|), and an
absolute error in an exponent is a relative error of its term; the terms in
turn cancel in the sum.  The oracle's error scale E is that first-order bound:
exp(-r t) sum_k |term_k| (1 + size of term k's exponent parts).  The bar is
1e-9 x max(1, |price|) + DBL_EPSILON x E; on well-conditioned inputs E is far
below the first part, and the observed error stays under 0.1 DBL_EPSILON x E.
The entry checks' NaN and intrinsic results, and the 0 that the reference's
max(0, NaN) gives for degenerate parameters, agree exactly.
"""

import json
import math
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_mc.json").read_text())
EPS = 2.220446049250313e-16
KEYS = ["spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho", "option_type",
        "n_terms", "truncation_width"]


def _args(d):
    return {k: (float.fromhex(v) if isinstance(v, str) else v) for k, v in d.items()}


def _tol(oracle, a, want):
    s = oracle.heston_cos_error_scale(*(a[k] for k in KEYS))
    s = s if math.isfinite(s) else 0.0  # NaN terms: the max(0, NaN) = 0 cases match exactly
    return 1e-9 * max(1.0, abs(want)) + EPS * s, s


def _batch(qk, cases):
    cols = {k: np.array([c[k] for c in cases]) for k in KEYS}
    return qk.cos_method_fang_oosterlee_heston_price_batch(*(cols[k] for k in KEYS))


def test_reference_fixtures(qk, oracle):
    cases = [_args(c["args"]) for c in GOLDEN["heston_cos"]]
    want = [float.fromhex(c["price"]) for c in GOLDEN["heston_cos"]]
    got = _batch(qk, cases)
    bad, worst = [], 0.0
    for a, g, w in zip(cases, got, want):
        if math.isnan(w):
            ok = math.isnan(g)
        else:
            tol, s = _tol(oracle, a, w)
            ok = abs(g - w) <= tol
            worst = max(worst, abs(g - w) / max(EPS * s, 1e-300))
        if not ok:
            bad.append((a, g, w))
    print(f"\nCOS fixtures: max |gpu - reference| / (DBL_EPSILON x E) = {worst:.3e}")
    assert not bad, bad[:5]


def test_scalar_equals_batch_and_defaults(qk):
    cases = [_args(c["args"]) for c in GOLDEN["heston_cos"]]
    batch = _batch(qk, cases)
    for a, b in zip(cases, batch):
        s = qk._lib.qk_ftm_cos_fang_oosterlee_heston_price(*(a[k] for k in KEYS))
        assert (math.isnan(s) and math.isnan(b)) or s == b, (a, s, b)
    # engine.py:742-750 defaults: 256 terms, width 10
    p = qk.cos_method_fang_oosterlee_heston_price(100.0, 100.0, 1.0, 0.03, 0.01, 0.04, 2.0, 0.04,
                                                  0.3, -0.7, 0)
    assert p == batch[[i for i, a in enumerate(cases) if a["option_type"] == 0 and
                       a["n_terms"] == 256 and a["truncation_width"] == 10.0 and
                       a["strike"] == 100.0 and a["sigma"] == 0.3 and a["kappa"] == 2.0 and
                       a["t"] == 1.0 and a["v0"] == 0.04 and a["rho"] == -0.7][0]]


def test_random_batch_against_oracle(qk, oracle):
    rng = np.random.default_rng(55)
    n = 1024
    cols = dict(
        spot=rng.uniform(50, 150, n), strike=rng.uniform(40, 200, n), t=rng.uniform(0.02, 5, n),
        r=rng.uniform(-0.01, 0.08, n), q=rng.uniform(0, 0.05, n), v0=rng.uniform(0.0, 0.3, n),
        kappa=rng.uniform(0.05, 8, n), theta=rng.uniform(0.0, 0.3, n),
        sigma=rng.uniform(0.02, 2.0, n), rho=rng.uniform(-0.99, 0.99, n),
        option_type=rng.integers(0, 2, n).astype(np.int32),
        n_terms=rng.choice([8, 64, 256, 1024], n).astype(np.int32),
        truncation_width=rng.choice([4.0, 10.0, 14.0], n))
    got = qk.cos_method_fang_oosterlee_heston_price_batch(*(cols[k] for k in KEYS))
    bad = []
    for i in range(n):
        a = {k: cols[k][i].item() for k in KEYS}
        want = oracle.heston_cos(*a.values())
        ok = math.isnan(got[i]) if math.isnan(want) else \
            abs(got[i] - want) <= _tol(oracle, a, want)[0]
        if not ok:
            bad.append((i, got[i], want))
    assert not bad, bad[:5]


def test_agrees_with_cf_pricer(qk):
    """The reference's own check (test_heston_fourier.py:24-46): COS within 1.5
    of the CF price; on well-posed inputs the two GPU pricers agree far closer."""
    a = [100.0, 100.0, 1.0, 0.03, 0.01, 0.04, 2.0, 0.04, 0.3, -0.7]
    for ot in (0, 1):
        cf = qk.heston_price_cf(*a, ot, integration_steps=8192, integration_limit=500.0)
        cos = qk.cos_method_fang_oosterlee_heston_price(*a, ot)
        assert abs(cos - cf) < 1.5
        assert abs(cos - cf) < 1e-4, (ot, cos, cf)
