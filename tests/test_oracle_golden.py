"""Pins the CPU oracle: reference golden seeds, fixtures generated from the
reference library, closed-form known values, and the Philox/Box-Muller layout.

Runs on CPU (no GPU marker)."""

import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import (ANTITHETIC, EULER, HESTON, HESTON_LR_DELTA, LOCAL_VOL, MILSTEIN,
                           STANDARD, TERMINAL_PLAIN)

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_mc.json").read_text())


def _args(d):
    return {k: (float.fromhex(v) if isinstance(v, str) else v) for k, v in d.items()}


def _same(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


# cpp/tests/test_monte_carlo.cpp:57-73 of the reference.
def test_reference_golden_seeds(oracle):
    p, _ = oracle.price(STANDARD, 100.0, 100.0, 1.0, 0.2, 0.05, 0.0, 0, 50000, 1, 12345)
    assert abs(p - 10.533371511490282) < 1e-12
    p, _ = oracle.price(STANDARD, 100.0, 100.0, 1.0, 0.2, 0.05, 0.0, 1, 50000, 1, 12345)
    assert abs(p - 5.6296577522043556) < 1e-12
    p, _ = oracle.price(EULER, 100.0, 100.0, 1.0, 0.2, 0.05, 0.0, 0, 10000, 100, 12345)
    assert abs(p - 10.218359279533905) < 1e-12


@pytest.mark.parametrize("i", range(len(GOLDEN["mc_cases"])))
def test_oracle_bitwise_equals_reference_fixture(oracle, i):
    case = GOLDEN["mc_cases"][i]
    a = _args(case["args"])
    want = float.fromhex(case["price"])
    got, _ = oracle.price(case["model"], **a)
    assert _same(got, want), f"case {i} model {case['model']}: {got!r} != {want!r}"


def test_oracle_bitwise_equals_reference_live(oracle, ref):
    rng = np.random.default_rng(7)
    for model in (STANDARD, ANTITHETIC, EULER, MILSTEIN, LOCAL_VOL, HESTON, HESTON_LR_DELTA):
        for _ in range(5):
            a = dict(spot=float(rng.uniform(50, 150)), strike=float(rng.uniform(50, 150)),
                     t=float(rng.uniform(0.05, 3.0)), vol=float(rng.uniform(0.05, 0.8)),
                     r=float(rng.uniform(-0.01, 0.08)), q=float(rng.uniform(0.0, 0.05)),
                     option_type=int(rng.integers(0, 2)), paths=int(rng.integers(2, 2000)),
                     steps=int(rng.integers(1, 40)), seed=int(rng.integers(0, 2**64, dtype=np.uint64)),
                     v0=float(rng.uniform(0, 0.2)), kappa=float(rng.uniform(0, 6)),
                     theta=float(rng.uniform(0, 0.2)), sigma=float(rng.uniform(0, 1.5)),
                     rho=float(rng.uniform(-1, 1)))
            got, _ = oracle.price(model, **a)
            want = ref.price(model, **a)
            assert _same(got, want), (model, a, got, want)


def test_oracle_heston_extreme_drift_equals_reference_live(oracle, ref):
    """Heston accepts any r and q (heston_monte_carlo.cpp:18-24 checks neither):
    drifts that pin every path to the 1e-12 floor, send it to +inf, or are
    NaN give the same prices in the oracle as in the reference."""
    inf = math.inf
    base = dict(spot=100.0, strike=95.0, t=1.5, vol=0.0, v0=0.04, kappa=1.5, theta=0.05,
                sigma=0.6, rho=-0.6, paths=501, steps=17, seed=77)
    for r, q in ((0.03, inf), (0.03, 1e4), (-inf, 0.0), (inf, 0.0), (0.03, -inf), (-1e4, 0.0),
                 (math.nan, 0.0), (0.03, math.nan), (0.7, 0.0), (0.0, 0.9)):
        for ot in (0, 1):
            a = dict(base, r=r, q=q, option_type=ot)
            got, _ = oracle.price(HESTON, **a)
            want = ref.price(HESTON, **a)
            assert _same(got, want), (a, got, want)


@pytest.mark.parametrize("i", range(len(GOLDEN["heston_cf"])))
def test_heston_cf_matches_reference(oracle, i):
    case = GOLDEN["heston_cf"][i]
    a = _args(case["args"])
    want = float.fromhex(case["price"])
    got = oracle.heston_cf(**a)
    # Gauss-Legendre nodes are computed here, tabulated there: agreement to ~1e-10.
    assert abs(got - want) < 1e-8, (a, got, want)


@pytest.mark.parametrize("i", range(len(GOLDEN["heston_cf_edges"])))
def test_heston_cf_edges_match_reference(oracle, i):
    """Integration settings 16..8192 steps, limits 1e-5..500, the entry checks
    of heston.cpp:10-24 (NaN, intrinsic) and extreme parameters."""
    case = GOLDEN["heston_cf_edges"][i]
    a = _args(case["args"])
    want = float.fromhex(case["price"])
    got = oracle.heston_cf(**a)
    if math.isnan(want):
        assert math.isnan(got), (a, got)
    else:
        assert abs(got - want) < 1e-8 * max(1.0, abs(want)), (a, got, want)


@pytest.mark.parametrize("i", range(len(GOLDEN["heston_cos"])))
def test_heston_cos_matches_reference_bitwise(oracle, i):
    """The COS restatement (cos_method.cpp:30-58) equals the reference bit for
    bit: same characteristic-function expression order, same sequential sum,
    including its NaN and max(0, NaN) = 0 outcomes on degenerate inputs."""
    case = GOLDEN["heston_cos"][i]
    a = _args(case["args"])
    want = float.fromhex(case["price"])
    got = oracle.heston_cos(**a)
    assert _same(got, want), (a, got, want)
    # the rounding scale the GPU parity bar uses bounds the call price it sums to
    s = oracle.heston_cos_error_scale(**a)
    if a["option_type"] == 0 and math.isfinite(want) and want > 0.0 and s > 0.0:
        assert s >= want * (1 - 1e-12), (a, s)


def test_heston_cos_agrees_with_cf(oracle):
    """Two independent Fourier methods of the reference agree on well-posed
    inputs (the COS method is the CF oracle's independent check)."""
    rng = np.random.default_rng(41)
    for _ in range(40):
        a = dict(spot=100.0, strike=float(rng.uniform(70, 130)), t=float(rng.uniform(0.25, 2)),
                 r=float(rng.uniform(0, 0.05)), q=0.0, v0=float(rng.uniform(0.01, 0.09)),
                 kappa=float(rng.uniform(0.5, 5)), theta=float(rng.uniform(0.01, 0.09)),
                 sigma=float(rng.uniform(0.1, 1.0)), rho=float(rng.uniform(-0.9, 0.0)),
                 option_type=int(rng.integers(0, 2)))
        cf = oracle.heston_cf(**a, integration_steps=4096, integration_limit=300.0)
        cos = oracle.heston_cos(**a, n_terms=1024, truncation_width=12.0)
        assert abs(cf - cos) < 2e-4, (a, cf, cos)


def test_heston_cf_converged_and_small_volvol_limit(oracle):
    base = dict(spot=100.0, strike=105.0, t=1.0, r=0.03, q=0.01, v0=0.04, kappa=1.5,
                theta=0.04, sigma=1e-4, rho=-0.5, option_type=0)
    # vol-of-vol -> 0 with v0 = theta is BSM with vol = 0.2
    h = oracle.heston_cf(**base)
    b = oracle.bsm(100.0, 105.0, 1.0, 0.2, 0.03, 0.01, 0)
    assert abs(h - b) < 1e-4
    # the integration default (1024 steps, limit 120) is converged to ~3e-7,
    # far below any Monte Carlo standard error it is compared with
    base.update(sigma=0.6, rho=-0.7)
    p1 = oracle.heston_cf(**base)
    p2 = oracle.heston_cf(**base, integration_steps=8192, integration_limit=500.0)
    assert abs(p1 - p2) < 1e-6
    # put-call parity
    c = oracle.heston_cf(**base)
    p = oracle.heston_cf(**{**base, "option_type": 1})
    assert abs((c - p) - (100.0 * math.exp(-0.01) - 105.0 * math.exp(-0.03))) < 1e-10


def test_bsm_known_values_and_reference_cdf(oracle):
    # cpp/tests/test_closed_form.cpp:7-15
    assert abs(oracle.bsm(100, 100, 1, 0.2, 0.05, 0, 0) - 10.4506) < 0.01
    assert abs(oracle.bsm(100, 100, 1, 0.2, 0.05, 0, 1) - 5.5735) < 0.01
    c = oracle.bsm(100, 105, 0.5, 0.25, 0.05, 0.02, 0)
    p = oracle.bsm(100, 105, 0.5, 0.25, 0.05, 0.02, 1)
    assert abs((c - p) - (100 * math.exp(-0.01) - 105 * math.exp(-0.025))) < 1e-10
    # the reference uses A&S 7.1.26 (|error| <= 1.5e-7 in the CDF)
    for case in GOLDEN["bsm_cf_reference_as_cdf"]:
        a = _args(case["args"])
        assert abs(oracle.bsm(**a) - float.fromhex(case["price"])) < 1e-4


def test_standard_error_matches_seed_dispersion(oracle):
    prices, ses = [], []
    for seed in range(300):
        p, se = oracle.price(STANDARD, 100.0, 100.0, 1.0, 0.2, 0.05, 0.0, 0, 2000, 1, seed)
        prices.append(p)
        ses.append(se)
    ratio = np.std(prices, ddof=1) / np.mean(ses)
    assert 0.85 < ratio < 1.15, ratio
    prices, ses = [], []
    for seed in range(200):
        p, se = oracle.price(HESTON, 100.0, 100.0, 1.0, 0.0, 0.05, 0.02, 0, 500, 10, seed,
                             v0=0.04, kappa=2.0, theta=0.04, sigma=0.3, rho=-0.7)
        prices.append(p)
        ses.append(se)
    ratio = np.std(prices, ddof=1) / np.mean(ses)
    assert 0.8 < ratio < 1.2, ratio


def test_polar_normals_are_standard(oracle):
    z = oracle.normals(12345, 200000)
    assert abs(z.mean()) < 0.01
    assert abs(z.var() - 1.0) < 0.01


# --- Philox4x32-10: restated independently here in Python ------------------------------
def _philox_py(ctr, key):
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    M = 0xFFFFFFFF
    for _ in range(10):
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & M, p1 & M, ((p0 >> 32) ^ c3 ^ k1) & M, p0 & M
        k0 = (k0 + 0x9E3779B9) & M
        k1 = (k1 + 0xBB67AE85) & M
    return [c0, c1, c2, c3]


def test_philox_matches_python_restatement(oracle):
    rng = np.random.default_rng(3)
    for _ in range(200):
        ctr = [int(x) for x in rng.integers(0, 2**32, 4, dtype=np.uint64)]
        key = [int(x) for x in rng.integers(0, 2**32, 2, dtype=np.uint64)]
        assert oracle.philox(ctr, key) == _philox_py(ctr, key)
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == _philox_py([0, 0, 0, 0], [0, 0])


def test_philox_published_known_answers(oracle):
    """Philox4x32-10 known-answer vectors published with the algorithm
    (Salmon et al., SC'11; the Random123 distribution's kat_vectors): zero
    counter and key, all-ones, and the digits of pi."""
    kat = [([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
           ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
           ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
            [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1])]
    for ctr, key, want in kat:
        assert list(oracle.philox(ctr, key)) == want
        assert list(_philox_py(ctr, key)) == want


def test_philox_box_muller_layout(oracle):
    """The terminal models' FP64 normals: a quad is two Philox calls (blocks
    c1 and c1 + 1), each one Box-Muller pair with a 52-bit radius word
    x0 << 20 | x1 >> 12 and a 52-bit angle word x2 << 20 | x3 >> 12."""
    seed = 0x123456789ABCDEF
    key = [seed & 0xFFFFFFFF, seed >> 32]
    for c0, c1, c3 in [(0, 0, 0), (5, 7, 0), (2**31, 99, 1)]:
        z = oracle.philox_normals4(seed, c0, c1, c3)
        want = []
        for blk in (c1, c1 + 1):
            x = _philox_py([c0, blk, 0, c3], key)
            ub = (x[0] << 20) | (x[1] >> 12)
            gb = (x[2] << 20) | (x[3] >> 12)
            u = (ub + 0.5) * 2.0**-52
            g = (gb + 0.5) * 2.0**-51 - 1.0
            assert 0.0 < u < 1.0 and -1.0 < g < 1.0
            rad = math.sqrt(-2.0 * math.log(u))
            want += [rad * math.cos(math.pi * g), rad * math.sin(math.pi * g)]
        assert np.array_equal(z, want)
    # the replayed stream is standard normal
    zs = np.concatenate([oracle.philox_normals4(seed, i, 0, 0) for i in range(20000)])
    assert abs(zs.mean()) < 0.02 and abs(zs.var() - 1.0) < 0.02


def test_philox_six_normal_layout(oracle):
    """The Heston kernels draw three Box-Muller pairs per Philox call: 23-bit
    radii from the top of words 0-2, angles of 16, 16 and 18 bits from word 3
    and the low 9 bits of words 0 and 1."""
    from scipy import stats

    seed = 0xFEDCBA9876543210
    key = [seed & 0xFFFFFFFF, seed >> 32]
    for c0, c1, c3 in [(0, 0, 0), (3, 11, 1), (2**31 + 5, 66, 0)]:
        x = _philox_py([c0, c1, 0, c3], key)
        z = oracle.philox_normals6(seed, c0, c1, c3)
        want = []
        for ub, gb, n in ((x[0] >> 9, x[3] & 0xFFFF, 16), (x[1] >> 9, x[3] >> 16, 16),
                          (x[2] >> 9, (x[0] & 0x1FF) | ((x[1] & 0x1FF) << 9), 18)):
            u = (ub + 0.5) * 2.0**-23
            g = (gb + 0.5) * 2.0**-(n - 1) - 1.0
            rad = math.sqrt(-2.0 * math.log(u))
            want += [rad * math.cos(math.pi * g), rad * math.sin(math.pi * g)]
        assert np.allclose(z, want, rtol=0, atol=1e-14)
    zs = np.stack([oracle.philox_normals6(seed, i, 0, 0) for i in range(40000)])
    flat = zs.ravel()
    assert abs(flat.mean()) < 0.01 and abs(flat.var() - 1.0) < 0.01
    # each of the six slots is N(0, 1) and the slots are uncorrelated
    for k in range(6):
        assert stats.kstest(zs[:, k], "norm").pvalue > 1e-4, k
    c = np.corrcoef(zs.T)
    assert np.abs(c - np.eye(6)).max() < 0.03


def test_philox_replay_estimator_is_statistically_the_reference(oracle):
    """The replay (the GPU's stream in FP64) and the reference (mt19937) price the
    same option within 4 combined standard errors, for every model."""
    base = dict(spot=100.0, strike=95.0, t=1.0, vol=0.25, r=0.03, q=0.01, option_type=0,
                v0=0.05, kappa=1.5, theta=0.04, sigma=0.5, rho=-0.6)
    for model in (STANDARD, ANTITHETIC, TERMINAL_PLAIN, EULER, MILSTEIN, LOCAL_VOL, HESTON):
        steps = 16
        a, sa = oracle.philox_price(model, paths=20000, steps=steps, seed=11, **base)
        b, sb = oracle.price(model, paths=20000, steps=steps, seed=11, **base)
        z = (a - b) / math.hypot(sa, sb)
        assert abs(z) < 4.0, (model, a, b, z)


@pytest.mark.parametrize("model", ["heston", 0, 1, 2, 3, 4])
def test_cpu_timer_calls_the_reference_batch(ref, model):
    """The C++ timing harness behind the benchmark's CPU baselines calls the
    reference's batch entry points (Heston, terminal, stepwise signatures)
    with the benchmark's inputs: its prices sum to the Python binding's, bit
    for bit."""
    from oracle import oracle as orc

    if not orc.timer_available():
        pytest.skip("cpu_timer not built")
    rng = np.random.default_rng(3)
    n = 6
    b = dict(spot=np.full(n, 100.0), strike=rng.uniform(80, 120, n), t=rng.uniform(0.2, 2, n),
             vol=rng.uniform(0.1, 0.5, n), r=rng.uniform(0, 0.05, n), q=np.zeros(n),
             v0=rng.uniform(0.01, 0.09, n), kappa=rng.uniform(0.5, 5, n),
             theta=rng.uniform(0.01, 0.09, n), sigma=rng.uniform(0.1, 1, n),
             rho=rng.uniform(-0.9, 0, n), option_type=(np.arange(n) % 2).astype(np.int32),
             paths=np.full(n, 500, np.int32), steps=np.full(n, 20, np.int32),
             seed=np.arange(n, dtype=np.uint64) + 7)
    if model == "heston":
        symbol = "qk_mcm_heston_monte_carlo_price_batch"
        want = float(np.sum(ref.heston_batch(**{k: v for k, v in b.items() if k != "vol"})))
    else:
        symbol = orc.MODEL_BATCH_SYMBOL[model]
        want = float(np.sum([ref.price(model, b["spot"][i], b["strike"][i], b["t"][i], b["vol"][i],
                                       b["r"][i], b["q"][i], int(b["option_type"][i]),
                                       int(b["paths"][i]), int(b["steps"][i]), int(b["seed"][i]))
                             for i in range(n)]))
    secs, price_sum = orc.time_reference_batch(symbol, b, reps=2)
    assert len(secs) == 2 and all(s > 0 for s in secs)
    assert price_sum == want
