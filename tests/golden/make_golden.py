"""Generates tests/golden/reference_mc.json from the reference library.

The reference (yluoc/Quant-Kernel) is compiled from its own sources by
`make -C oracle ref` into oracle/_ref/libquantkernel.so; this script calls its
C ABI on seeded inputs and stores every result as an exact hex float, so the
CPU oracle can be pinned bit for bit on machines without the reference.

    python tests/golden/make_golden.py      # needs oracle/_ref/libquantkernel.so

Cases: random small-size inputs for each Monte Carlo pricer on the hot path
(odd and even path counts, 1..64 steps), the edge cases the reference's own
tests and pricers define (t <= 1e-12, zero vol, invalid option type,
paths <= 1, steps <= 0, NaN inputs that Heston does not reject, extreme rho),
the five terminal variance-reduction estimators (control variates,
importance sampling, stratified, Sobol and Halton quasi-Monte Carlo), Heston
characteristic-function prices and the reference's BSM closed form.
"""

import json
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import (  # noqa: E402
    ANTITHETIC, EULER, HESTON, HESTON_LR_DELTA, IMPORTANCE_SAMPLING, LOCAL_VOL, MILSTEIN,
    QMC_HALTON, QMC_SOBOL, STANDARD, VR_MODELS, Reference)

OUT = Path(__file__).resolve().parent / "reference_mc.json"


def hx(x: float) -> str:
    return float(x).hex()


def main() -> None:
    ref = Reference()
    rng = np.random.default_rng(20261203)
    cases = []

    def add(model, **kw):
        args = dict(spot=100.0, strike=100.0, t=1.0, vol=0.2, r=0.05, q=0.0, option_type=0,
                    paths=1000, steps=10, seed=1, v0=0.04, kappa=2.0, theta=0.04, sigma=0.3,
                    rho=-0.7)
        args.update(kw)
        price = ref.price(model, **args)
        cases.append({"model": model, "args": {k: (hx(v) if isinstance(v, float) else int(v))
                                                for k, v in args.items()},
                      "price": hx(price)})

    # the reference's own golden seeds (cpp/tests/test_monte_carlo.cpp:57-73)
    add(STANDARD, paths=50000, seed=12345, option_type=0)
    add(STANDARD, paths=50000, seed=12345, option_type=1)
    add(EULER, paths=10000, steps=100, seed=12345, option_type=0)

    for model in (STANDARD, ANTITHETIC, EULER, MILSTEIN, LOCAL_VOL, HESTON):
        for _ in range(10):
            paths = int(rng.integers(2, 3000))
            kw = dict(spot=float(rng.uniform(80, 120)), strike=float(rng.uniform(80, 120)),
                      t=float(rng.uniform(0.1, 2.0)), vol=float(rng.uniform(0.1, 0.5)),
                      r=float(rng.uniform(0.0, 0.05)), q=float(rng.uniform(0.0, 0.03)),
                      option_type=int(rng.integers(0, 2)), paths=paths,
                      steps=int(rng.integers(1, 65)), seed=int(rng.integers(0, 2**63)))
            if model == HESTON:
                kw.update(v0=float(rng.uniform(0.01, 0.09)), kappa=float(rng.uniform(0.5, 5)),
                          theta=float(rng.uniform(0.01, 0.09)), sigma=float(rng.uniform(0.1, 1.0)),
                          rho=float(rng.uniform(-0.9, 0.0)))
            add(model, **kw)
        # edge cases of the pricers' entry checks
        add(model, t=1e-14, spot=110.0)                  # undiscounted intrinsic
        add(model, t=1e-14, spot=90.0, option_type=1)
        add(model, option_type=7)                        # invalid type -> NaN
        add(model, paths=1)                              # paths <= 1 -> NaN
        add(model, paths=3, seed=123)                    # odd path count
        add(model, paths=2, seed=123)
        add(model, spot=-1.0)                            # bad spot -> NaN
        if model in (EULER, MILSTEIN, LOCAL_VOL, HESTON):
            add(model, steps=0)                          # steps <= 0 -> NaN
    add(STANDARD, vol=0.0)                               # zero-vol discounted forward
    add(STANDARD, vol=0.0, option_type=1, spot=90.0)
    add(ANTITHETIC, vol=0.0)                             # no zero-vol branch here
    add(STANDARD, vol=float("nan"))                      # non-finite -> NaN
    add(EULER, r=float("inf"))
    for rho in (-0.99, 0.0, 0.99, -1.0, 1.0):
        add(HESTON, rho=rho, paths=2000, steps=20)
    add(HESTON, rho=1.5)                                 # out of range -> NaN
    add(HESTON, v0=0.0, paths=500, steps=8)
    add(HESTON, sigma=0.0, paths=500, steps=8)
    add(HESTON, kappa=0.0, paths=500, steps=8)
    # NaN parameters Heston does not reject (heston_monte_carlo.cpp:18-24)
    for field in ("spot", "strike", "q", "v0", "kappa", "theta", "sigma", "rho", "t", "r"):
        for ot in (0, 1):
            add(HESTON, **{field: float("nan")}, option_type=ot, paths=64, steps=4)

    # Heston likelihood-ratio delta (heston_lr_delta.cpp); `vol` carries weight_clip
    for _ in range(10):
        add(HESTON_LR_DELTA, spot=float(rng.uniform(80, 120)), strike=float(rng.uniform(80, 120)),
            t=float(rng.uniform(0.1, 2.0)), r=float(rng.uniform(0.0, 0.05)),
            q=float(rng.uniform(0.0, 0.03)), option_type=int(rng.integers(0, 2)),
            paths=int(rng.integers(2, 3000)), steps=int(rng.integers(1, 40)),
            seed=int(rng.integers(0, 2**63)), v0=float(rng.uniform(0.01, 0.09)),
            kappa=float(rng.uniform(0.5, 5)), theta=float(rng.uniform(0.01, 0.09)),
            sigma=float(rng.uniform(0.1, 1.0)), rho=float(rng.uniform(-0.9, 0.0)),
            vol=float(rng.choice([0.5, 2.0, 6.0])))
    add(HESTON_LR_DELTA, vol=6.0, t=1e-14, spot=110.0)              # intrinsic delta 1
    add(HESTON_LR_DELTA, vol=6.0, t=1e-14, spot=90.0, option_type=1)  # -1
    add(HESTON_LR_DELTA, vol=0.0)                                     # clip <= 0 -> NaN
    add(HESTON_LR_DELTA, vol=6.0, v0=0.0, paths=100, steps=4)         # zero score -> 0
    add(HESTON_LR_DELTA, vol=6.0, paths=3, seed=5)                    # odd count
    add(HESTON_LR_DELTA, vol=6.0, paths=1)                            # NaN

    # terminal variance-reduction estimators (own generator: the draws above
    # and the closed-form lists below keep their values)
    rng_vr = np.random.default_rng(20261206)
    for model in VR_MODELS:
        for _ in range(10):
            kw = dict(spot=float(rng_vr.uniform(80, 120)), strike=float(rng_vr.uniform(80, 120)),
                      t=float(rng_vr.uniform(0.1, 2.0)), vol=float(rng_vr.uniform(0.1, 0.5)),
                      r=float(rng_vr.uniform(0.0, 0.05)), q=float(rng_vr.uniform(0.0, 0.03)),
                      option_type=int(rng_vr.integers(0, 2)), paths=int(rng_vr.integers(2, 3000)),
                      steps=1, seed=int(rng_vr.integers(0, 2**63)))
            if model == IMPORTANCE_SAMPLING:
                kw["shift"] = float(rng_vr.uniform(-1.0, 1.0))
            add(model, **kw)
        extra = {"shift": 0.4} if model == IMPORTANCE_SAMPLING else {}
        add(model, t=1e-14, spot=110.0, **extra)         # undiscounted intrinsic
        add(model, t=1e-14, spot=90.0, option_type=1, **extra)
        add(model, option_type=7, **extra)               # invalid type -> NaN
        add(model, paths=1, **extra)                     # NaN
        add(model, paths=2, seed=123, **extra)           # NaN for control variates only
        add(model, paths=3, seed=123, **extra)
        add(model, vol=0.0, **extra)                     # no zero-vol branch here
        add(model, vol=float("nan"), **extra)
        add(model, spot=-1.0, **extra)
        add(model, paths=16384, **extra)                 # the reference's QMC test size
    add(IMPORTANCE_SAMPLING, shift=float("nan"))          # non-finite shift -> NaN
    add(IMPORTANCE_SAMPLING, shift=float("inf"))
    add(IMPORTANCE_SAMPLING, shift=0.0, paths=500)
    add(IMPORTANCE_SAMPLING, shift=2.5, strike=150.0, paths=4000)  # deep OTM call, shifted up
    for model in (QMC_SOBOL, QMC_HALTON):
        add(model, paths=1 << 20)                        # 2^20 points
        add(model, paths=1000003, option_type=1, strike=90.0)

    cf = []
    for _ in range(24):
        a = dict(spot=100.0, strike=float(rng.uniform(70, 130)), t=float(rng.uniform(0.25, 2)),
                 r=float(rng.uniform(0, 0.05)), q=0.0, v0=float(rng.uniform(0.01, 0.09)),
                 kappa=float(rng.uniform(0.5, 5)), theta=float(rng.uniform(0.01, 0.09)),
                 sigma=float(rng.uniform(0.1, 1.0)), rho=float(rng.uniform(-0.9, 0.0)),
                 option_type=int(rng.integers(0, 2)))
        price = ref.heston_cf(**a)
        cf.append({"args": {k: (hx(v) if isinstance(v, float) else v) for k, v in a.items()},
                   "price": hx(price)})

    bsm = []
    for _ in range(24):
        a = dict(spot=float(rng.uniform(80, 120)), strike=float(rng.uniform(80, 120)),
                 t=float(rng.uniform(0.1, 2)), vol=float(rng.uniform(0.1, 0.5)),
                 r=float(rng.uniform(0, 0.05)), q=float(rng.uniform(0, 0.03)),
                 option_type=int(rng.integers(0, 2)))
        bsm.append({"args": {k: (hx(v) if isinstance(v, float) else v) for k, v in a.items()},
                    "price": hx(ref.bsm(**a))})

    # Heston CF with explicit integration settings and the entry checks of
    # heston.cpp:10-24 (kept after the lists above so their draws do not move)
    cf_edges = []

    def add_cf(**kw):
        a = dict(spot=100.0, strike=100.0, t=1.0, r=0.03, q=0.01, v0=0.04, kappa=2.0,
                 theta=0.04, sigma=0.3, rho=-0.7, option_type=0, integration_steps=1024,
                 integration_limit=120.0)
        a.update(kw)
        cf_edges.append({"args": {k: (hx(v) if isinstance(v, float) else int(v))
                                  for k, v in a.items()},
                         "price": hx(ref.heston_cf(**a))})

    rng_cf = np.random.default_rng(20261204)
    for steps in (16, 17, 64, 65, 100, 512, 1024, 4096, 8192):
        for lim in (1e-5, 50.0, 120.0, 500.0):
            add_cf(integration_steps=steps, integration_limit=lim,
                   strike=float(rng_cf.uniform(60, 150)), t=float(rng_cf.uniform(0.05, 3)),
                   v0=float(rng_cf.uniform(0.005, 0.2)), kappa=float(rng_cf.uniform(0.2, 6)),
                   theta=float(rng_cf.uniform(0.005, 0.2)), sigma=float(rng_cf.uniform(0.05, 1.5)),
                   rho=float(rng_cf.uniform(-0.95, 0.5)), q=float(rng_cf.uniform(0, 0.04)),
                   option_type=int(rng_cf.integers(0, 2)))
    # the reference's own Python cases (test_closed_form_api.py:18-46,
    # test_heston_fourier.py:18-33)
    add_cf(r=0.02, sigma=0.5, rho=-0.5)
    for steps in (64, 512):
        add_cf(strike=130.0, t=2.0, r=0.05, q=0.01, v0=0.09, kappa=0.8, theta=0.09, sigma=1.0,
               rho=-0.9, integration_limit=300.0, integration_steps=steps)
    for ot in (0, 1):
        add_cf(option_type=ot, integration_steps=8192, integration_limit=500.0)
    add_cf(integration_steps=15)                 # < 16 -> NaN
    add_cf(integration_steps=0)
    add_cf(integration_steps=-5)
    add_cf(integration_limit=1e-6)               # <= 1e-6 -> NaN
    add_cf(option_type=2)                        # invalid type -> NaN
    add_cf(option_type=-1)
    add_cf(t=1e-14, spot=110.0)                  # intrinsic, undiscounted
    add_cf(t=1e-14, spot=90.0, option_type=1)
    add_cf(t=0.0, spot=90.0)
    add_cf(t=-0.1)                               # NaN
    add_cf(spot=0.0)
    add_cf(strike=-1.0)
    add_cf(v0=-0.01)
    add_cf(v0=0.0)                               # allowed
    add_cf(theta=0.0)                            # allowed
    add_cf(theta=-0.01)
    add_cf(kappa=0.0)
    add_cf(sigma=0.0)
    add_cf(sigma=1e-4)                           # near-BSM limit
    add_cf(rho=-1.0)
    add_cf(rho=1.0)
    add_cf(rho=0.999)
    add_cf(rho=-0.999)
    add_cf(r=float("nan"))
    add_cf(q=float("inf"))
    add_cf(sigma=float("nan"))
    add_cf(t=30.0, kappa=0.1, sigma=2.0)         # long maturity, strong vol of vol
    add_cf(strike=1000.0)                        # deep OTM call -> ~0
    add_cf(strike=1.0, option_type=1)            # deep OTM put -> ~0
    add_cf(strike=1.0)                           # deep ITM call
    add_cf(t=1e-6)                               # just above the intrinsic cut
    # beta(-i) = kappa - rho sigma <= 0: phi(-i) is NaN (0/0 or x/0 in g), so
    # P1 is NaN and the price is NaN; = 0 exactly, and < 0
    add_cf(kappa=0.5, rho=0.5, sigma=1.0)
    add_cf(kappa=0.1922, rho=0.3328, sigma=1.83, v0=0.2991, theta=0.2253, t=0.0552)
    # wide ranges: positive rho, large vol of vol, short and long maturities
    rng_w = np.random.default_rng(20261205)
    for _ in range(40):
        add_cf(spot=float(rng_w.uniform(50, 150)), strike=float(rng_w.uniform(40, 200)),
               t=float(rng_w.uniform(0.02, 5)), r=float(rng_w.uniform(-0.01, 0.08)),
               q=float(rng_w.uniform(0, 0.05)), v0=float(rng_w.uniform(0, 0.3)),
               kappa=float(rng_w.uniform(0.05, 8)), theta=float(rng_w.uniform(0, 0.3)),
               sigma=float(rng_w.uniform(0.02, 2)), rho=float(rng_w.uniform(-0.99, 0.99)),
               option_type=int(rng_w.integers(0, 2)),
               integration_steps=int(rng_w.choice([16, 64, 200, 512, 1024, 2048])),
               integration_limit=float(rng_w.choice([30.0, 120.0, 300.0])))

    # Heston COS expansion (cos_method.cpp:30-58): settings, entry checks and
    # the degenerate parameters the COS entry does not reject
    cos = []

    def add_cos(**kw):
        a = dict(spot=100.0, strike=100.0, t=1.0, r=0.03, q=0.01, v0=0.04, kappa=2.0,
                 theta=0.04, sigma=0.3, rho=-0.7, option_type=0, n_terms=256,
                 truncation_width=10.0)
        a.update(kw)
        cos.append({"args": {k: (hx(v) if isinstance(v, float) else int(v)) for k, v in a.items()},
                    "price": hx(ref.heston_cos(**a))})

    rng_cos = np.random.default_rng(20261207)
    for _ in range(60):
        add_cos(spot=float(rng_cos.uniform(50, 150)), strike=float(rng_cos.uniform(40, 200)),
                t=float(rng_cos.uniform(0.02, 5)), r=float(rng_cos.uniform(-0.01, 0.08)),
                q=float(rng_cos.uniform(0, 0.05)), v0=float(rng_cos.uniform(0, 0.3)),
                kappa=float(rng_cos.uniform(0.05, 8)), theta=float(rng_cos.uniform(0, 0.3)),
                sigma=float(rng_cos.uniform(0.02, 2)), rho=float(rng_cos.uniform(-0.99, 0.99)),
                option_type=int(rng_cos.integers(0, 2)),
                n_terms=int(rng_cos.choice([8, 16, 64, 128, 256, 512, 1024])),
                truncation_width=float(rng_cos.choice([2.0, 6.0, 10.0, 14.0])))
    for ot in (0, 1):  # the reference's own case (test_heston_fourier.py:18-21)
        add_cos(option_type=ot)
    add_cos(n_terms=7)                    # < 8 -> NaN
    add_cos(truncation_width=0.0)         # <= 0 -> NaN
    add_cos(truncation_width=-1.0)
    add_cos(option_type=2)
    add_cos(t=1e-14, spot=110.0)          # intrinsic
    add_cos(t=0.0, spot=90.0, option_type=1)
    add_cos(t=-0.1)
    add_cos(spot=0.0)
    add_cos(v0=-0.01)
    add_cos(v0=0.0)
    add_cos(v0=0.0, theta=0.0)            # empty interval -> NaN
    add_cos(sigma=0.0)                    # NaN sum -> max(0, NaN) = 0
    add_cos(sigma=0.0, option_type=1)
    add_cos(kappa=0.0)
    add_cos(kappa=-1.0)
    add_cos(rho=1.0)
    add_cos(rho=-1.0)
    add_cos(sigma=-0.3)
    add_cos(r=float("nan"))
    add_cos(truncation_width=float("inf"))
    add_cos(strike=1000.0)                # log K beyond b: no sum, call 0
    add_cos(strike=1.0, option_type=1)

    doc = {
        "source": "yluoc/Quant-Kernel C ABI, compiled from cpp/src by oracle/Makefile (ref)",
        "generator": "tests/golden/make_golden.py",
        "mc_cases": cases,
        "heston_cf": cf,
        "heston_cf_edges": cf_edges,
        "heston_cos": cos,
        "bsm_cf_reference_as_cdf": bsm,
    }
    OUT.write_text(json.dumps(doc, indent=1))
    n_nan = sum(math.isnan(float.fromhex(c["price"])) for c in cases)
    print(f"wrote {OUT} ({len(cases)} MC cases, {n_nan} NaN results, {len(cf)} CF, {len(bsm)} BSM)")


if __name__ == "__main__":
    main()
