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
Heston characteristic-function prices and the reference's BSM closed form.
"""

import json
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import (  # noqa: E402
    ANTITHETIC, EULER, HESTON, HESTON_LR_DELTA, LOCAL_VOL, MILSTEIN, STANDARD, Reference)

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

    doc = {
        "source": "yluoc/Quant-Kernel C ABI, compiled from cpp/src by oracle/Makefile (ref)",
        "generator": "tests/golden/make_golden.py",
        "mc_cases": cases,
        "heston_cf": cf,
        "bsm_cf_reference_as_cdf": bsm,
    }
    OUT.write_text(json.dumps(doc, indent=1))
    n_nan = sum(math.isnan(float.fromhex(c["price"])) for c in cases)
    print(f"wrote {OUT} ({len(cases)} MC cases, {n_nan} NaN results, {len(cf)} CF, {len(bsm)} BSM)")


if __name__ == "__main__":
    main()
