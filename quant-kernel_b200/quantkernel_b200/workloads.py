"""Seeded synthetic option batches with the shapes of the benchmark workloads.

No market data is involved: every batch is drawn from numpy's
``default_rng(seed)`` with the distributions below, and option i gets the
Monte Carlo seed ``seed_base + i``.

* ``bsm_terminal``  -- 64 European calls/puts, terminal GBM, 131072 paths.
* ``heston``        -- 1024 Heston calls, 200 steps, 262144 paths.
* ``heston_cf``     -- Heston calls/puts for the characteristic-function
  pricer: the Heston batch's parameter ranges, 1024 integration steps,
  integration limit 120 (the reference engine's defaults).
* ``mixed``         -- 4096 options, BSM-Euler / BSM-Milstein / constant
  local-vol / Heston in 1:1:1:1, paths log-uniform in [2^12, 2^20], steps
  log-uniform in [16, 512].
"""

import numpy as np

from ._abi import QK_MC_EULER, QK_MC_HESTON, QK_MC_LOCAL_VOL, QK_MC_MILSTEIN


def bsm_terminal(n=64, paths=131072, seed=1, seed_base=1000):
    rng = np.random.default_rng(seed)
    return dict(
        spot=rng.uniform(80.0, 120.0, n),
        strike=rng.uniform(80.0, 120.0, n),
        t=rng.uniform(0.1, 2.0, n),
        vol=rng.uniform(0.1, 0.5, n),
        r=rng.uniform(0.0, 0.05, n),
        q=rng.uniform(0.0, 0.03, n),
        option_type=(np.arange(n) & 1).astype(np.int32),
        paths=np.full(n, paths, np.int32),
        seed=(np.arange(n, dtype=np.uint64) + np.uint64(seed_base)),
    )


def heston(n=1024, paths=262144, steps=200, seed=2, seed_base=5000):
    rng = np.random.default_rng(seed)
    return dict(
        spot=np.full(n, 100.0),
        strike=rng.uniform(70.0, 130.0, n),
        t=rng.uniform(0.25, 2.0, n),
        r=rng.uniform(0.0, 0.05, n),
        q=np.zeros(n),
        v0=rng.uniform(0.01, 0.09, n),
        kappa=rng.uniform(0.5, 5.0, n),
        theta=rng.uniform(0.01, 0.09, n),
        sigma=rng.uniform(0.1, 1.0, n),
        rho=rng.uniform(-0.9, 0.0, n),
        option_type=np.zeros(n, np.int32),
        paths=np.full(n, paths, np.int32),
        steps=np.full(n, steps, np.int32),
        seed=(np.arange(n, dtype=np.uint64) + np.uint64(seed_base)),
    )


def heston_cf(n=65536, seed=4, integration_steps=1024, integration_limit=120.0):
    h = heston(n, paths=2, steps=1, seed=seed)
    out = {k: h[k] for k in ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma",
                             "rho")}
    out["option_type"] = (np.arange(n) & 1).astype(np.int32)
    out["integration_steps"] = np.full(n, integration_steps, np.int32)
    out["integration_limit"] = np.full(n, integration_limit)
    return out


def mixed(n=4096, seed=3, seed_base=9000, log2_paths=(12.0, 20.0), log2_steps=(4.0, 9.0)):
    rng = np.random.default_rng(seed)
    kinds = np.array([QK_MC_EULER, QK_MC_MILSTEIN, QK_MC_LOCAL_VOL, QK_MC_HESTON], np.int32)
    model = kinds[np.arange(n) % 4]
    paths = np.floor(2.0 ** rng.uniform(*log2_paths, n)).astype(np.int32)
    steps = np.floor(2.0 ** rng.uniform(*log2_steps, n)).astype(np.int32)
    bsm = bsm_terminal(n, seed=seed + 100)
    hes = heston(n, seed=seed + 200)
    is_h = model == QK_MC_HESTON
    out = dict(
        model=model,
        spot=np.where(is_h, hes["spot"], bsm["spot"]),
        strike=np.where(is_h, hes["strike"], bsm["strike"]),
        t=np.where(is_h, hes["t"], bsm["t"]),
        vol=bsm["vol"],
        r=np.where(is_h, hes["r"], bsm["r"]),
        q=np.where(is_h, hes["q"], bsm["q"]),
        v0=hes["v0"], kappa=hes["kappa"], theta=hes["theta"], sigma=hes["sigma"], rho=hes["rho"],
        option_type=np.where(is_h, 0, bsm["option_type"]).astype(np.int32),
        paths=paths,
        steps=steps,
        seed=(np.arange(n, dtype=np.uint64) + np.uint64(seed_base)),
    )
    return out


def path_steps(batch, model=None) -> int:
    """Algorithmic path-steps of a batch (terminal models count one step)."""
    p = batch["paths"].astype(np.int64)
    s = batch.get("steps")
    if s is None:
        return int(p.sum())
    return int((p * s.astype(np.int64)).sum())
