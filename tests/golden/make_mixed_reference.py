"""Reference CPU Monte Carlo prices and standard errors for a model-stratified
subset of the uneven mixed-model workload (quantkernel_b200.workloads.mixed():
4096 options, BSM-Euler / Milstein / constant-sigma local vol / Heston 1:1:1:1,
paths 2^U[12,20], steps 2^U[4,9]).

The subset has 64 options of each model: for every model the options with the
most steps, the most paths and the most path-steps in the draw (the corner of
up to 511 steps and 2^20 paths, where FP32 path state has the most steps to
drift over), and a seeded random draw of the rest.  Prices come from the
oracle's restatement of the reference pricers (euler_maruyama.cpp,
milstein.cpp, local_vol_monte_carlo.cpp, heston_monte_carlo.cpp with
mt19937_64 + polar normals), which equals the reference bit for bit; the
script re-checks one option per model against the compiled reference
(oracle/_ref) before writing, and adds the standard error the reference does
not compute.

    OMP_NUM_THREADS=<cores> python tests/golden/make_mixed_reference.py

About two minutes on 8 cores (2e10 path-steps).
"""

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "quant-kernel_b200"))

from oracle.oracle import HESTON, Oracle, Reference, reference_available  # noqa: E402
from quantkernel_b200 import workloads  # noqa: E402

OUT = Path(__file__).resolve().parent / "mixed_reference.json"
PER_MODEL = 64
CORNER = 4  # per model: options with the most steps, paths and path-steps
KEYS = ("spot", "strike", "t", "vol", "r", "q", "v0", "kappa", "theta", "sigma", "rho",
        "option_type", "paths", "steps", "seed")


def select(b, seed=17):
    """Indices of the subset, sorted: per model the corners, then random."""
    rng = np.random.default_rng(seed)
    out = []
    for m in np.unique(b["model"]):
        idx = np.nonzero(b["model"] == m)[0]
        paths = b["paths"][idx].astype(np.int64)
        steps = b["steps"][idx].astype(np.int64)
        chosen = []
        for key in (steps, paths, paths * steps):
            taken = 0
            for j in np.argsort(-key, kind="stable"):
                if int(idx[j]) in chosen:
                    continue
                chosen.append(int(idx[j]))
                taken += 1
                if taken == CORNER:
                    break
        rest = np.setdiff1d(idx, chosen)
        chosen += [int(x) for x in rng.choice(rest, PER_MODEL - len(chosen), replace=False)]
        out += chosen
    return np.array(sorted(out), np.int64)


def fingerprint(b, idx):
    """SHA-256 over the subset's inputs, so a test sees a changed workload."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(b["model"][idx], np.int32).tobytes())
    for k in KEYS:
        h.update(np.ascontiguousarray(b[k][idx]).tobytes())
    return h.hexdigest()


def main() -> None:
    b = workloads.mixed()
    idx = select(b)
    sub = {k: v[idx] for k, v in b.items()}
    orc = Oracle()
    price = np.empty(idx.size)
    se = np.empty(idx.size)
    t0 = time.perf_counter()
    for m in np.unique(sub["model"]):
        k = np.nonzero(sub["model"] == m)[0]
        part = {key: v[k] for key, v in sub.items()}
        if int(m) == HESTON:
            price[k], se[k] = orc.heston_batch(**{key: part[key] for key in
                                                  ("spot", "strike", "t", "r", "q", "v0", "kappa",
                                                   "theta", "sigma", "rho", "option_type", "paths",
                                                   "steps", "seed")})
        else:
            price[k], se[k] = orc.bsm_family_batch(int(m), *(part[key] for key in
                                                            ("spot", "strike", "t", "vol", "r",
                                                             "q", "option_type", "paths", "steps",
                                                             "seed")))
    dt = time.perf_counter() - t0
    checked = 0
    if reference_available():
        ref = Reference()
        for m in np.unique(sub["model"]):
            i = int(np.nonzero(sub["model"] == m)[0][0])
            a = {k: sub[k][i].item() for k in KEYS}
            want = ref.price(int(m), a["spot"], a["strike"], a["t"], a["vol"], a["r"], a["q"],
                             int(a["option_type"]), int(a["paths"]), int(a["steps"]),
                             int(a["seed"]), v0=a["v0"], kappa=a["kappa"], theta=a["theta"],
                             sigma=a["sigma"], rho=a["rho"])
            assert want == price[i], (int(m), want, price[i])
            checked += 1
    doc = {
        "source": "oracle restatement of yluoc/Quant-Kernel euler_maruyama.cpp, milstein.cpp, "
                  "local_vol_monte_carlo.cpp, heston_monte_carlo.cpp (bit-exact; "
                  f"{checked} options re-checked against the compiled reference)",
        "generator": "tests/golden/make_mixed_reference.py",
        "workload": "quantkernel_b200.workloads.mixed(): 4096 options, models 2/3/4/6 1:1:1:1, "
                    "paths 2^U[12,20], steps 2^U[4,9]",
        "subset": f"{PER_MODEL} per model: the {CORNER} with the most steps, most paths and most "
                  "path-steps, the rest seeded-random (seed 17)",
        "fingerprint": fingerprint(b, idx),
        "path_steps": int((sub["paths"].astype(np.int64) * sub["steps"]).sum()),
        "cpu_seconds": dt,
        "index": [int(i) for i in idx],
        "price": [float(x).hex() for x in price],
        "stderr": [float(x).hex() for x in se],
    }
    OUT.write_text(json.dumps(doc))
    print(f"wrote {OUT}: {idx.size} options, {doc['path_steps']:.3g} path-steps in {dt:.0f} s")


if __name__ == "__main__":
    main()
