"""Reference CPU Monte Carlo prices and standard errors for the full Heston
benchmark workload (1024 calls x 262144 paths x 200 steps: the
quantkernel_b200.workloads.heston() draw, seed 2, option seeds 5000 + i).

The prices come from the oracle's restatement of the reference pricer
(heston_monte_carlo.cpp with mt19937_64 + polar normals), which equals the
reference bit for bit; the script re-checks three options against the
compiled reference (oracle/_ref) before writing, and adds the standard error
the reference does not compute.

    OMP_NUM_THREADS=<cores> python tests/golden/make_heston_full_reference.py

About 10 minutes on 8 cores (5.37e10 path-steps).
"""

import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "quant-kernel_b200"))

from oracle.oracle import Oracle, Reference, reference_available  # noqa: E402
from quantkernel_b200 import workloads  # noqa: E402

OUT = Path(__file__).resolve().parent / "heston_full_reference.json"


def main() -> None:
    h = workloads.heston()
    t0 = time.perf_counter()
    price, se = Oracle().heston_batch(**h)
    dt = time.perf_counter() - t0
    checked = 0
    if reference_available():
        ref = Reference()
        for i in (0, 511, 1023):
            one = {k: v[i:i + 1] for k, v in h.items()}
            assert ref.heston_batch(**one)[0] == price[i], i
            checked += 1
    doc = {
        "source": "oracle restatement of yluoc/Quant-Kernel heston_monte_carlo.cpp "
                  f"(bit-exact; {checked} options re-checked against the compiled reference)",
        "generator": "tests/golden/make_heston_full_reference.py",
        "workload": "quantkernel_b200.workloads.heston(): 1024 calls x 262144 paths x 200 steps",
        "cpu_seconds": dt,
        "price": [float(x).hex() for x in price],
        "stderr": [float(x).hex() for x in se],
    }
    OUT.write_text(json.dumps(doc))
    print(f"wrote {OUT} in {dt:.0f} s")


if __name__ == "__main__":
    main()
