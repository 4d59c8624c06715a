"""API parity guards, after the reference's own (python/tests/test_parity_guard.py:
scalar/batch pairs complete, header and implementation in sync, accelerator
routing covers every batch method).  They read source files and the built
library's export table; no GPU.

Scope: the reference-named pricing calls this library exports (the Monte Carlo
path and the Heston Fourier pricers).  The library's own additions (plans,
devices, the surrogate, the allocation-free entry) have no scalar/batch pairing
to keep.
"""

import re
import subprocess
from pathlib import Path

import pytest

from quantkernel_b200 import QuantAccelerator, QuantKernel

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "qk_api.h"
ENGINE = ROOT / "quant-kernel_b200" / "quantkernel_b200" / "engine.py"
LIB = ROOT / "quant-kernel_b200" / "quantkernel_b200" / "libqk_b200.so"
PRICING_PREFIXES = ("qk_mcm_", "qk_cf_", "qk_ftm_")
NOT_PRICING = ("qk_mcm_plan_", "qk_mcm_mixed_", "qk_mcm_heston_monte_carlo_price_batch_noalloc")


def _header_funcs():
    text = "".join(h.read_text() for h in sorted((ROOT / "include").glob("*.h")))
    return re.findall(r"QK_EXPORT\s+[\w\s\*]+?\b(qk_\w+)\s*\(", text)


def _pricing_scalars(funcs):
    return sorted(f for f in funcs if f.startswith(PRICING_PREFIXES) and not f.endswith("_batch")
                  and not f.startswith(NOT_PRICING))


def test_c_api_scalar_batch_pairs_are_complete():
    """Every scalar pricing call has its batch and price+SE variants (the
    Fourier pricers are deterministic: batch only)."""
    funcs = set(_header_funcs())
    scalars = _pricing_scalars(funcs)
    assert len(scalars) == 14, scalars
    missing = [f for f in scalars if f + "_batch" not in funcs]
    assert not missing, f"scalar calls without *_batch: {missing}"
    mc = [f for f in scalars if f.startswith("qk_mcm_")]
    missing_se = [f for f in mc if f + "_se_batch" not in funcs]
    assert not missing_se, f"Monte Carlo calls without *_se_batch: {missing_se}"


def test_c_api_header_and_library_stay_in_sync():
    funcs = set(_header_funcs())
    if not LIB.exists():
        pytest.skip("library not built")
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines()
                if ln.split() and ln.split()[-1].startswith("qk_") and " T " in ln}
    assert funcs == exported, (sorted(funcs - exported), sorted(exported - funcs))


def test_engine_scalar_batch_pairs_are_complete():
    methods = re.findall(r"^    def ([a-zA-Z0-9_]+)\(", ENGINE.read_text(), re.M)
    qk_methods = set(m for m in methods if hasattr(QuantKernel, m))
    pricing = sorted(m for m in qk_methods
                     if (m.endswith("_price") or m.endswith("_price_cf") or m == "heston_lr_delta"))
    assert len(pricing) == 14, pricing
    missing = [m for m in pricing if m + "_batch" not in qk_methods]
    assert not missing, f"engine scalar methods without *_batch: {missing}"


def test_accelerator_native_batch_map_covers_all_scalar_methods():
    """The reference requires every batch-capable scalar method to be routed
    (test_parity_guard.py:111-121); here every one routes to the GPU batch."""
    methods = re.findall(r"^    def ([a-zA-Z0-9_]+)\(", ENGINE.read_text(), re.M)
    pricing = sorted(m for m in set(methods) if hasattr(QuantKernel, m)
                     and (m.endswith("_price") or m.endswith("_price_cf") or m == "heston_lr_delta"))
    native = QuantAccelerator._NATIVE_BATCH_METHODS
    missing = [m for m in pricing if m not in native]
    assert not missing, f"scalar methods the accelerator does not route: {missing}"
    for scalar, batch in native.items():
        assert batch == scalar + "_batch" and hasattr(QuantKernel, batch), (scalar, batch)


def test_python_constants_match_the_header():
    """Every #define of include/qk_abi.h and include/qk_api.h that the Python
    package mirrors (ABI version, option types, error codes, model codes,
    plan flags) has the header's value."""
    import quantkernel_b200._abi as abi

    text = (ROOT / "include" / "qk_abi.h").read_text() + HEADER.read_text()
    defines = dict(re.findall(r"#define\s+(QK_[A-Z0-9_]+)\s+\(?(-?(?:0x)?[0-9A-Fa-f]+)\)?", text))
    checked = 0
    for name, value in defines.items():
        if hasattr(abi, name):
            assert getattr(abi, name) == int(value, 0), name
            checked += 1
    assert checked >= 25, checked
    for flag in ("QK_PLAN_PERSISTENT", "QK_PLAN_GRAPH", "QK_PLAN_NO_ANTITHETIC", "QK_PLAN_TIMING",
                 "QK_PLAN_AUTOTUNE", "QK_PLAN_FAMILY_GRIDS", "QK_PLAN_STEP_UNROLL2"):
        assert hasattr(abi, flag) and flag in defines, flag
