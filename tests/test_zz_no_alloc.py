"""The allocation-free Heston entry point, qk_mcm_heston_monte_carlo_price_batch_noalloc.

It exists for callers that cannot call cudaMalloc -- a service whose host
framework owns every device allocation, a process whose GPU footprint is fixed
after start-up, a latency-bound path that cannot pay for an allocation -- and
keeps all its device buffers in one fixed array per GPU.  These tests call it
through the C ABI and require the same prices and standard errors as the
regular entry point, on two calls in a row (the second reuses the array the
first left behind), and a clear rejection of batches beyond its limits.

This file is collected last, so a run that stops at its first failure has
already run every other test; it also passes alone in a fresh process.
"""

import ctypes as ct

import numpy as np
import pytest

from quantkernel_b200 import workloads

pytestmark = pytest.mark.gpu

PD = ct.POINTER(ct.c_double)
PI32 = ct.POINTER(ct.c_int32)
PU64 = ct.POINTER(ct.c_uint64)
KEYS = ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho",
        "option_type", "paths", "steps", "seed")


def _noalloc(qk, batch):
    arrs = []
    for k in KEYS:
        a = np.ascontiguousarray(batch[k])
        arrs.append(a)
    ptrs = [a.ctypes.data_as(PD if a.dtype == np.float64 else PI32 if a.dtype == np.int32 else PU64)
            for a in arrs]
    n = len(arrs[0])
    out = np.full(n, -1.0)
    se = np.full(n, -1.0)
    rc = qk._lib.qk_mcm_heston_monte_carlo_price_batch_noalloc(*ptrs, n, out.ctypes.data_as(PD),
                                                                se.ctypes.data_as(PD))
    return rc, out, se


def test_noalloc_matches_regular_entry_on_two_calls_in_a_row(qk):
    first = workloads.heston(96, paths=50001, steps=40, seed=21)
    first["spot"][5] = -1.0          # invalid element -> NaN, as in the regular call
    first["t"][7] = 1e-14            # intrinsic value
    second = workloads.heston(40, paths=262144, steps=24, seed=22)
    for batch in (first, second):
        want_p, want_se = qk.heston_monte_carlo_price_se_batch(**batch)
        rc, got_p, got_se = _noalloc(qk, batch)
        assert rc == 0, qk.get_last_error()
        # the tolerance the other parity tests use between launch strategies
        np.testing.assert_allclose(got_p, want_p, rtol=1e-13, atol=0, equal_nan=True)
        np.testing.assert_allclose(got_se, want_se, rtol=1e-10, atol=0, equal_nan=True)
    assert np.isnan(got_p).sum() == 0


def test_noalloc_rejects_batches_beyond_its_limits(qk):
    too_many = workloads.heston(4097, paths=64, steps=2, seed=1)
    qk.clear_last_error()
    rc, _, _ = _noalloc(qk, too_many)
    assert rc == -2
    assert "no-allocation limit of 4096" in qk.get_last_error()
    # an option never has more than 4096 tiles: 65 options of 2^22 paths need 266,240
    too_long = workloads.heston(65, paths=2**22, steps=2, seed=1)
    rc, _, _ = _noalloc(qk, too_long)
    assert rc == -2
    assert "tiles exceed the no-allocation limit of 262144" in qk.get_last_error()


def test_noalloc_tile_geometry_past_2_22_paths(qk):
    # one option of 2^23 paths: past 2^22 paths an option keeps 4096 tiles and
    # each tile holds more than 512 pairs
    big = workloads.heston(1, paths=2**23, steps=3, seed=23)
    want_p, want_se = qk.heston_monte_carlo_price_se_batch(**big)
    rc, got_p, got_se = _noalloc(qk, big)
    assert rc == 0, qk.get_last_error()
    np.testing.assert_allclose(got_p, want_p, rtol=1e-13, atol=0)
    np.testing.assert_allclose(got_se, want_se, rtol=1e-10, atol=0)


def test_noalloc_at_exactly_the_tile_limit(qk):
    # 64 options of 2^22 paths take 64 x 4096 = 262,144 tiles: the limit itself
    edge = workloads.heston(64, paths=2**22, steps=2, seed=24)
    rc, got_p, got_se = _noalloc(qk, edge)
    assert rc == 0, qk.get_last_error()
    want_p, want_se = qk.heston_monte_carlo_price_se_batch(**edge)
    np.testing.assert_allclose(got_p, want_p, rtol=1e-13, atol=0)
    np.testing.assert_allclose(got_se, want_se, rtol=1e-10, atol=0)


@pytest.mark.parametrize("site,err", [("launch", "cudaErrorLaunchFailure"),
                                      ("copy", "cudaErrorUnknown")])
def test_noalloc_injected_failures_leave_the_next_call_correct(qk, monkeypatch, site, err):
    # host-side injection: the call reports the failure without touching the
    # GPU at that site, and the next call, disarmed, prices as the regular entry
    batch = workloads.heston(8, paths=8192, steps=16, seed=25)
    want_p, want_se = qk.heston_monte_carlo_price_se_batch(**batch)
    monkeypatch.setenv("QK_B200_FAULT", site)
    rc, _, _ = _noalloc(qk, batch)
    assert rc == -4
    msg = qk.get_last_error()
    assert err in msg and "[injected]" in msg
    monkeypatch.delenv("QK_B200_FAULT")
    rc, got_p, got_se = _noalloc(qk, batch)
    assert rc == 0, qk.get_last_error()
    np.testing.assert_allclose(got_p, want_p, rtol=1e-13, atol=0)
    np.testing.assert_allclose(got_se, want_se, rtol=1e-10, atol=0)
