"""Failure detection without a GPU fault.

QK_B200_FAULT makes the host runtime report an allocation, launch or copy
failure at the point where it would call CUDA, without calling it (and
without touching the GPU).  Each call must come back as the reference's
error contract -- QK_ERR_RUNTIME_INIT with a "cuda error: ..." message, here
marked "[injected]" -- and the next call, disarmed, must succeed with the
same results as before: the context stays usable.
"""

import numpy as np
import pytest

from quantkernel_b200 import QK_MC_HESTON, QKRuntimeError, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture
def batch():
    return workloads.heston(4, paths=4096, steps=16, seed=21)


def test_injected_allocation_failure(qk, batch, monkeypatch):
    want = qk.heston_monte_carlo_price_batch(**batch)
    monkeypatch.setenv("QK_B200_FAULT", "alloc")
    with pytest.raises(QKRuntimeError, match=r"cudaErrorMemoryAllocation.*\[injected\]"):
        qk.plan(model=np.full(4, QK_MC_HESTON, np.int32), **batch)  # a new plan allocates
    monkeypatch.delenv("QK_B200_FAULT")
    plan = qk.plan(model=np.full(4, QK_MC_HESTON, np.int32), **batch)
    plan.execute()
    got, _ = plan.results()
    plan.close()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("site,err", [("launch", "cudaErrorLaunchFailure"),
                                      ("copy", "cudaErrorUnknown")])
def test_injected_launch_and_copy_failures(qk, batch, monkeypatch, site, err):
    want = qk.heston_monte_carlo_price_batch(**batch)
    monkeypatch.setenv("QK_B200_FAULT", site)
    with pytest.raises(QKRuntimeError, match=err + r".*\[injected\]"):
        qk.heston_monte_carlo_price_batch(**batch)
    # the scalar call of the same path returns NaN with the message set
    assert np.isnan(qk._lib.qk_mcm_heston_monte_carlo_price(100.0, 100.0, 1.0, 0.03, 0.0, 0.04,
                                                            2.0, 0.04, 0.3, -0.7, 0, 1000, 8, 1))
    assert "[injected]" in qk.get_last_error()
    monkeypatch.delenv("QK_B200_FAULT")
    assert np.array_equal(qk.heston_monte_carlo_price_batch(**batch), want)


def test_injected_failure_in_heston_cf(qk, monkeypatch):
    args = [np.array([v]) for v in (100.0, 100.0, 1.0, 0.03, 0.0, 0.04, 2.0, 0.04, 0.3, -0.7)]
    tail = [np.array([0], np.int32), np.array([1024], np.int32), np.array([120.0])]
    want = qk.heston_price_cf_batch(*args, *tail)
    monkeypatch.setenv("QK_B200_FAULT", "launch")
    with pytest.raises(QKRuntimeError, match=r"\[injected\]"):
        qk.heston_price_cf_batch(*args, *tail)
    monkeypatch.delenv("QK_B200_FAULT")
    assert np.array_equal(qk.heston_price_cf_batch(*args, *tail), want)
