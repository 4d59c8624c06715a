"""One batch across GPUs through the library's own NCCL path, on one GPU.

This pool gives one GPU per run, so the communicator here has one rank: the
sharded execute then runs its whole code path -- the tiling check, the tile
range launch, the grouped broadcast, the finalize over all options -- and
must equal a plain execute bit for bit.  The partition itself is checked with
several ranks by running each rank's tile range of the same plan in turn
(execute_tiles, no exchange needed in one memory) and finalizing: any range
or group-clipping error changes the bits.  No two processes share the GPU
(NCCL refuses one GPU for two ranks, and ranks that wait on each other must
not share one GPU).
"""

import numpy as np
import pytest

from quantkernel_b200 import (QK_MC_HESTON, QK_PLAN_FAMILY_GRIDS, QK_PLAN_NO_ANTITHETIC,
                              QK_PLAN_PERSISTENT, QKInvalidInputError, QKRuntimeError, workloads)
from quantkernel_b200.sharding import DistContext, new_id

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dist(qk):
    qk.set_device(0)
    ctx = DistContext(new_id(qk), 1, 0, qk)
    yield ctx
    ctx.close()


def _plans(qk):
    h = workloads.heston(40, paths=30001, steps=23, seed=31)
    m = workloads.mixed(120, seed=32, log2_paths=(8.0, 14.0), log2_steps=(2.0, 6.0))
    return [
        ("heston", dict(model=np.full(40, QK_MC_HESTON, np.int32), **h), 0),
        ("heston plain paths", dict(model=np.full(40, QK_MC_HESTON, np.int32), **h),
         QK_PLAN_NO_ANTITHETIC),
        ("mixed, persistent kernel", m, QK_PLAN_PERSISTENT),
        ("mixed, per-family grids", m, QK_PLAN_FAMILY_GRIDS),
        ("terminal", dict(model=np.full(64, 1, np.int32), **workloads.bsm_terminal(64, paths=9001)),
         0),
    ]


def test_sharded_execute_equals_execute(qk, dist):
    for name, batch, flags in _plans(qk):
        plan = qk.plan(**batch, flags=flags)
        plan.execute()
        want_p, want_se = plan.results()
        for _ in range(2):  # and again on the same plan and communicator
            dist.execute(plan)
            p, se = plan.results()
            assert np.array_equal(p, want_p, equal_nan=True), name
            assert np.array_equal(se, want_se, equal_nan=True), name
        plan.close()


@pytest.mark.parametrize("world", [2, 3, 5, 8])
def test_every_ranks_tile_range_then_finalize_equals_execute(qk, world):
    for name, batch, flags in _plans(qk):
        plan = qk.plan(**batch, flags=flags)
        plan.execute()
        want_p, want_se = plan.results()
        b = plan.shard_bounds(world)
        _, n_tiles, nbytes = plan.device_partials()
        assert b[0] == 0 and b[-1] == n_tiles and np.all(np.diff(b) >= 0) and nbytes == 64
        for k in reversed(range(world)):  # any order: tile sums land in their own slots
            plan.execute_tiles(int(b[k]), int(b[k + 1]))
        plan.finalize()
        p, se = plan.results()
        assert np.array_equal(p, want_p, equal_nan=True), (name, world)
        assert np.array_equal(se, want_se, equal_nan=True), (name, world)
        with pytest.raises(QKInvalidInputError):
            plan.execute_tiles(0, n_tiles + 1)
        plan.close()


def test_sharded_mixed_batch_equals_mixed_batch(qk, dist):
    b = workloads.mixed(200, seed=33, log2_paths=(8.0, 13.0), log2_steps=(2.0, 5.0))
    b["spot"][3] = -1.0  # invalid element: NaN on every path the same way
    want_p, want_se = qk.mixed_price_batch(**b)
    p, se = dist.mixed_price_batch(**b)
    assert np.array_equal(p, want_p, equal_nan=True)
    assert np.array_equal(se, want_se, equal_nan=True)
    assert np.isnan(p[3])


def test_injected_collective_failure_leaves_the_next_call_correct(qk, dist, monkeypatch):
    b = workloads.mixed(32, seed=34, log2_paths=(8.0, 11.0), log2_steps=(2.0, 4.0))
    want_p, _ = qk.mixed_price_batch(**b)
    monkeypatch.setenv("QK_B200_FAULT", "collective")
    with pytest.raises(QKRuntimeError, match=r"\[injected\]"):
        dist.mixed_price_batch(**b)
    monkeypatch.delenv("QK_B200_FAULT")
    p, _ = dist.mixed_price_batch(**b)
    assert np.array_equal(p, want_p)


def test_aborted_communicator_refuses_further_work(qk):
    # host-side failure handling: after qk_dist_abort (what a watchdog thread
    # calls when a peer is lost) the communicator is never used again
    qk.set_device(0)
    ctx = DistContext(new_id(qk), 1, 0, qk)
    b = workloads.mixed(16, seed=35, log2_paths=(8.0, 10.0), log2_steps=(2.0, 3.0))
    plan = qk.plan(**b)
    ctx.execute(plan)
    want = plan.results()[0]
    ctx.abort()
    with pytest.raises(QKInvalidInputError, match="aborted"):
        ctx.execute(plan)
    ctx.close()
    plan.execute()  # the plan and the device stay usable
    assert np.array_equal(plan.results()[0], want)
    plan.close()
