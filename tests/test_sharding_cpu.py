"""Multi-rank host logic of the sharded path, on CPU with the gloo backend
(world size 2).  The pricer is a deterministic stand-in computed from each
option's own inputs, so the test checks partitioning, ordering and the gather
-- the parts that do not need a GPU."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from quantkernel_b200 import workloads
from quantkernel_b200.sharding import option_cost, partition_by_cost, price_sharded


def _fake_pricer(b):
    # depends only on the option itself, like the real per-option estimator
    p = np.asarray(b["spot"]) * 0.01 + np.asarray(b["paths"]) * 1e-6 + np.asarray(b["seed"], np.float64) * 1e-9
    return p, p * 1e-3


def test_partition_covers_in_order_and_balances():
    b = workloads.mixed(4096, seed=3)
    cost = option_cost(b)
    for world in (1, 2, 3, 4, 8):
        ranges = partition_by_cost(cost, world)
        assert len(ranges) == world
        assert ranges[0][0] == 0 and ranges[-1][1] == 4096
        for (b0, e0), (b1, _) in zip(ranges, ranges[1:]):
            assert e0 == b1 and b0 <= e0
        loads = np.array([cost[b0:e0].sum() for b0, e0 in ranges])
        # contiguous ranges: each rank within one option's cost of the ideal share
        assert loads.max() - cost.sum() / world <= cost.max() + 1
    assert partition_by_cost([], 4) == [(0, 0)] * 4
    one = partition_by_cost([5.0], 3)
    assert sum(e - b for b, e in one) == 1 and one[0][0] == 0 and one[-1][1] == 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = workloads.mixed(257, seed=8)
        p, se = price_sharded(b, _fake_pricer)
        out_q.put((rank, p, se))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_price_sharded_gloo_world2_equals_unsharded():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=90) for _ in range(2)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    b = workloads.mixed(257, seed=8)
    want_p, want_se = _fake_pricer(b)
    for _, p, se in results:
        np.testing.assert_array_equal(p, want_p)
        np.testing.assert_array_equal(se, want_se)
