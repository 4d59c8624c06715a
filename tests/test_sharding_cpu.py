"""Host side of one batch priced across several GPUs, on CPU.

* The partition rule (qk_dist_partition, the one the sharded execute applies
  to a plan's tiles) against a numpy statement of the same rule: contiguous
  ranges, cut at the item boundary whose cumulative cost is nearest r/world of
  the total.
* Two ranks as gloo processes (world size 2): each takes its range from the
  library's partition, prices it with a deterministic stand-in computed from
  each item alone (as the GPU's per-tile sums depend only on their tile), and
  the ranks exchange their ranges; every rank must end with the unsharded
  answer.  The exchange here is the test's own (gloo); the library's is NCCL.
* Without a GPU the communicator calls fail loudly (no CPU fallback), and
  without NCCL they say so.
"""

import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from quantkernel_b200 import QKRuntimeError, workloads
from quantkernel_b200.sharding import DistContext, new_id, partition


def _rule(cost, world):
    """Nearest-boundary partition, restated in numpy."""
    cost = np.asarray(cost, np.float64)
    n = cost.size
    if world <= 1 or n == 0:
        return np.array([0] + [n] * world)
    before = np.concatenate([[0.0], np.cumsum(cost)])  # before[i] = cost of items [0, i)
    total = before[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        # the first item whose inclusive cumulative cost reaches the target
        i = int(np.searchsorted(before[1:], target, side="left"))
        if i >= n:
            bounds.append(n)
            continue
        cut = i if target - before[i] <= before[i + 1] - target else i + 1
        bounds.append(max(cut, bounds[-1]))
    bounds.append(n)
    return np.array(bounds)


def _option_cost(b):
    return b["paths"].astype(np.float64) * np.maximum(b["steps"], 1)


def test_partition_is_the_stated_rule_and_balances():
    rng = np.random.default_rng(4)
    cases = [_option_cost(workloads.mixed(4096, seed=3)), rng.uniform(0, 1, 1000),
             rng.integers(0, 5, 333).astype(float), np.ones(7), np.array([1, 2, 3, 4, 5, 6.0])]
    for cost in cases:
        for world in (1, 2, 3, 4, 7, 8):
            b = partition(cost, world)
            np.testing.assert_array_equal(b, _rule(cost, world))
            assert b[0] == 0 and b[-1] == cost.size and np.all(np.diff(b) >= 0)
            loads = np.array([cost[b[k]:b[k + 1]].sum() for k in range(world)])
            # contiguous ranges: every rank within one item's cost of its share
            assert np.abs(loads - cost.sum() / world).max() <= cost.max() + 1e-9
    np.testing.assert_array_equal(partition([1, 2, 3, 4, 5, 6], 3), [0, 3, 5, 6])
    np.testing.assert_array_equal(partition([], 4), [0, 0, 0, 0, 0])
    np.testing.assert_array_equal(partition([5.0], 3), [0, 0, 1, 1])


def _fake_pricer(b):
    # depends only on the option itself, like the real per-tile sums
    p = np.asarray(b["spot"]) * 0.01 + np.asarray(b["paths"]) * 1e-6 + np.asarray(b["seed"], np.float64) * 1e-9
    return p, p * 1e-3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_q):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = workloads.mixed(257, seed=8)
        bounds = partition(_option_cost(b), world)
        lo, hi = int(bounds[rank]), int(bounds[rank + 1])
        p, se = _fake_pricer({k: v[lo:hi] for k, v in b.items()})
        # every rank's range to every rank (padded to the widest range)
        width = max(1, int(np.diff(bounds).max()))
        buf = np.full((2, width), np.nan)
        buf[0, :hi - lo], buf[1, :hi - lo] = p, se
        parts = [torch.empty(2, width, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(parts, torch.from_numpy(buf))
        prices, stderr = np.empty(len(b["spot"])), np.empty(len(b["spot"]))
        for k in range(world):
            a, e = int(bounds[k]), int(bounds[k + 1])
            prices[a:e] = parts[k][0, :e - a].numpy()
            stderr[a:e] = parts[k][1, :e - a].numpy()
        out_q.put((rank, bounds, prices, stderr))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_assemble_the_unsharded_answer():
    import torch.multiprocessing as mp

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
    assert np.array_equal(results[0][1], results[1][1]), "ranks disagree on the partition"
    for _, _, p, se in results:
        np.testing.assert_array_equal(p, want_p)
        np.testing.assert_array_equal(se, want_se)


def _gpu_present():
    try:
        import torch

        return torch.cuda.is_available()
    except ImportError:
        return False


def test_communicator_without_gpu_is_an_error_not_a_fallback():
    if _gpu_present():
        pytest.skip("a GPU is present")
    ident = new_id()  # NCCL makes ids without a GPU
    assert isinstance(ident, bytes) and len(ident) == 128
    with pytest.raises(QKRuntimeError, match="cuda error"):
        DistContext(ident, 1, 0)


def test_missing_nccl_is_reported():
    code = ("import sys; sys.path.insert(0, {pkg!r})\n"
            "from quantkernel_b200 import QKRuntimeError\n"
            "from quantkernel_b200.sharding import new_id\n"
            "try:\n    new_id()\nexcept QKRuntimeError as e:\n    print(e)\n")
    pkg = str(Path(__file__).resolve().parents[1] / "quant-kernel_b200")
    env = dict(os.environ, QK_B200_NCCL_PATH="/nonexistent/libnccl.so.2")
    r = subprocess.run([sys.executable, "-c", code.format(pkg=pkg)], env=env, capture_output=True,
                       text=True, timeout=120)
    assert "nccl unavailable" in r.stdout, (r.stdout, r.stderr)
