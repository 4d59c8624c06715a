"""Pricing one batch across several GPUs, one process per GPU.

Options are independent, so a batch shards by option with no exchange during
pricing: each rank prices a contiguous range whose Monte Carlo cost
(paths x steps) is about 1/world of the total, then one all-gather of
(price, standard error) puts every result on every rank in the original
option order.  Each rank's results are computed exactly as a single-GPU call
would compute them (a path's random stream depends only on its option's seed
and path index), so the sharded answer equals the unsharded one bit for bit.
"""

import numpy as np


def option_cost(batch) -> np.ndarray:
    """Relative Monte Carlo cost of each option: paths x max(steps, 1)."""
    p = np.asarray(batch["paths"], np.int64)
    s = batch.get("steps")
    s = np.ones_like(p) if s is None else np.maximum(np.asarray(s, np.int64), 1)
    return np.maximum(p, 0) * s


def partition_by_cost(cost, world: int):
    """Contiguous [begin, end) ranges, one per rank, with near-equal total cost.

    Boundary r is the first option whose cumulative cost reaches r/world of
    the total; every rank gets a (possibly empty) range and the ranges cover
    0..n exactly once in order."""
    cost = np.asarray(cost, np.float64)
    n = cost.size
    if world <= 1 or n == 0:
        return [(0, n)] + [(n, n)] * max(world - 1, 0)
    cum = np.cumsum(cost)
    total = cum[-1] if cum.size else 0.0
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left"))
        bounds.append(min(max(b, bounds[-1]), n))
    bounds.append(n)
    return [(bounds[i], bounds[i + 1]) for i in range(world)]


def price_sharded(batch, pricer, group=None, device=None):
    """Price `batch` (dict of equal-length arrays) across the ranks of `group`.

    `pricer(sub_batch) -> (prices, stderr)` runs on this rank's range (for a
    GPU library: ``lambda b: qk.mixed_price_batch(**b)``).  Returns the full
    (prices, stderr) on every rank.  Uses torch.distributed: NCCL for CUDA
    tensors (pass `device`), gloo on CPU."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = len(next(iter(batch.values())))
    ranges = partition_by_cost(option_cost(batch), world)
    b0, b1 = ranges[rank]
    sub = {k: np.asarray(v)[b0:b1] for k, v in batch.items()}
    if b1 > b0:
        p, se = pricer(sub)
    else:
        p, se = np.empty(0), np.empty(0)
    width = max(e - b for b, e in ranges)
    buf = np.full((2, max(width, 1)), np.nan)
    buf[0, : b1 - b0] = p
    buf[1, : b1 - b0] = se
    t = torch.from_numpy(buf)
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    prices = np.empty(n)
    stderr = np.empty(n)
    for r, (b, e) in enumerate(ranges):
        arr = parts[r].cpu().numpy()
        prices[b:e] = arr[0, : e - b]
        stderr[b:e] = arr[1, : e - b]
    return prices, stderr
