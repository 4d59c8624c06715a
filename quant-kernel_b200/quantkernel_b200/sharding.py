"""One batch priced across several GPUs, one rank (process or thread) per GPU.

Thin wrapper over the library's C ABI (qk_dist_*, qk_mcm_*_sharded in
include/qk_api.h); no framework is needed.  Every rank builds the same plan
from the same inputs; a sharded execute simulates this rank's contiguous range
of the plan's tiles (balanced by path-steps), exchanges every rank's tile sums
over NCCL in one grouped step, and finalizes every option on every rank.  A
path's random stream depends only on its option's seed and path index and the
merge order is fixed, so each rank ends up with exactly the single-GPU
results.

The communicator id (QK_DIST_ID_BYTES bytes) is made once, by one rank, with
`new_id()` and handed to the others by any channel the job already has (a
shared file, a socket, the launcher's key-value store).
"""

import ctypes as ct

import numpy as np

from ._abi import QK_DIST_ID_BYTES, QK_OK
from .engine import McPlan, QuantKernel


def new_id(qk: QuantKernel = None) -> bytes:
    """A fresh communicator id; call on one rank only."""
    qk = qk or QuantKernel()
    buf = (ct.c_uint8 * QK_DIST_ID_BYTES)()
    rc = qk._lib.qk_dist_unique_id(buf)
    if rc != QK_OK:
        qk._raise_rc("qk_dist_unique_id", rc)
    return bytes(buf)


def partition(cost, world: int) -> np.ndarray:
    """The sharded execute's partition rule on a list of costs: `world` + 1
    bounds of contiguous ranges with near-equal total cost (host only)."""
    qk = QuantKernel()
    c = np.ascontiguousarray(cost, np.float64)
    bounds = np.empty(int(world) + 1, np.int64)
    rc = qk._lib.qk_dist_partition(c.ctypes.data_as(ct.POINTER(ct.c_double)), int(c.size),
                                   int(world), bounds.ctypes.data_as(ct.POINTER(ct.c_int64)))
    if rc != QK_OK:
        qk._raise_rc("qk_dist_partition", rc)
    return bounds


class DistContext:
    """Rank `rank` of `world`, on the calling thread's current device (set it
    first with QuantKernel.set_device)."""

    def __init__(self, unique_id: bytes, world: int, rank: int, qk: QuantKernel = None):
        if len(unique_id) != QK_DIST_ID_BYTES:
            raise ValueError(f"communicator id must be {QK_DIST_ID_BYTES} bytes")
        self.qk = qk or QuantKernel()
        self._lib = self.qk._lib
        self._h = ct.c_void_p()
        buf = (ct.c_uint8 * QK_DIST_ID_BYTES).from_buffer_copy(unique_id)
        rc = self._lib.qk_dist_create(buf, int(world), int(rank), ct.byref(self._h))
        if rc != QK_OK:
            self.qk._raise_rc("qk_dist_create", rc)
        self.world, self.rank = int(world), int(rank)

    def execute(self, plan: McPlan, stream: int = 0) -> None:
        """This rank's share of `plan`; then plan.results() holds every option."""
        rc = self._lib.qk_mcm_plan_execute_sharded(plan._h, self._h,
                                                   ct.c_void_p(stream) if stream else None)
        if rc != QK_OK:
            self.qk._raise_rc("qk_mcm_plan_execute_sharded", rc)

    def mixed_price_batch(self, model, spot, strike, t, vol=None, r=None, q=None, v0=None,
                          kappa=None, theta=None, sigma=None, rho=None, option_type=None,
                          paths=None, steps=None, seed=None):
        """QuantKernel.mixed_price_batch across the ranks: every rank passes the
        whole batch and gets (prices, standard errors) of every option."""
        arrays = self.qk._mixed_arrays(model, spot, strike, t, vol, r, q, v0, kappa, theta,
                                       sigma, rho, option_type, paths, steps, seed)
        n = int(arrays[0].shape[0])
        out = np.empty(n)
        se = np.empty(n)
        from .engine import _ptr

        rc = self._lib.qk_mcm_mixed_price_batch_sharded(
            self._h, *[_ptr(a) for a in arrays], n, out.ctypes.data_as(ct.POINTER(ct.c_double)),
            se.ctypes.data_as(ct.POINTER(ct.c_double)))
        if rc != QK_OK:
            self.qk._raise_rc("qk_mcm_mixed_price_batch_sharded", rc)
        return out, se

    def abort(self) -> None:
        if self._h:
            self._lib.qk_dist_abort(self._h)

    def close(self) -> None:
        if self._h:
            self._lib.qk_dist_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
