"""Batch routing of the Monte Carlo pricers onto the GPU library.

Mirrors yluoc/Quant-Kernel python/quantkernel/accelerator.py:313-347
(``QuantAccelerator``: ``suggest_strategy``, ``price_batch``, jobs given as a
sequence of keyword dicts, one per scalar call) for the methods this library
implements.  Where the reference routes ``backend="gpu"`` Monte Carlo methods
through CuPy -- materialising every path as a (batch x paths [x steps]) array
with NumPy-seeded normals (accelerator.py:1009-1191), and with no Heston path
at all -- every method here is one call of the library's batch entry, which
simulates in registers on the GPU.  ``price_many`` goes further: jobs of
different Monte Carlo methods share one persistent work-stealing launch.

There is no CPU strategy: ``backend="cpu"`` is refused and a missing GPU
raises from the library (QKRuntimeError), never a silent CPU result.
"""

from __future__ import annotations

import inspect
from typing import Any, Mapping, Sequence

import numpy as np

from ._abi import (QK_MC_ANTITHETIC, QK_MC_CONTROL_VARIATES, QK_MC_EULER, QK_MC_HESTON,
                   QK_MC_HESTON_LR_DELTA, QK_MC_IMPORTANCE_SAMPLING, QK_MC_LOCAL_VOL,
                   QK_MC_MILSTEIN, QK_MC_QMC_HALTON, QK_MC_QMC_SOBOL, QK_MC_STANDARD,
                   QK_MC_STRATIFIED)
from .engine import QuantKernel


class QuantAccelerator:
    """GPU batch pricing with the reference accelerator's interface.

    Parameters
    ----------
    qk:
        Existing ``QuantKernel`` instance.  If omitted, one is created.
    backend:
        ``"auto"`` (default) or ``"gpu"``; both run on the GPU.  ``"cpu"`` is
        refused: this library has no CPU path.
    max_workers:
        Accepted for interface compatibility; unused (no thread pool).
    """

    # scalar method -> batch method, as accelerator.py:226-283 maps them
    _NATIVE_BATCH_METHODS = {
        "standard_monte_carlo_price": "standard_monte_carlo_price_batch",
        "antithetic_variates_price": "antithetic_variates_price_batch",
        "euler_maruyama_price": "euler_maruyama_price_batch",
        "milstein_price": "milstein_price_batch",
        "local_vol_monte_carlo_price": "local_vol_monte_carlo_price_batch",
        "heston_monte_carlo_price": "heston_monte_carlo_price_batch",
        "heston_lr_delta": "heston_lr_delta_batch",
        "importance_sampling_price": "importance_sampling_price_batch",
        "control_variates_price": "control_variates_price_batch",
        "stratified_sampling_price": "stratified_sampling_price_batch",
        "quasi_monte_carlo_sobol_price": "quasi_monte_carlo_sobol_price_batch",
        "quasi_monte_carlo_halton_price": "quasi_monte_carlo_halton_price_batch",
        "heston_price_cf": "heston_price_cf_batch",
        "cos_method_fang_oosterlee_heston_price": "cos_method_fang_oosterlee_heston_price_batch",
    }

    # Monte Carlo methods that the mixed-model launch can price together
    _MIXED_MODELS = {
        "standard_monte_carlo_price": QK_MC_STANDARD,
        "antithetic_variates_price": QK_MC_ANTITHETIC,
        "euler_maruyama_price": QK_MC_EULER,
        "milstein_price": QK_MC_MILSTEIN,
        "local_vol_monte_carlo_price": QK_MC_LOCAL_VOL,
        "heston_monte_carlo_price": QK_MC_HESTON,
        "heston_lr_delta": QK_MC_HESTON_LR_DELTA,
        "control_variates_price": QK_MC_CONTROL_VARIATES,
        "importance_sampling_price": QK_MC_IMPORTANCE_SAMPLING,
        "stratified_sampling_price": QK_MC_STRATIFIED,
        "quasi_monte_carlo_sobol_price": QK_MC_QMC_SOBOL,
        "quasi_monte_carlo_halton_price": QK_MC_QMC_HALTON,
    }

    def __init__(self, qk: QuantKernel | None = None, backend: str = "auto",
                 max_workers: int | None = None):
        if backend not in {"auto", "cpu", "gpu"}:
            raise ValueError("backend must be one of: auto, cpu, gpu")
        if backend == "cpu":
            raise RuntimeError("backend='cpu' is not available: quantkernel_b200 prices on the "
                               "GPU only (use the reference package for CPU pricing)")
        self.qk = qk if qk is not None else QuantKernel()
        self.backend = backend
        self.max_workers = max_workers
        self._defaults: dict[str, dict[str, Any]] = {}

    @property
    def gpu_available(self) -> bool:
        """True when the library can reach a CUDA device."""
        import ctypes as ct

        dev = ct.c_int32(-1)
        return self.qk._lib.qk_get_device(ct.byref(dev)) == 0 and dev.value >= 0

    def suggest_strategy(self, method: str, batch_size: int) -> str:
        """``"native_batch"`` for every supported method (the batch entry runs
        on the GPU); a RuntimeError for any other method, as the reference's
        ``backend="gpu"`` does for methods it cannot vectorise."""
        if method in self._NATIVE_BATCH_METHODS:
            return "native_batch"
        raise RuntimeError(f"backend='{self.backend}' not supported for method '{method}' "
                           f"(quantkernel_b200 implements the Monte Carlo path and the Heston "
                           f"characteristic-function and COS pricers)")

    def _scalar_defaults(self, method: str) -> dict[str, Any]:
        d = self._defaults.get(method)
        if d is None:
            sig = inspect.signature(getattr(self.qk, method))
            d = {k: p.default for k, p in sig.parameters.items()
                 if p.default is not inspect.Parameter.empty}
            self._defaults[method] = d
        return d

    def _columns(self, method: str, jobs: Sequence[Mapping[str, Any]]) -> dict[str, list]:
        """Job dicts -> argument columns, missing keys taken from the scalar
        method's defaults (e.g. ``seed=42``, ``integration_steps=1024``)."""
        defaults = self._scalar_defaults(method)
        keys = list(jobs[0].keys())
        for k in defaults:
            if k not in keys:
                keys.append(k)
        cols = {}
        for k in keys:
            cols[k] = [job[k] if k in job else defaults[k] for job in jobs]
        return cols

    def price_batch(self, method: str, jobs: Sequence[Mapping[str, Any]]) -> np.ndarray:
        """Price a batch of jobs for one method (accelerator.py:313-347)."""
        if not hasattr(self.qk, method):
            raise AttributeError(f"Unknown method: {method}")
        n = len(jobs)
        if n == 0:
            return np.empty((0,), dtype=np.float64)
        self.suggest_strategy(method, n)
        batch_fn = getattr(self.qk, self._NATIVE_BATCH_METHODS[method])
        return np.asarray(batch_fn(**self._columns(method, jobs)), dtype=np.float64)

    def price_many(self, requests: Sequence[tuple[str, Mapping[str, Any]]],
                   with_stderr: bool = False):
        """Price ``(method, job)`` pairs of different methods in one go.

        All Monte Carlo jobs go into one mixed-model batch -- one persistent
        work-stealing launch over every option's tiles, so a few long Heston
        jobs and many short terminal ones finish together; the Heston Fourier
        jobs go into one batch call per method.  Results come
        back in request order; with ``with_stderr`` a second array holds the
        Monte Carlo standard errors (NaN for closed-form jobs).
        """
        n = len(requests)
        prices = np.full(n, np.nan)
        stderr = np.full(n, np.nan)
        if n == 0:
            return (prices, stderr) if with_stderr else prices
        mc_idx: list[int] = []
        fourier_idx: dict[str, list[int]] = {}
        for i, (method, _) in enumerate(requests):
            if not hasattr(self.qk, method):
                raise AttributeError(f"Unknown method: {method}")
            self.suggest_strategy(method, 1)
            if method in self._MIXED_MODELS:
                mc_idx.append(i)
            else:
                fourier_idx.setdefault(method, []).append(i)
        for method, idx in fourier_idx.items():
            prices[idx] = self.price_batch(method, [requests[i][1] for i in idx])
        if mc_idx:
            m = len(mc_idx)
            cols = {k: np.zeros(m) for k in ("spot", "strike", "t", "vol", "r", "q", "v0",
                                             "kappa", "theta", "sigma", "rho")}
            model = np.empty(m, np.int32)
            option_type = np.zeros(m, np.int32)
            paths = np.zeros(m, np.int32)
            steps = np.ones(m, np.int32)
            seed = np.zeros(m, np.uint64)
            for j, i in enumerate(mc_idx):
                method, job = requests[i]
                job = {**self._scalar_defaults(method), **job}
                model[j] = self._MIXED_MODELS[method]
                for k in ("spot", "strike", "t", "r", "q"):
                    cols[k][j] = job[k]
                option_type[j] = job["option_type"]
                paths[j] = job["paths"]
                steps[j] = job.get("steps", 1)
                seed[j] = job.get("seed", 0)
                if "vol" in job:
                    cols["vol"][j] = job["vol"]
                for k in ("v0", "kappa", "theta", "sigma", "rho"):
                    if k in job:
                        cols[k][j] = job[k]
                if method == "heston_lr_delta":
                    cols["vol"][j] = job["weight_clip"]  # the mixed call's clip column
                if method == "importance_sampling_price":
                    cols["v0"][j] = job["shift"]  # the mixed call's shift column
            p, se = self.qk.mixed_price_batch(model=model, option_type=option_type, paths=paths,
                                              steps=steps, seed=seed, **cols)
            prices[mc_idx] = p
            stderr[mc_idx] = se
        return (prices, stderr) if with_stderr else prices
