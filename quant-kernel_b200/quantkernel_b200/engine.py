"""QuantKernel (B200) -- Python API of the GPU batch Monte Carlo pricing path.

Mirrors the Monte Carlo methods of yluoc/Quant-Kernel python/quantkernel/engine.py:
the same method names, argument names and order, array coercion
(``_as_f64_array`` & co., engine.py:100-125), length checks, and return-code to
exception mapping (engine.py:37-41, 163-193).  Scalar methods raise
``ValueError`` when the library returns NaN, as ``_call_checked`` does
(engine.py:93-97).  Every call runs on the GPU through libqk_b200.so; there is
no CPU path.

Additions (ABI 2.13): ``*_price_se_batch`` (price and standard error),
``mixed_price_batch`` and ``McPlan`` (device-resident batches).
"""

import ctypes as ct
import math

import numpy as np

from ._abi import (
    ABI_MAJOR,
    ABI_MINOR,
    QK_CALL,
    QK_ERR_BAD_SIZE,
    QK_ERR_INVALID_INPUT,
    QK_ERR_NULL_PTR,
    QK_ERR_RUNTIME_INIT,
    QK_OK,
    QK_PUT,
)
from ._loader import QKPluginAPI, load_library


class QKError(RuntimeError):
    """Base exception for QuantKernel errors."""


class QKNullPointerError(QKError):
    """Raised when a null pointer is passed to a batch API."""


class QKBadSizeError(QKError):
    """Raised when an invalid batch size is passed."""


class QKInvalidInputError(QKError):
    """Raised when invalid input parameters are detected."""


class QKRuntimeError(QKError):
    """Raised when the GPU runtime fails (no device, launch or copy error)."""


_ERROR_CODE_MAP = {
    QK_ERR_NULL_PTR: QKNullPointerError,
    QK_ERR_BAD_SIZE: QKBadSizeError,
    QK_ERR_INVALID_INPUT: QKInvalidInputError,
    QK_ERR_RUNTIME_INIT: QKRuntimeError,
}

_PD = ct.POINTER(ct.c_double)
_PI32 = ct.POINTER(ct.c_int32)
_PU64 = ct.POINTER(ct.c_uint64)


def _ptr(arr):
    if arr is None:
        return None
    if arr.dtype == np.float64:
        return arr.ctypes.data_as(_PD)
    if arr.dtype == np.int32:
        return arr.ctypes.data_as(_PI32)
    if arr.dtype == np.uint64:
        return arr.ctypes.data_as(_PU64)
    raise TypeError(f"Unsupported dtype for batch call: {arr.dtype}")


class QuantKernel:
    """GPU batch Monte Carlo option pricing (B200).

    Example::

        qk = QuantKernel()
        prices = qk.heston_monte_carlo_price_batch(
            spot=[100.0] * 1024, strike=..., t=..., r=..., q=..., v0=..., kappa=...,
            theta=..., sigma=..., rho=..., option_type=[qk.CALL] * 1024,
            paths=[262144] * 1024, steps=[200] * 1024, seed=np.arange(1024))
    """

    __slots__ = ("_lib", "_fn_cache")

    CALL = QK_CALL
    PUT = QK_PUT

    def __init__(self):
        self._lib = load_library()
        self._fn_cache = {}

    # ------------------------------------------------------------------ plumbing
    def _get_fn(self, fn_name: str):
        fn = self._fn_cache.get(fn_name)
        if fn is None:
            fn = getattr(self._lib, fn_name)
            self._fn_cache[fn_name] = fn
        return fn

    def _call_checked(self, fn_name: str, *args) -> float:
        out = self._get_fn(fn_name)(*args)
        if math.isnan(out):
            detail = self.get_last_error()
            msg = f"{fn_name} returned NaN; check inputs."
            if detail:
                msg += f" ({detail})"
            raise ValueError(msg)
        return out

    @staticmethod
    def _as_f64_array(x, name: str) -> np.ndarray:
        arr = np.asarray(x, dtype=np.float64)
        if arr.ndim != 1:
            raise ValueError(f"{name} must be a 1D array-like")
        return np.ascontiguousarray(arr)

    @staticmethod
    def _as_i32_array(x, name: str) -> np.ndarray:
        arr = np.asarray(x, dtype=np.int32)
        if arr.ndim != 1:
            raise ValueError(f"{name} must be a 1D array-like")
        return np.ascontiguousarray(arr)

    @staticmethod
    def _as_u64_array(x, name: str) -> np.ndarray:
        arr = np.asarray(x, dtype=np.uint64)
        if arr.ndim != 1:
            raise ValueError(f"{name} must be a 1D array-like")
        return np.ascontiguousarray(arr)

    @staticmethod
    def _check_same_length(n: int, **arrays) -> None:
        for name, arr in arrays.items():
            if arr.shape[0] != n:
                raise ValueError(f"{name} length mismatch: expected {n}, got {arr.shape[0]}")

    def _raise_rc(self, fn_name: str, rc: int) -> None:
        detail = self.get_last_error()
        exc_cls = _ERROR_CODE_MAP.get(rc, QKError)
        msg = f"{fn_name} failed (rc={rc})"
        if detail:
            msg += f": {detail}"
        raise exc_cls(msg)

    def _call_batch_ctypes(self, fn_name: str, *arrays, with_se: bool = False):
        n = arrays[0].shape[0]
        out = np.empty(n, dtype=np.float64)
        se = np.empty(n, dtype=np.float64) if with_se else None
        args = [_ptr(a) for a in arrays] + [int(n), out.ctypes.data_as(_PD)]
        if with_se:
            args.append(se.ctypes.data_as(_PD))
        rc = self._get_fn(fn_name)(*args)
        if rc != QK_OK:
            self._raise_rc(fn_name, rc)
        return (out, se) if with_se else out

    # ------------------------------------------------------------------ ABI
    def abi_version(self) -> tuple[int, int]:
        major = ct.c_int32(-1)
        minor = ct.c_int32(-1)
        self._get_fn("qk_abi_version")(ct.byref(major), ct.byref(minor))
        return int(major.value), int(minor.value)

    def plugin_get_api(self, host_abi_major: int = ABI_MAJOR, host_abi_minor: int = ABI_MINOR):
        out_api = ct.POINTER(QKPluginAPI)()
        rc = self._get_fn("qk_plugin_get_api")(int(host_abi_major), int(host_abi_minor), ct.byref(out_api))
        if rc != QK_OK:
            raise QKError(f"qk_plugin_get_api failed (rc={rc}, host_abi={host_abi_major}.{host_abi_minor})")
        if not out_api:
            raise QKError("qk_plugin_get_api returned null API pointer")
        info = out_api.contents
        name = info.plugin_name.decode("utf-8", errors="replace") if info.plugin_name else ""
        return int(info.abi_major), int(info.abi_minor), name

    def get_last_error(self) -> str:
        raw = self._get_fn("qk_get_last_error")()
        return raw.decode("utf-8", errors="replace") if raw else ""

    def clear_last_error(self) -> None:
        self._get_fn("qk_clear_last_error")()

    def set_device(self, device: int) -> None:
        """Run this thread's later calls on CUDA device `device`."""
        rc = self._get_fn("qk_set_device")(int(device))
        if rc != QK_OK:
            self._raise_rc("qk_set_device", rc)

    def get_device(self) -> int:
        d = ct.c_int32(-1)
        rc = self._get_fn("qk_get_device")(ct.byref(d))
        if rc != QK_OK:
            self._raise_rc("qk_get_device", rc)
        return int(d.value)

    # ------------------------------------------------------------------ terminal
    def _term_arrays(self, spot, strike, t, vol, r, q, option_type, paths, seed):
        s = self._as_f64_array(spot, "spot")
        k = self._as_f64_array(strike, "strike")
        tau = self._as_f64_array(t, "t")
        sig = self._as_f64_array(vol, "vol")
        rr = self._as_f64_array(r, "r")
        qq = self._as_f64_array(q, "q")
        ot = self._as_i32_array(option_type, "option_type")
        pp = self._as_i32_array(paths, "paths")
        sd = self._as_u64_array(seed, "seed")
        self._check_same_length(s.shape[0], strike=k, t=tau, vol=sig, r=rr, q=qq,
                                option_type=ot, paths=pp, seed=sd)
        return s, k, tau, sig, rr, qq, ot, pp, sd

    def _step_arrays(self, spot, strike, t, vol, r, q, option_type, paths, steps, seed):
        s, k, tau, sig, rr, qq, ot, pp, sd = self._term_arrays(spot, strike, t, vol, r, q,
                                                               option_type, paths, seed)
        st = self._as_i32_array(steps, "steps")
        self._check_same_length(s.shape[0], steps=st)
        return s, k, tau, sig, rr, qq, ot, pp, st, sd

    def standard_monte_carlo_price(self, spot: float, strike: float, t: float, vol: float,
                                   r: float, q: float, option_type: int, paths: int,
                                   seed: int = 42) -> float:
        """Terminal GBM Monte Carlo with antithetic pairs (standard_monte_carlo.cpp:11-33)."""
        return self._call_checked("qk_mcm_standard_monte_carlo_price",
                                  spot, strike, t, vol, r, q, option_type, paths, seed)

    def standard_monte_carlo_price_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                         seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_standard_monte_carlo_price_batch",
                                       *self._term_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, seed))

    def standard_monte_carlo_price_se_batch(self, spot, strike, t, vol, r, q, option_type,
                                            paths, seed):
        return self._call_batch_ctypes("qk_mcm_standard_monte_carlo_price_se_batch",
                                       *self._term_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, seed),
                                       with_se=True)

    def antithetic_variates_price(self, spot: float, strike: float, t: float, vol: float,
                                  r: float, q: float, option_type: int, paths: int,
                                  seed: int = 42) -> float:
        """Terminal GBM with antithetic variates (antithetic_variates.cpp:11-29)."""
        return self._call_checked("qk_mcm_antithetic_variates_price",
                                  spot, strike, t, vol, r, q, option_type, paths, seed)

    def antithetic_variates_price_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                        seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_antithetic_variates_price_batch",
                                       *self._term_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, seed))

    def antithetic_variates_price_se_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                           seed):
        return self._call_batch_ctypes("qk_mcm_antithetic_variates_price_se_batch",
                                       *self._term_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, seed),
                                       with_se=True)

    # ------------------------------------------------------------------ stepwise
    def euler_maruyama_price(self, spot: float, strike: float, t: float, vol: float, r: float,
                             q: float, option_type: int, paths: int, steps: int,
                             seed: int = 42) -> float:
        return self._call_checked("qk_mcm_euler_maruyama_price",
                                  spot, strike, t, vol, r, q, option_type, paths, steps, seed)

    def euler_maruyama_price_batch(self, spot, strike, t, vol, r, q, option_type, paths, steps,
                                   seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_euler_maruyama_price_batch",
                                       *self._step_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, steps, seed))

    def euler_maruyama_price_se_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                      steps, seed):
        return self._call_batch_ctypes("qk_mcm_euler_maruyama_price_se_batch",
                                       *self._step_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, steps, seed),
                                       with_se=True)

    def milstein_price(self, spot: float, strike: float, t: float, vol: float, r: float,
                       q: float, option_type: int, paths: int, steps: int,
                       seed: int = 42) -> float:
        return self._call_checked("qk_mcm_milstein_price",
                                  spot, strike, t, vol, r, q, option_type, paths, steps, seed)

    def milstein_price_batch(self, spot, strike, t, vol, r, q, option_type, paths, steps,
                             seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_milstein_price_batch",
                                       *self._step_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, steps, seed))

    def milstein_price_se_batch(self, spot, strike, t, vol, r, q, option_type, paths, steps,
                                seed):
        return self._call_batch_ctypes("qk_mcm_milstein_price_se_batch",
                                       *self._step_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, steps, seed),
                                       with_se=True)

    def local_vol_monte_carlo_price(self, spot: float, strike: float, t: float, vol: float,
                                    r: float, q: float, option_type: int, paths: int,
                                    steps: int, seed: int = 42) -> float:
        """Constant local-vol Euler (local_vol_monte_carlo.cpp:57-73)."""
        return self._call_checked("qk_mcm_local_vol_monte_carlo_price",
                                  spot, strike, t, vol, r, q, option_type, paths, steps, seed)

    def local_vol_monte_carlo_price_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                          steps, seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_local_vol_monte_carlo_price_batch",
                                       *self._step_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, steps, seed))

    def local_vol_monte_carlo_price_se_batch(self, spot, strike, t, vol, r, q, option_type,
                                             paths, steps, seed):
        return self._call_batch_ctypes("qk_mcm_local_vol_monte_carlo_price_se_batch",
                                       *self._step_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, steps, seed),
                                       with_se=True)

    # ------------------------------------------------------------------ Heston
    def _heston_arrays(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                       option_type, paths, steps, seed):
        s = self._as_f64_array(spot, "spot")
        k = self._as_f64_array(strike, "strike")
        tau = self._as_f64_array(t, "t")
        rr = self._as_f64_array(r, "r")
        qq = self._as_f64_array(q, "q")
        v0a = self._as_f64_array(v0, "v0")
        ka = self._as_f64_array(kappa, "kappa")
        th = self._as_f64_array(theta, "theta")
        si = self._as_f64_array(sigma, "sigma")
        rh = self._as_f64_array(rho, "rho")
        ot = self._as_i32_array(option_type, "option_type")
        pp = self._as_i32_array(paths, "paths")
        st = self._as_i32_array(steps, "steps")
        sd = self._as_u64_array(seed, "seed")
        self._check_same_length(s.shape[0], strike=k, t=tau, r=rr, q=qq, v0=v0a, kappa=ka,
                                theta=th, sigma=si, rho=rh, option_type=ot, paths=pp,
                                steps=st, seed=sd)
        return s, k, tau, rr, qq, v0a, ka, th, si, rh, ot, pp, st, sd

    def heston_monte_carlo_price(self, spot: float, strike: float, t: float, r: float, q: float,
                                 v0: float, kappa: float, theta: float, sigma: float,
                                 rho: float, option_type: int, paths: int, steps: int,
                                 seed: int = 42) -> float:
        """Heston full-truncation Euler Monte Carlo (heston_monte_carlo.cpp:11-36)."""
        return self._call_checked("qk_mcm_heston_monte_carlo_price",
                                  spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                  option_type, paths, steps, seed)

    def heston_monte_carlo_price_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma,
                                       rho, option_type, paths, steps, seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_heston_monte_carlo_price_batch",
                                       *self._heston_arrays(spot, strike, t, r, q, v0, kappa,
                                                            theta, sigma, rho, option_type,
                                                            paths, steps, seed))

    def heston_monte_carlo_price_se_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma,
                                          rho, option_type, paths, steps, seed):
        return self._call_batch_ctypes("qk_mcm_heston_monte_carlo_price_se_batch",
                                       *self._heston_arrays(spot, strike, t, r, q, v0, kappa,
                                                            theta, sigma, rho, option_type,
                                                            paths, steps, seed),
                                       with_se=True)

    def heston_lr_delta(self, spot: float, strike: float, t: float, r: float, q: float,
                        v0: float, kappa: float, theta: float, sigma: float, rho: float,
                        option_type: int, paths: int, steps: int, seed: int = 42,
                        weight_clip: float = 6.0) -> float:
        """Likelihood-ratio delta under Heston (heston_lr_delta.cpp:37-132)."""
        return self._call_checked("qk_mcm_heston_lr_delta", spot, strike, t, r, q, v0, kappa,
                                  theta, sigma, rho, option_type, paths, steps, seed, weight_clip)

    def _lr_arrays(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type, paths,
                   steps, seed, weight_clip):
        arrs = self._heston_arrays(spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                   option_type, paths, steps, seed)
        wc = self._as_f64_array(weight_clip, "weight_clip")
        self._check_same_length(arrs[0].shape[0], weight_clip=wc)
        return (*arrs, wc)

    def heston_lr_delta_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                              option_type, paths, steps, seed, weight_clip) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_heston_lr_delta_batch",
                                       *self._lr_arrays(spot, strike, t, r, q, v0, kappa, theta,
                                                        sigma, rho, option_type, paths, steps,
                                                        seed, weight_clip))

    def heston_lr_delta_se_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                 option_type, paths, steps, seed, weight_clip):
        return self._call_batch_ctypes("qk_mcm_heston_lr_delta_se_batch",
                                       *self._lr_arrays(spot, strike, t, r, q, v0, kappa, theta,
                                                        sigma, rho, option_type, paths, steps,
                                                        seed, weight_clip), with_se=True)

    # ------------------------------------------------------------------ variance reduction
    def control_variates_price(self, spot: float, strike: float, t: float, vol: float,
                               r: float, q: float, option_type: int, paths: int,
                               seed: int = 42) -> float:
        """Terminal GBM with S_T as control variate (control_variates.cpp:10-52)."""
        return self._call_checked("qk_mcm_control_variates_price",
                                  spot, strike, t, vol, r, q, option_type, paths, seed)

    def control_variates_price_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                     seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_control_variates_price_batch",
                                       *self._term_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, seed))

    def control_variates_price_se_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                        seed):
        return self._call_batch_ctypes("qk_mcm_control_variates_price_se_batch",
                                       *self._term_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, seed),
                                       with_se=True)

    def stratified_sampling_price(self, spot: float, strike: float, t: float, vol: float,
                                  r: float, q: float, option_type: int, paths: int,
                                  seed: int = 42) -> float:
        """One draw per stratum of [0, 1) (stratified_sampling.cpp:11-35)."""
        return self._call_checked("qk_mcm_stratified_sampling_price",
                                  spot, strike, t, vol, r, q, option_type, paths, seed)

    def stratified_sampling_price_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                        seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_stratified_sampling_price_batch",
                                       *self._term_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, seed))

    def stratified_sampling_price_se_batch(self, spot, strike, t, vol, r, q, option_type,
                                           paths, seed):
        return self._call_batch_ctypes("qk_mcm_stratified_sampling_price_se_batch",
                                       *self._term_arrays(spot, strike, t, vol, r, q,
                                                          option_type, paths, seed),
                                       with_se=True)

    def _is_arrays(self, spot, strike, t, vol, r, q, option_type, paths, shift, seed):
        s, k, tau, sig, rr, qq, ot, pp, sd = self._term_arrays(spot, strike, t, vol, r, q,
                                                               option_type, paths, seed)
        sh = self._as_f64_array(shift, "shift")
        self._check_same_length(s.shape[0], shift=sh)
        return s, k, tau, sig, rr, qq, ot, pp, sh, sd

    def importance_sampling_price(self, spot: float, strike: float, t: float, vol: float,
                                  r: float, q: float, option_type: int, paths: int,
                                  shift: float, seed: int = 42) -> float:
        """Normal shifted by `shift` with likelihood-ratio weights
        (importance_sampling.cpp:11-36)."""
        return self._call_checked("qk_mcm_importance_sampling_price",
                                  spot, strike, t, vol, r, q, option_type, paths, shift, seed)

    def importance_sampling_price_batch(self, spot, strike, t, vol, r, q, option_type, paths,
                                        shift, seed) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_importance_sampling_price_batch",
                                       *self._is_arrays(spot, strike, t, vol, r, q,
                                                        option_type, paths, shift, seed))

    def importance_sampling_price_se_batch(self, spot, strike, t, vol, r, q, option_type,
                                           paths, shift, seed):
        return self._call_batch_ctypes("qk_mcm_importance_sampling_price_se_batch",
                                       *self._is_arrays(spot, strike, t, vol, r, q,
                                                        option_type, paths, shift, seed),
                                       with_se=True)

    def _qmc_arrays(self, spot, strike, t, vol, r, q, option_type, paths):
        s = self._as_f64_array(spot, "spot")
        arrs = dict(strike=self._as_f64_array(strike, "strike"), t=self._as_f64_array(t, "t"),
                    vol=self._as_f64_array(vol, "vol"), r=self._as_f64_array(r, "r"),
                    q=self._as_f64_array(q, "q"),
                    option_type=self._as_i32_array(option_type, "option_type"),
                    paths=self._as_i32_array(paths, "paths"))
        self._check_same_length(s.shape[0], **arrs)
        return (s, *arrs.values())

    def quasi_monte_carlo_sobol_price(self, spot: float, strike: float, t: float, vol: float,
                                      r: float, q: float, option_type: int, paths: int) -> float:
        """Sobol points 1..paths through Acklam's inverse normal (quasi_monte_carlo.cpp:10-32)."""
        return self._call_checked("qk_mcm_quasi_monte_carlo_sobol_price",
                                  spot, strike, t, vol, r, q, option_type, paths)

    def quasi_monte_carlo_sobol_price_batch(self, spot, strike, t, vol, r, q, option_type,
                                            paths) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_quasi_monte_carlo_sobol_price_batch",
                                       *self._qmc_arrays(spot, strike, t, vol, r, q,
                                                         option_type, paths))

    def quasi_monte_carlo_sobol_price_se_batch(self, spot, strike, t, vol, r, q, option_type,
                                               paths):
        return self._call_batch_ctypes("qk_mcm_quasi_monte_carlo_sobol_price_se_batch",
                                       *self._qmc_arrays(spot, strike, t, vol, r, q,
                                                         option_type, paths), with_se=True)

    def quasi_monte_carlo_halton_price(self, spot: float, strike: float, t: float, vol: float,
                                       r: float, q: float, option_type: int, paths: int) -> float:
        """Halton base-2 points (quasi_monte_carlo.cpp:34-56)."""
        return self._call_checked("qk_mcm_quasi_monte_carlo_halton_price",
                                  spot, strike, t, vol, r, q, option_type, paths)

    def quasi_monte_carlo_halton_price_batch(self, spot, strike, t, vol, r, q, option_type,
                                             paths) -> np.ndarray:
        return self._call_batch_ctypes("qk_mcm_quasi_monte_carlo_halton_price_batch",
                                       *self._qmc_arrays(spot, strike, t, vol, r, q,
                                                         option_type, paths))

    def quasi_monte_carlo_halton_price_se_batch(self, spot, strike, t, vol, r, q, option_type,
                                                paths):
        return self._call_batch_ctypes("qk_mcm_quasi_monte_carlo_halton_price_se_batch",
                                       *self._qmc_arrays(spot, strike, t, vol, r, q,
                                                         option_type, paths), with_se=True)

    # ------------------------------------------------------------------ Heston CF
    def heston_price_cf(self, spot: float, strike: float, t: float, r: float, q: float,
                        v0: float, kappa: float, theta: float, sigma: float, rho: float,
                        option_type: int, integration_steps: int = 1024,
                        integration_limit: float = 120.0) -> float:
        """Heston characteristic-function price (heston.cpp:7-53; engine.py:362-372)."""
        return self._call_checked("qk_cf_heston_price_cf", spot, strike, t, r, q, v0, kappa,
                                  theta, sigma, rho, option_type, integration_steps,
                                  integration_limit)

    def heston_price_cf_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                              option_type, integration_steps, integration_limit) -> np.ndarray:
        """Batch of heston_price_cf on the GPU, one CTA per option (engine.py:422-449)."""
        s = self._as_f64_array(spot, "spot")
        arrs = dict(
            strike=self._as_f64_array(strike, "strike"), t=self._as_f64_array(t, "t"),
            r=self._as_f64_array(r, "r"), q=self._as_f64_array(q, "q"),
            v0=self._as_f64_array(v0, "v0"), kappa=self._as_f64_array(kappa, "kappa"),
            theta=self._as_f64_array(theta, "theta"), sigma=self._as_f64_array(sigma, "sigma"),
            rho=self._as_f64_array(rho, "rho"),
            option_type=self._as_i32_array(option_type, "option_type"),
            integration_steps=self._as_i32_array(integration_steps, "integration_steps"),
            integration_limit=self._as_f64_array(integration_limit, "integration_limit"),
        )
        self._check_same_length(s.shape[0], **arrs)
        return self._call_batch_ctypes("qk_cf_heston_price_cf_batch", s, *arrs.values())

    def cos_method_fang_oosterlee_heston_price(self, spot: float, strike: float, t: float,
                                               r: float, q: float, v0: float, kappa: float,
                                               theta: float, sigma: float, rho: float,
                                               option_type: int, n_terms: int = 256,
                                               truncation_width: float = 10.0) -> float:
        """Heston price by the COS expansion (cos_method.cpp:30-58; engine.py:742-750)."""
        return self._call_checked("qk_ftm_cos_fang_oosterlee_heston_price", spot, strike, t, r, q,
                                  v0, kappa, theta, sigma, rho, option_type, n_terms,
                                  truncation_width)

    def cos_method_fang_oosterlee_heston_price_batch(self, spot, strike, t, r, q, v0, kappa,
                                                     theta, sigma, rho, option_type, n_terms,
                                                     truncation_width) -> np.ndarray:
        """Batch of the COS pricer on the GPU, one CTA per option (engine.py:752-778)."""
        s = self._as_f64_array(spot, "spot")
        arrs = dict(
            strike=self._as_f64_array(strike, "strike"), t=self._as_f64_array(t, "t"),
            r=self._as_f64_array(r, "r"), q=self._as_f64_array(q, "q"),
            v0=self._as_f64_array(v0, "v0"), kappa=self._as_f64_array(kappa, "kappa"),
            theta=self._as_f64_array(theta, "theta"), sigma=self._as_f64_array(sigma, "sigma"),
            rho=self._as_f64_array(rho, "rho"),
            option_type=self._as_i32_array(option_type, "option_type"),
            n_terms=self._as_i32_array(n_terms, "n_terms"),
            truncation_width=self._as_f64_array(truncation_width, "truncation_width"),
        )
        self._check_same_length(s.shape[0], **arrs)
        return self._call_batch_ctypes("qk_ftm_cos_fang_oosterlee_heston_price_batch", s,
                                       *arrs.values())

    # ------------------------------------------------------------------ mixed / plans
    def _mixed_arrays(self, model, spot, strike, t, vol, r, q, v0, kappa, theta, sigma, rho,
                      option_type, paths, steps, seed):
        m = self._as_i32_array(model, "model")
        n = m.shape[0]

        def f64(x, name):
            return self._as_f64_array(np.zeros(n) if x is None else x, name)

        arrs = dict(
            spot=f64(spot, "spot"), strike=f64(strike, "strike"), t=f64(t, "t"),
            vol=f64(vol, "vol"), r=f64(r, "r"), q=f64(q, "q"), v0=f64(v0, "v0"),
            kappa=f64(kappa, "kappa"), theta=f64(theta, "theta"), sigma=f64(sigma, "sigma"),
            rho=f64(rho, "rho"),
            option_type=self._as_i32_array(option_type, "option_type"),
            paths=self._as_i32_array(paths, "paths"),
            steps=self._as_i32_array(np.ones(n, np.int32) if steps is None else steps, "steps"),
            seed=self._as_u64_array(seed, "seed"),
        )
        self._check_same_length(n, **arrs)
        return [m] + list(arrs.values())

    def mixed_price_batch(self, model, spot, strike, t, vol=None, r=None, q=None, v0=None,
                          kappa=None, theta=None, sigma=None, rho=None, option_type=None,
                          paths=None, steps=None, seed=None):
        """Price a batch mixing QK_MC_* models in one persistent work-stealing launch.

        Returns (prices, standard_errors)."""
        arrays = self._mixed_arrays(model, spot, strike, t, vol, r, q, v0, kappa, theta, sigma,
                                    rho, option_type, paths, steps, seed)
        return self._call_batch_ctypes("qk_mcm_mixed_price_batch", *arrays, with_se=True)

    def plan(self, model, spot, strike, t, vol=None, r=None, q=None, v0=None, kappa=None,
             theta=None, sigma=None, rho=None, option_type=None, paths=None, steps=None,
             seed=None, flags: int = 0) -> "McPlan":
        arrays = self._mixed_arrays(model, spot, strike, t, vol, r, q, v0, kappa, theta, sigma,
                                    rho, option_type, paths, steps, seed)
        return McPlan(self, arrays, flags)


class McPlan:
    """A validated, uploaded batch that can be re-run with inputs resident on the GPU."""

    def __init__(self, qk: QuantKernel, arrays, flags: int):
        self._qk = qk
        self._lib = qk._lib
        self.n = int(arrays[0].shape[0])
        self._h = ct.c_void_p()
        args = [_ptr(a) for a in arrays] + [self.n, int(flags), ct.byref(self._h)]
        rc = self._lib.qk_mcm_plan_create(*args)
        if rc != QK_OK:
            qk._raise_rc("qk_mcm_plan_create", rc)

    def execute(self, stream: int = 0) -> None:
        rc = self._lib.qk_mcm_plan_execute(self._h, ct.c_void_p(stream) if stream else None)
        if rc != QK_OK:
            self._qk._raise_rc("qk_mcm_plan_execute", rc)

    def results(self):
        out = np.empty(self.n, np.float64)
        se = np.empty(self.n, np.float64)
        rc = self._lib.qk_mcm_plan_results(self._h, out.ctypes.data_as(_PD), se.ctypes.data_as(_PD))
        if rc != QK_OK:
            self._qk._raise_rc("qk_mcm_plan_results", rc)
        return out, se

    def device_results(self):
        p = ct.c_void_p()
        s = ct.c_void_p()
        self._lib.qk_mcm_plan_device_results(self._h, ct.byref(p), ct.byref(s))
        return p.value, s.value

    def shard_bounds(self, world: int) -> np.ndarray:
        """Tile bounds of the sharded execute's partition (world + 1 entries)."""
        b = np.empty(int(world) + 1, np.int64)
        rc = self._lib.qk_mcm_plan_shard_bounds(self._h, int(world),
                                                b.ctypes.data_as(ct.POINTER(ct.c_int64)))
        if rc != QK_OK:
            self._qk._raise_rc("qk_mcm_plan_shard_bounds", rc)
        return b

    def execute_tiles(self, tile_begin: int, tile_end: int, stream: int = 0) -> None:
        """The simulate kernels over tiles [tile_begin, tile_end) only."""
        rc = self._lib.qk_mcm_plan_execute_tiles(self._h, int(tile_begin), int(tile_end),
                                                 ct.c_void_p(stream) if stream else None)
        if rc != QK_OK:
            self._qk._raise_rc("qk_mcm_plan_execute_tiles", rc)

    def finalize(self, stream: int = 0) -> None:
        """The finalize kernel over every option (after all tiles' sums are in place)."""
        rc = self._lib.qk_mcm_plan_finalize(self._h, ct.c_void_p(stream) if stream else None)
        if rc != QK_OK:
            self._qk._raise_rc("qk_mcm_plan_finalize", rc)

    def device_partials(self):
        """(device pointer, tiles, bytes per tile) of the per-tile sums."""
        p, n, b = ct.c_void_p(), ct.c_int64(0), ct.c_int32(0)
        self._lib.qk_mcm_plan_device_partials(self._h, ct.byref(p), ct.byref(n), ct.byref(b))
        return p.value, n.value, b.value

    def stats(self):
        ms = ct.c_double(0.0)
        launches = ct.c_int32(0)
        ps = ct.c_int64(0)
        rc = self._lib.qk_mcm_plan_stats(self._h, ct.byref(ms), ct.byref(launches), ct.byref(ps))
        if rc != QK_OK:
            self._qk._raise_rc("qk_mcm_plan_stats", rc)
        return {"simulate_ms": ms.value, "launches": launches.value, "path_steps": ps.value}

    def config(self):
        b, u, c = ct.c_int32(0), ct.c_int32(0), ct.c_int32(0)
        self._lib.qk_mcm_plan_config(self._h, ct.byref(b), ct.byref(u), ct.byref(c))
        su = ct.c_int32(1)
        self._lib.qk_mcm_plan_step_unroll(self._h, ct.byref(su))
        return {"block": b.value, "units_per_thread": u.value, "ctas": c.value,
                "step_unroll": su.value}

    def close(self) -> None:
        if self._h:
            self._lib.qk_mcm_plan_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
