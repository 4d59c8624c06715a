"""Heston price surrogate: an MLP 9 -> 256 -> 256 -> 256 -> 1 trained on the GPU.

Features, in this order: S/K, T, r, q, v0, kappa, theta, sigma (vol of vol),
rho.  Target: call price / S (prices are homogeneous of degree one in S and
K, so the network works at S = 1).  The network learns the residual over a
base, the Black-Scholes call / S at the Heston mean variance over [0, T]
(theta + (v0 - theta)(1 - exp(-kappa T))/(kappa T)), which the library
computes in FP64 and adds to the network's output.  Inputs are normalised to
[-1, 1] over the training box; `price_batch` prices options inside the box
with the network and the others with the plain GPU Monte Carlo.  Training and inference run on
libqk_b200.so's tcgen05 BF16 GEMMs (FP32 accumulation, FP32 master weights)
and Adam kernels.
"""

import ctypes as ct

import numpy as np

from ._abi import QK_OK
from .engine import QuantKernel

PD = ct.POINTER(ct.c_double)
PI32 = ct.POINTER(ct.c_int32)

FEATURES = ("S/K", "T", "r", "q", "v0", "kappa", "theta", "sigma", "rho")
N_PARAMS = 134401

# The training box of the benchmark's Heston workload: S = 100, K in [70, 130],
# T in [0.25, 2], r in [0, 0.05], q = 0, v0 and theta in [0.01, 0.09],
# kappa in [0.5, 5], vol of vol in [0.1, 1], rho in [-0.9, 0].
HESTON_BOX_LO = np.array([100.0 / 130.0, 0.25, 0.0, 0.0, 0.01, 0.5, 0.01, 0.1, -0.9])
HESTON_BOX_HI = np.array([100.0 / 70.0, 2.0, 0.05, 0.0, 0.09, 5.0, 0.09, 1.0, 0.0])


def _pd(a):
    return a.ctypes.data_as(PD)


def features_of(spot, strike, t, r, q, v0, kappa, theta, sigma, rho):
    """Row-major n x 9 feature matrix."""
    spot = np.asarray(spot, np.float64)
    return np.ascontiguousarray(np.stack([spot / np.asarray(strike, np.float64), t, r, q, v0, kappa,
                                          theta, sigma, rho], axis=1).astype(np.float64))


def sample_box(n, seed, lo=HESTON_BOX_LO, hi=HESTON_BOX_HI, spot=100.0):
    """Uniform Heston parameters in the box as the benchmark draws them (K
    uniform in [spot/hi, spot/lo]); returns a dict of arrays for the MC API."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(size=(n, 9))
    k_lo, k_hi = spot / hi[0], spot / lo[0]
    out = dict(spot=np.full(n, spot), strike=k_lo + (k_hi - k_lo) * u[:, 0])
    for c, name in ((1, "t"), (2, "r"), (3, "q"), (4, "v0"), (5, "kappa"), (6, "theta"),
                    (7, "sigma"), (8, "rho")):
        out[name] = lo[c] + (hi[c] - lo[c]) * u[:, c]
    return out


class HestonSurrogate:
    def __init__(self, qk: QuantKernel = None, box_lo=HESTON_BOX_LO, box_hi=HESTON_BOX_HI,
                 seed: int = 0):
        self.qk = qk or QuantKernel()
        self.lib = self.qk._lib
        self.box_lo = np.ascontiguousarray(box_lo, np.float64)
        self.box_hi = np.ascontiguousarray(box_hi, np.float64)
        self._h = ct.c_void_p()
        self._check(self.lib.qk_sur_heston_create(_pd(self.box_lo), _pd(self.box_hi), int(seed),
                                                  ct.byref(self._h)), "create")

    def _check(self, rc, what):
        if rc != QK_OK:
            self.qk._raise_rc(f"qk_sur_heston_{what}", rc)

    def set_dataset(self, features, target):
        f = np.ascontiguousarray(features, np.float64)
        t = np.ascontiguousarray(target, np.float64)
        assert f.ndim == 2 and f.shape[1] == 9 and t.shape == (f.shape[0],)
        self._check(self.lib.qk_sur_heston_set_dataset(self._h, _pd(f), _pd(t), f.shape[0]), "set_dataset")

    def train(self, epochs, batch=8192, lr=1e-3, shuffle_seed=0):
        losses = np.empty(epochs)
        self._check(self.lib.qk_sur_heston_train(self._h, int(epochs), int(batch), float(lr),
                                                 int(shuffle_seed), _pd(losses)), "train")
        return losses

    def predict(self, features):
        f = np.ascontiguousarray(features, np.float64)
        out = np.empty(f.shape[0])
        self._check(self.lib.qk_sur_heston_predict(self._h, _pd(f), f.shape[0], _pd(out)), "predict")
        return out

    def predict_device(self, x_rows_ptr, base_ptr, n, y_ptr, stream=0, layered=False):
        """Device rows and base in, device price/S out.  The rows are
        features()/features_device() rows: features in columns 0..8, zeros
        in 9..63 (the fused kernel reads columns 0..15).  The fused kernel by
        default; layered=True runs the layer-by-layer GEMMs it is tested
        against."""
        fn = (self.lib.qk_sur_heston_predict_device_layered if layered
              else self.lib.qk_sur_heston_predict_device)
        self._check(fn(self._h, ct.c_void_p(x_rows_ptr), ct.c_void_p(base_ptr) if base_ptr else None,
                       int(n), ct.c_void_p(y_ptr), ct.c_void_p(stream) if stream else None),
                    "predict_device")

    def features_device(self, f_ptr, n, rows_ptr, base_ptr, stream=0):
        """Device features (n x 9 float64) -> device rows [n][64] bf16 and base
        (float32), one launch on `stream`."""
        self._check(self.lib.qk_sur_heston_features_device(
            self._h, ct.c_void_p(f_ptr), int(n), ct.c_void_p(rows_ptr), ct.c_void_p(base_ptr),
            ct.c_void_p(stream) if stream else None), "features_device")

    def features(self, features):
        """Normalised bf16 rows [n][64] as uint16 and the rows' base (float32), host."""
        f = np.ascontiguousarray(features, np.float64)
        out = np.empty((f.shape[0], 64), np.uint16)
        base = np.empty(f.shape[0], np.float32)
        self._check(self.lib.qk_sur_heston_features(self._h, _pd(f), f.shape[0],
                                                    out.ctypes.data_as(ct.c_void_p),
                                                    base.ctypes.data_as(ct.c_void_p)), "features")
        return out, base

    def feature_rows(self, features):
        """Normalised bf16 rows [n][64] as uint16 (host)."""
        return self.features(features)[0]

    def gradients(self, features, target):
        f = np.ascontiguousarray(features, np.float64)
        t = np.ascontiguousarray(target, np.float64)
        g = np.empty(N_PARAMS)
        loss = ct.c_double()
        self._check(self.lib.qk_sur_heston_gradients(self._h, _pd(f), _pd(t), f.shape[0], _pd(g),
                                                     ct.byref(loss)), "gradients")
        return loss.value, g

    def parameters(self):
        p = np.empty(N_PARAMS)
        self._check(self.lib.qk_sur_heston_parameters(self._h, _pd(p)), "parameters")
        return p

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, np.float64)
        assert p.shape == (N_PARAMS,)
        self._check(self.lib.qk_sur_heston_set_parameters(self._h, _pd(p)), "set_parameters")

    def save(self, path):
        self._check(self.lib.qk_sur_heston_save(self._h, str(path).encode()), "save")

    def load(self, path):
        self._check(self.lib.qk_sur_heston_load(self._h, str(path).encode()), "load")

    def price_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                    fallback_paths=262144, fallback_steps=200, fallback_seed=0):
        arrs = [np.ascontiguousarray(x, np.float64) for x in (spot, strike, t, r, q, v0, kappa,
                                                             theta, sigma, rho)]
        ot = np.ascontiguousarray(option_type, np.int32)
        n = arrs[0].shape[0]
        out = np.empty(n)
        src = np.empty(n, np.int32)
        self._check(self.lib.qk_sur_heston_price_batch(
            self._h, *[_pd(a) for a in arrs], ot.ctypes.data_as(PI32), n, int(fallback_paths),
            int(fallback_steps), int(fallback_seed), _pd(out), src.ctypes.data_as(PI32)), "price_batch")
        return out, src

    def close(self):
        if self._h:
            self.lib.qk_sur_heston_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
