"""ctypes binding of the CPU oracle (libqk_oracle.so) and of the reference
library compiled from its own sources (oracle/_ref/libquantkernel.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the checker or the timed CPU baseline,
never as a product path.
"""

import ctypes as ct
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "libqk_oracle.so"
REF_SO = HERE / "_ref" / "libquantkernel.so"

D = ct.c_double
I32 = ct.c_int32
U32 = ct.c_uint32
U64 = ct.c_uint64
PD = ct.POINTER(D)
PI32 = ct.POINTER(I32)
PU64 = ct.POINTER(U64)
PU32 = ct.POINTER(U32)

# Model codes shared with the GPU library (QK_MC_* in include/qk_api.h).
STANDARD, ANTITHETIC, EULER, MILSTEIN, LOCAL_VOL, TERMINAL_PLAIN, HESTON, HESTON_LR_DELTA = range(8)
CONTROL_VARIATES, IMPORTANCE_SAMPLING, STRATIFIED, QMC_SOBOL, QMC_HALTON = range(8, 13)
VR_MODELS = (CONTROL_VARIATES, IMPORTANCE_SAMPLING, STRATIFIED, QMC_SOBOL, QMC_HALTON)


def _pd(a):
    return a.ctypes.data_as(PD)


class Oracle:
    """The C restatement: bit-exact reference pricers + SE, closed forms, Philox replay."""

    def __init__(self, path: Path = ORACLE_SO):
        if not path.exists():
            raise OSError(f"{path} missing; run `make -C oracle`")
        lib = ct.CDLL(str(path))
        term = [D, D, D, D, D, D, I32, I32, U64, PD]
        step = [D, D, D, D, D, D, I32, I32, I32, U64, PD]
        sig = {
            "qko_standard_mc": (D, term), "qko_antithetic": (D, term),
            "qko_terminal_plain": (D, term), "qko_euler": (D, step),
            "qko_milstein": (D, step), "qko_local_vol": (D, step),
            "qko_heston": (D, [D] * 10 + [I32, I32, I32, U64, PD]),
            "qko_heston_batch": (None, [PD] * 10 + [PI32, PI32, PI32, PU64, I32, PD, PD]),
            "qko_heston_lr_delta": (D, [D] * 10 + [I32, I32, I32, U64, D, PD]),
            "qko_bsm_family_batch": (None, [I32] + [PD] * 6 + [PI32, PI32, PI32, PU64, I32, PD, PD]),
            "qko_bsm_price": (D, [D] * 6 + [I32]),
            "qko_heston_cf_price": (D, [D] * 10 + [I32, I32, D]),
            "qko_heston_cos_price": (D, [D] * 10 + [I32, I32, D]),
            "qko_heston_cos_error_scale": (D, [D] * 10 + [I32, I32, D]),
            "qko_normals": (None, [U64, I32, PD]),
            "qko_philox4x32_10": (None, [PU32, PU32, PU32]),
            "qko_philox_normals4": (None, [U64, U32, U32, U32, PD]),
            "qko_philox_normals6": (None, [U64, U32, U32, U32, PD]),
            "qko_philox_price": (D, [I32] + [D] * 11 + [I32, I32, I32, U64, I32, PD]),
            "qko_control_variates": (D, term),
            "qko_stratified": (D, term),
            "qko_importance_sampling": (D, [D] * 6 + [I32, I32, D, U64, PD]),
            "qko_qmc_sobol": (D, [D] * 6 + [I32, I32, PD]),
            "qko_qmc_halton": (D, [D] * 6 + [I32, I32, PD]),
            "qko_philox_vr_price": (D, [I32] + [D] * 7 + [I32, I32, U64, PD]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        self.lib = lib

    # -- reference pricers (bit-exact) -------------------------------------------
    def price(self, model, spot, strike, t, vol, r, q, option_type, paths, steps=1, seed=0,
              v0=0.0, kappa=0.0, theta=0.0, sigma=0.0, rho=0.0, shift=0.0):
        se = D()
        L = self.lib
        if model == CONTROL_VARIATES:
            p = L.qko_control_variates(spot, strike, t, vol, r, q, option_type, paths, seed, ct.byref(se))
        elif model == IMPORTANCE_SAMPLING:
            p = L.qko_importance_sampling(spot, strike, t, vol, r, q, option_type, paths, shift,
                                          seed, ct.byref(se))
        elif model == STRATIFIED:
            p = L.qko_stratified(spot, strike, t, vol, r, q, option_type, paths, seed, ct.byref(se))
        elif model == QMC_SOBOL:
            p = L.qko_qmc_sobol(spot, strike, t, vol, r, q, option_type, paths, ct.byref(se))
        elif model == QMC_HALTON:
            p = L.qko_qmc_halton(spot, strike, t, vol, r, q, option_type, paths, ct.byref(se))
        elif model == STANDARD:
            p = L.qko_standard_mc(spot, strike, t, vol, r, q, option_type, paths, seed, ct.byref(se))
        elif model == ANTITHETIC:
            p = L.qko_antithetic(spot, strike, t, vol, r, q, option_type, paths, seed, ct.byref(se))
        elif model == TERMINAL_PLAIN:
            p = L.qko_terminal_plain(spot, strike, t, vol, r, q, option_type, paths, seed, ct.byref(se))
        elif model == EULER:
            p = L.qko_euler(spot, strike, t, vol, r, q, option_type, paths, steps, seed, ct.byref(se))
        elif model == MILSTEIN:
            p = L.qko_milstein(spot, strike, t, vol, r, q, option_type, paths, steps, seed, ct.byref(se))
        elif model == LOCAL_VOL:
            p = L.qko_local_vol(spot, strike, t, vol, r, q, option_type, paths, steps, seed, ct.byref(se))
        elif model == HESTON:
            p = L.qko_heston(spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                             paths, steps, seed, ct.byref(se))
        elif model == HESTON_LR_DELTA:  # vol holds weight_clip
            p = L.qko_heston_lr_delta(spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                      option_type, paths, steps, seed, vol, ct.byref(se))
        else:
            raise ValueError(model)
        return p, se.value

    def heston_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                     paths, steps, seed):
        a = [np.ascontiguousarray(x, np.float64) for x in (spot, strike, t, r, q, v0, kappa, theta, sigma, rho)]
        ot = np.ascontiguousarray(option_type, np.int32)
        pp = np.ascontiguousarray(paths, np.int32)
        st = np.ascontiguousarray(steps, np.int32)
        sd = np.ascontiguousarray(seed, np.uint64)
        n = a[0].shape[0]
        out = np.empty(n)
        se = np.empty(n)
        self.lib.qko_heston_batch(*[_pd(x) for x in a], ot.ctypes.data_as(PI32), pp.ctypes.data_as(PI32),
                                  st.ctypes.data_as(PI32), sd.ctypes.data_as(PU64), n, _pd(out), _pd(se))
        return out, se

    def bsm_family_batch(self, model, spot, strike, t, vol, r, q, option_type, paths, steps, seed):
        a = [np.ascontiguousarray(x, np.float64) for x in (spot, strike, t, vol, r, q)]
        ot = np.ascontiguousarray(option_type, np.int32)
        pp = np.ascontiguousarray(paths, np.int32)
        st = np.ascontiguousarray(steps if steps is not None else np.ones(len(pp)), np.int32)
        sd = np.ascontiguousarray(seed, np.uint64)
        n = a[0].shape[0]
        out = np.empty(n)
        se = np.empty(n)
        self.lib.qko_bsm_family_batch(int(model), *[_pd(x) for x in a], ot.ctypes.data_as(PI32),
                                      pp.ctypes.data_as(PI32), st.ctypes.data_as(PI32),
                                      sd.ctypes.data_as(PU64), n, _pd(out), _pd(se))
        return out, se

    # -- closed forms -------------------------------------------------------------
    def bsm(self, spot, strike, t, vol, r, q, option_type):
        return self.lib.qko_bsm_price(spot, strike, t, vol, r, q, option_type)

    def heston_cf(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                  integration_steps=1024, integration_limit=120.0):
        return self.lib.qko_heston_cf_price(spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                            option_type, integration_steps, integration_limit)

    def heston_cos(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                   n_terms=256, truncation_width=10.0):
        return self.lib.qko_heston_cos_price(spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                             option_type, n_terms, truncation_width)

    def heston_cos_error_scale(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                               option_type, n_terms=256, truncation_width=10.0):
        """First-order rounding-error scale of the COS price: exp(-r t) sum_k
        |term_k| (1 + size of term k's exponent parts before they cancel)."""
        return self.lib.qko_heston_cos_error_scale(spot, strike, t, r, q, v0, kappa, theta, sigma,
                                               rho, option_type, n_terms, truncation_width)

    # -- streams ------------------------------------------------------------------
    def normals(self, seed, n):
        out = np.empty(n)
        self.lib.qko_normals(seed, n, _pd(out))
        return out

    def philox(self, ctr, key):
        c = (U32 * 4)(*ctr)
        k = (U32 * 2)(*key)
        o = (U32 * 4)()
        self.lib.qko_philox4x32_10(c, k, o)
        return list(o)

    def philox_normals6(self, seed, c0, c1, c3):
        z = np.empty(6)
        self.lib.qko_philox_normals6(seed, c0, c1, c3, _pd(z))
        return z

    def philox_normals4(self, seed, c0, c1, c3):
        z = np.empty(4)
        self.lib.qko_philox_normals4(seed, c0, c1, c3, _pd(z))
        return z

    def philox_vr_price(self, model, spot, strike, t, vol, r, q, option_type, paths, seed=0,
                        shift=0.0):
        """Models 8-12 on the GPU's stream and estimators, FP64."""
        se = D()
        p = self.lib.qko_philox_vr_price(model, spot, strike, t, vol, r, q, shift, option_type,
                                         paths, seed, ct.byref(se))
        return p, se.value

    def philox_price(self, model, spot, strike, t, vol, r, q, option_type, paths, steps, seed,
                     v0=0.0, kappa=0.0, theta=0.0, sigma=0.0, rho=0.0, antithetic=True):
        se = D()
        p = self.lib.qko_philox_price(model, spot, strike, t, vol, r, q, v0, kappa, theta, sigma,
                                      rho, option_type, paths, steps, seed, 1 if antithetic else 0,
                                      ct.byref(se))
        return p, se.value


class Reference:
    """The reference library (compiled from its sources by `make -C oracle ref`)."""

    def __init__(self, path: Path = REF_SO):
        if not path.exists():
            raise OSError(f"{path} missing; run `make -C oracle ref` where the reference is present")
        lib = ct.CDLL(str(path))
        term = [D, D, D, D, D, D, I32, I32, U64]
        step = [D, D, D, D, D, D, I32, I32, I32, U64]
        sig = {
            "qk_mcm_standard_monte_carlo_price": (D, term),
            "qk_mcm_antithetic_variates_price": (D, term),
            "qk_mcm_euler_maruyama_price": (D, step),
            "qk_mcm_milstein_price": (D, step),
            "qk_mcm_local_vol_monte_carlo_price": (D, step),
            "qk_mcm_heston_monte_carlo_price": (D, [D] * 10 + [I32, I32, I32, U64]),
            "qk_mcm_heston_lr_delta": (D, [D] * 10 + [I32, I32, I32, U64, D]),
            "qk_mcm_heston_monte_carlo_price_batch": (I32, [PD] * 10 + [PI32, PI32, PI32, PU64, I32, PD]),
            "qk_mcm_standard_monte_carlo_price_batch": (I32, [PD] * 6 + [PI32, PI32, PU64, I32, PD]),
            "qk_mcm_euler_maruyama_price_batch": (I32, [PD] * 6 + [PI32, PI32, PI32, PU64, I32, PD]),
            "qk_cf_black_scholes_merton_price": (D, [D] * 6 + [I32]),
            "qk_cf_heston_price_cf": (D, [D] * 10 + [I32, I32, D]),
            "qk_cf_heston_price_cf_batch": (I32, [PD] * 10 + [PI32, PI32, PD, I32, PD]),
            "qk_ftm_cos_fang_oosterlee_heston_price": (D, [D] * 10 + [I32, I32, D]),
            "qk_ftm_cos_fang_oosterlee_heston_price_batch": (I32, [PD] * 10 + [PI32, PI32, PD, I32, PD]),
            "qk_mcm_control_variates_price": (D, term),
            "qk_mcm_stratified_sampling_price": (D, term),
            "qk_mcm_importance_sampling_price": (D, [D] * 6 + [I32, I32, D, U64]),
            "qk_mcm_quasi_monte_carlo_sobol_price": (D, [D] * 6 + [I32, I32]),
            "qk_mcm_quasi_monte_carlo_halton_price": (D, [D] * 6 + [I32, I32]),
            "qk_mcm_control_variates_price_batch": (I32, [PD] * 6 + [PI32, PI32, PU64, I32, PD]),
            "qk_mcm_stratified_sampling_price_batch": (I32, [PD] * 6 + [PI32, PI32, PU64, I32, PD]),
            "qk_mcm_importance_sampling_price_batch": (I32, [PD] * 6 + [PI32, PI32, PD, PU64, I32, PD]),
            "qk_mcm_quasi_monte_carlo_sobol_price_batch": (I32, [PD] * 6 + [PI32, PI32, I32, PD]),
            "qk_mcm_quasi_monte_carlo_halton_price_batch": (I32, [PD] * 6 + [PI32, PI32, I32, PD]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        self.lib = lib

    def price(self, model, spot, strike, t, vol, r, q, option_type, paths, steps=1, seed=0,
              v0=0.0, kappa=0.0, theta=0.0, sigma=0.0, rho=0.0, shift=0.0):
        L = self.lib
        if model == CONTROL_VARIATES:
            return L.qk_mcm_control_variates_price(spot, strike, t, vol, r, q, option_type, paths, seed)
        if model == IMPORTANCE_SAMPLING:
            return L.qk_mcm_importance_sampling_price(spot, strike, t, vol, r, q, option_type, paths,
                                                      shift, seed)
        if model == STRATIFIED:
            return L.qk_mcm_stratified_sampling_price(spot, strike, t, vol, r, q, option_type, paths, seed)
        if model == QMC_SOBOL:
            return L.qk_mcm_quasi_monte_carlo_sobol_price(spot, strike, t, vol, r, q, option_type, paths)
        if model == QMC_HALTON:
            return L.qk_mcm_quasi_monte_carlo_halton_price(spot, strike, t, vol, r, q, option_type, paths)
        if model == STANDARD:
            return L.qk_mcm_standard_monte_carlo_price(spot, strike, t, vol, r, q, option_type, paths, seed)
        if model == ANTITHETIC:
            return L.qk_mcm_antithetic_variates_price(spot, strike, t, vol, r, q, option_type, paths, seed)
        if model == EULER:
            return L.qk_mcm_euler_maruyama_price(spot, strike, t, vol, r, q, option_type, paths, steps, seed)
        if model == MILSTEIN:
            return L.qk_mcm_milstein_price(spot, strike, t, vol, r, q, option_type, paths, steps, seed)
        if model == LOCAL_VOL:
            return L.qk_mcm_local_vol_monte_carlo_price(spot, strike, t, vol, r, q, option_type, paths, steps, seed)
        if model == HESTON:
            return L.qk_mcm_heston_monte_carlo_price(spot, strike, t, r, q, v0, kappa, theta, sigma,
                                                     rho, option_type, paths, steps, seed)
        if model == HESTON_LR_DELTA:  # vol holds weight_clip
            return L.qk_mcm_heston_lr_delta(spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                            option_type, paths, steps, seed, vol)
        raise ValueError(model)

    def heston_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                     paths, steps, seed):
        a = [np.ascontiguousarray(x, np.float64) for x in (spot, strike, t, r, q, v0, kappa, theta, sigma, rho)]
        ot = np.ascontiguousarray(option_type, np.int32)
        pp = np.ascontiguousarray(paths, np.int32)
        st = np.ascontiguousarray(steps, np.int32)
        sd = np.ascontiguousarray(seed, np.uint64)
        n = a[0].shape[0]
        out = np.empty(n)
        rc = self.lib.qk_mcm_heston_monte_carlo_price_batch(
            *[_pd(x) for x in a], ot.ctypes.data_as(PI32), pp.ctypes.data_as(PI32),
            st.ctypes.data_as(PI32), sd.ctypes.data_as(PU64), n, _pd(out))
        if rc != 0:
            raise RuntimeError(f"reference batch rc={rc}")
        return out

    def vr_batch(self, model, spot, strike, t, vol, r, q, option_type, paths, seed=None,
                 shift=None):
        """The reference's OpenMP batch of a variance-reduction method."""
        a = [np.ascontiguousarray(x, np.float64) for x in (spot, strike, t, vol, r, q)]
        ot = np.ascontiguousarray(option_type, np.int32)
        pp = np.ascontiguousarray(paths, np.int32)
        n = a[0].shape[0]
        out = np.empty(n)
        args = [_pd(x) for x in a] + [ot.ctypes.data_as(PI32), pp.ctypes.data_as(PI32)]
        name = {CONTROL_VARIATES: "qk_mcm_control_variates_price_batch",
                STRATIFIED: "qk_mcm_stratified_sampling_price_batch",
                IMPORTANCE_SAMPLING: "qk_mcm_importance_sampling_price_batch",
                QMC_SOBOL: "qk_mcm_quasi_monte_carlo_sobol_price_batch",
                QMC_HALTON: "qk_mcm_quasi_monte_carlo_halton_price_batch"}[model]
        if model == IMPORTANCE_SAMPLING:
            sh = np.ascontiguousarray(shift, np.float64)
            args.append(_pd(sh))
        if model not in (QMC_SOBOL, QMC_HALTON):
            sd = np.ascontiguousarray(seed, np.uint64)
            args.append(sd.ctypes.data_as(PU64))
        rc = getattr(self.lib, name)(*args, n, _pd(out))
        if rc != 0:
            raise RuntimeError(f"reference batch rc={rc}")
        return out

    def bsm(self, spot, strike, t, vol, r, q, option_type):
        return self.lib.qk_cf_black_scholes_merton_price(spot, strike, t, vol, r, q, option_type)

    def heston_cf(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                  integration_steps=1024, integration_limit=120.0):
        return self.lib.qk_cf_heston_price_cf(spot, strike, t, r, q, v0, kappa, theta, sigma, rho,
                                              option_type, integration_steps, integration_limit)

    def heston_cos(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                   n_terms=256, truncation_width=10.0):
        return self.lib.qk_ftm_cos_fang_oosterlee_heston_price(
            spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type, n_terms,
            truncation_width)

    def heston_cf_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                        integration_steps, integration_limit):
        """qk_cf_heston_price_cf_batch (OpenMP over options for n >= 512)."""
        a = [np.ascontiguousarray(x, np.float64) for x in (spot, strike, t, r, q, v0, kappa, theta, sigma, rho)]
        ot = np.ascontiguousarray(option_type, np.int32)
        st = np.ascontiguousarray(integration_steps, np.int32)
        lim = np.ascontiguousarray(integration_limit, np.float64)
        n = a[0].shape[0]
        out = np.empty(n)
        rc = self.lib.qk_cf_heston_price_cf_batch(
            *[_pd(x) for x in a], ot.ctypes.data_as(PI32), st.ctypes.data_as(PI32), _pd(lim), n,
            _pd(out))
        if rc != 0:
            raise RuntimeError(f"reference batch rc={rc}")
        return out

    def heston_cos_batch(self, spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type,
                         n_terms, truncation_width):
        """qk_ftm_cos_fang_oosterlee_heston_price_batch."""
        a = [np.ascontiguousarray(x, np.float64) for x in (spot, strike, t, r, q, v0, kappa, theta, sigma, rho)]
        ot = np.ascontiguousarray(option_type, np.int32)
        nt = np.ascontiguousarray(n_terms, np.int32)
        w = np.ascontiguousarray(truncation_width, np.float64)
        n = a[0].shape[0]
        out = np.empty(n)
        rc = self.lib.qk_ftm_cos_fang_oosterlee_heston_price_batch(
            *[_pd(x) for x in a], ot.ctypes.data_as(PI32), nt.ctypes.data_as(PI32), _pd(w), n,
            _pd(out))
        if rc != 0:
            raise RuntimeError(f"reference batch rc={rc}")
        return out


def reference_available() -> bool:
    return REF_SO.exists()


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# --------------------------------------------------------------------------- C++ timing
CPU_TIMER = HERE / "_ref" / "cpu_timer"
_TERM_F64 = ("spot", "strike", "t", "vol", "r", "q")
_HES_F64 = ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho")
# The reference batch entry points the timer calls, with the batch keys of
# their float64 and int32 arguments in declaration order (qk_api.h).
TIMER_SIGNATURES = {
    "qk_mcm_heston_monte_carlo_price_batch": (_HES_F64, ("option_type", "paths", "steps")),
    "qk_mcm_standard_monte_carlo_price_batch": (_TERM_F64, ("option_type", "paths")),
    "qk_mcm_antithetic_variates_price_batch": (_TERM_F64, ("option_type", "paths")),
    "qk_mcm_euler_maruyama_price_batch": (_TERM_F64, ("option_type", "paths", "steps")),
    "qk_mcm_milstein_price_batch": (_TERM_F64, ("option_type", "paths", "steps")),
    "qk_mcm_local_vol_monte_carlo_price_batch": (_TERM_F64, ("option_type", "paths", "steps")),
}
# The reference batch entry point of each stepwise / terminal model code.
MODEL_BATCH_SYMBOL = {
    STANDARD: "qk_mcm_standard_monte_carlo_price_batch",
    ANTITHETIC: "qk_mcm_antithetic_variates_price_batch",
    EULER: "qk_mcm_euler_maruyama_price_batch",
    MILSTEIN: "qk_mcm_milstein_price_batch",
    LOCAL_VOL: "qk_mcm_local_vol_monte_carlo_price_batch",
    HESTON: "qk_mcm_heston_monte_carlo_price_batch",
}


def timer_available() -> bool:
    return CPU_TIMER.exists() and REF_SO.exists()


def write_timer_input(path, symbol, batch):
    """The cpu_timer input file for `symbol` on `batch` (dict of arrays)."""
    f64, i32 = TIMER_SIGNATURES[symbol]
    n = len(batch["spot"])
    with open(path, "wb") as fh:
        fh.write(np.array([len(f64), len(i32), 1, n], np.int32).tobytes())
        for k in f64:
            fh.write(np.ascontiguousarray(batch[k], np.float64).tobytes())
        for k in i32:
            fh.write(np.ascontiguousarray(batch[k], np.int32).tobytes())
        fh.write(np.ascontiguousarray(batch["seed"], np.uint64).tobytes())


def time_reference_batch(symbol, batch, reps=1, timeout=1800):
    """Calls the reference's batch entry point `symbol` on `batch` `reps` times
    from C++ (oracle/_ref/cpu_timer: dlopen, std::chrono::steady_clock around
    each call; OpenMP threads from OMP_NUM_THREADS).  Returns (seconds of each
    call, sum of the last call's prices)."""
    import json
    import subprocess
    import tempfile

    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        path = f.name
    try:
        write_timer_input(path, symbol, batch)
        r = subprocess.run([str(CPU_TIMER), str(REF_SO), symbol, path, str(reps)],
                           capture_output=True, text=True, timeout=timeout)
    finally:
        os.unlink(path)
    if r.returncode != 0:
        raise RuntimeError(f"cpu_timer failed: {r.stderr[-1000:]}")
    out = json.loads(r.stdout.strip().splitlines()[-1])
    return out["seconds"], out["price_sum"]
