"""The shipped surrogate (quantkernel_b200/data/heston_surrogate.qksur) against
its own accuracy contract: Heston call prices within 5e-4 x S of Monte Carlo,
judged by the library's plain GPU Monte Carlo.

* Judge: 1024 seeded queries drawn uniformly inside the training box, priced
  through qk_sur_heston_price_batch (in-box calls go to the network) and
  re-priced by the Heston MC at 200 steps x 4,194,304 paths, whose own
  standard error is about 5e-5 x S.  Bars, stated against that judge: at
  least 99% of the queries within 5e-4 x S, none beyond 1e-3 x S (twice the
  bar: the network's worst in-box error plus four judge standard errors),
  mean error at most 1.2e-4 x S.  Measured: mean 5.4e-5, p99 2.1e-4, max
  3.2e-4 x S, all 1024 within 5e-4 x S; the largest errors sit at Feller
  ratios 2 kappa theta / sigma^2 below 0.5 with sigma above 0.8 and long
  maturities, where the variance process spends most time at zero.
* Arithmetic: the fused inference kernel against the oracle's FP64
  evaluation of the same bf16 network (weights and the bf16 operands of
  layers 2 and 3 rounded as the GPU rounds them).  What is left is FP32
  summation order and the special-function tanh of the SiLU, which can move
  an activation to the neighbouring bf16 value; measured on 20,000 box rows
  of this checkpoint: mean 2.0e-7 x S, max 2.7e-5 x S, and the bars are
  mean 1e-6 and max 1e-4 (x S).  Against the FP64 network on the
  FP32 master weights (no bf16 rounding of weights or activations) the
  trained bf16 network differs by about 6.4e-4 x S on average and 5.4e-3 x S
  at most -- the network was trained in its bf16 form, which is the function
  it ships, so that comparison measures rounding, not the kernel.
"""

from pathlib import Path

import numpy as np
import pytest

from oracle import mlp_oracle as mo
from quantkernel_b200.surrogate import HestonSurrogate, features_of, sample_box

pytestmark = pytest.mark.gpu

CKPT = (Path(__file__).resolve().parents[1] / "quant-kernel_b200" / "quantkernel_b200" / "data" /
        "heston_surrogate.qksur")
KEYS = ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho")


@pytest.fixture(scope="module")
def shipped(qk):
    sur = HestonSurrogate(qk, seed=0)
    sur.load(str(CKPT))
    yield sur
    sur.close()


def test_shipped_surrogate_within_5e4_s_of_mc_judge(qk, shipped):
    n = 1024
    b = sample_box(n, seed=2027)
    ot = np.zeros(n, np.int32)
    price, src = shipped.price_batch(*(b[k] for k in KEYS), ot)
    assert np.all(src == 0), "every query is inside the box: none may fall back to MC"
    jp, jse = qk.heston_monte_carlo_price_se_batch(
        *(b[k] for k in KEYS), ot, np.full(n, 4194304, np.int32), np.full(n, 200, np.int32),
        np.arange(n, dtype=np.uint64) + np.uint64(424242))
    s = b["spot"]
    err = np.abs(price - jp) / s
    judge_se = jse / s
    frac = float((err <= 5e-4).mean())
    feller = 2.0 * b["kappa"] * b["theta"] / b["sigma"] ** 2
    print(f"surrogate vs MC judge (200 x 4194304, SE/S mean {judge_se.mean():.2e}): "
          f"mean {err.mean():.2e} p99 {np.quantile(err, 0.99):.2e} max {err.max():.2e} "
          f"within 5e-4: {frac:.4f}")
    for i in np.argsort(-err)[:8]:
        print(f"  err/S {err[i]:.2e} (judge SE/S {judge_se[i]:.1e}) S/K {s[i] / b['strike'][i]:.3f} "
              f"T {b['t'][i]:.3f} r {b['r'][i]:.4f} v0 {b['v0'][i]:.4f} kappa {b['kappa'][i]:.3f} "
              f"theta {b['theta'][i]:.4f} sigma {b['sigma'][i]:.3f} rho {b['rho'][i]:+.3f} "
              f"Feller {feller[i]:.3f}")
    assert np.all(judge_se < 2.5e-4)
    assert frac >= 0.99, frac
    assert err.max() <= 1e-3, err.max()
    assert err.mean() <= 1.2e-4, err.mean()


def test_shipped_surrogate_fused_kernel_vs_fp64_bf16_network(shipped):
    b = sample_box(20000, seed=2028)
    f = features_of(*(b[k] for k in KEYS))
    y = shipped.predict(f)
    p = shipped.parameters()
    x = mo.bf16_bits_to_float(shipped.feature_rows(f))[:, :9]
    base = mo.bsm_mean_var_base(f)
    err = np.abs(y - (mo.forward_bf16(p, x) + base))
    print(f"fused kernel vs FP64 bf16 network: mean {err.mean():.2e} p999 "
          f"{np.quantile(err, 0.999):.2e} max {err.max():.2e}")
    assert err.mean() <= 1e-6 and err.max() <= 1e-4, (err.mean(), err.max())
