"""Statistical agreement helpers shared by the GPU parity tests.

For each option z = (gpu - other) / combined SE.  With N options a perfect
estimator still exceeds |z| > 3 with probability 0.0027 each, so a check
allows up to the 99.9% binomial quantile of that count (multiplicity), bounds
max |z| and the mean of z (a biased estimator shifts it).  The observed
statistics are printed.
"""

import math

import numpy as np
from scipy import stats

P_EXCEED = 2.0 * stats.norm.sf(3.0)  # 0.0027


def z_scores(a, b, se):
    """z-score; an option whose payoffs are all zero on both sides (deep out of
    the money) has zero variance and must then agree exactly."""
    a, b, se = map(np.asarray, (a, b, se))
    zero = se == 0
    assert np.all(a[zero] == b[zero])
    return np.where(zero, 0.0, (a - b) / np.where(zero, 1.0, se))


def check_z(z, label, zmax=5.0):
    z = np.asarray(z)
    assert np.all(np.isfinite(z)), label
    n = z.size
    allowed = int(stats.binom.ppf(0.999, n, P_EXCEED))
    exceed = int((np.abs(z) > 3.0).sum())
    print(f"{label}: n={n} mean z={z.mean():+.3f} sd z={z.std():.3f} max|z|={np.abs(z).max():.2f} "
          f"|z|>3: {exceed} (expected {n * P_EXCEED:.2f}, allowed {allowed})")
    assert exceed <= allowed, label
    assert np.abs(z).max() < zmax, label
    # a biased estimator shifts the mean of z; its sd over n options is 1/sqrt(n)
    assert abs(z.mean()) < 4.0 / math.sqrt(n), label
