"""Mixed-model persistent launch, plans, CUDA graphs and the autotuner.

A path's normals depend only on (seed, path index), and sums are compensated
double-double in a fixed order, so every launch strategy must agree with the
per-method batch calls to a relative 1e-13 (bit for bit when the tile
geometry is the same)."""

import numpy as np
import pytest

from quantkernel_b200 import (QK_MC_EULER, QK_MC_HESTON, QK_MC_HESTON_LR_DELTA, QK_MC_LOCAL_VOL,
                              QK_MC_MILSTEIN, QK_MC_STANDARD, QK_PLAN_AUTOTUNE,
                              QK_PLAN_FAMILY_GRIDS, QK_PLAN_GRAPH, QK_PLAN_NO_ANTITHETIC,
                              QK_PLAN_PERSISTENT, QK_PLAN_STEP_UNROLL2, QK_PLAN_TIMING,
                              workloads)

pytestmark = pytest.mark.gpu


def _small_mixed(n=96, seed=5):
    return workloads.mixed(n, seed=seed, log2_paths=(8.0, 14.0), log2_steps=(2.0, 6.0))


def _per_method(qk, b):
    out = np.empty(len(b["model"]))
    se = np.empty_like(out)
    bsm_keys = ("spot", "strike", "t", "vol", "r", "q", "option_type", "paths", "steps", "seed")
    hes_keys = ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho",
                "option_type", "paths", "steps", "seed")
    for m, fn, keys in ((QK_MC_EULER, qk.euler_maruyama_price_se_batch, bsm_keys),
                        (QK_MC_MILSTEIN, qk.milstein_price_se_batch, bsm_keys),
                        (QK_MC_LOCAL_VOL, qk.local_vol_monte_carlo_price_se_batch, bsm_keys),
                        (QK_MC_HESTON, qk.heston_monte_carlo_price_se_batch, hes_keys)):
        idx = np.nonzero(b["model"] == m)[0]
        p, s = fn(**{k: b[k][idx] for k in keys})
        out[idx] = p
        se[idx] = s
    return out, se


def test_mixed_batch_equals_per_method_calls(qk):
    b = _small_mixed()
    p, se = qk.mixed_price_batch(**b)
    ref_p, ref_se = _per_method(qk, b)
    np.testing.assert_allclose(p, ref_p, rtol=1e-13, atol=0)
    np.testing.assert_allclose(se, ref_se, rtol=1e-10, atol=0)


def test_plan_graph_persistent_autotune_agree(qk):
    b = _small_mixed(64, seed=9)
    base = qk.plan(**b)
    base.execute()
    p0, s0 = base.results()
    for flags in (QK_PLAN_GRAPH, QK_PLAN_PERSISTENT | QK_PLAN_GRAPH | QK_PLAN_TIMING,
                  QK_PLAN_FAMILY_GRIDS, QK_PLAN_FAMILY_GRIDS | QK_PLAN_GRAPH,
                  QK_PLAN_AUTOTUNE, QK_PLAN_AUTOTUNE | QK_PLAN_GRAPH):
        plan = qk.plan(**b, flags=flags)
        for _ in range(3):  # graph replays are deterministic
            plan.execute()
            p, s = plan.results()
            if flags & QK_PLAN_AUTOTUNE:  # the tuner may change the block size
                np.testing.assert_allclose(p, p0, rtol=1e-13, atol=0)
            else:  # same tile geometry in every mode: bit for bit
                np.testing.assert_array_equal(p, p0)
        st = plan.stats()
        cfg = plan.config()
        if flags & QK_PLAN_FAMILY_GRIDS:
            assert cfg["units_per_thread"] == -1
        if flags & QK_PLAN_PERSISTENT:
            assert cfg["units_per_thread"] == 0
        # persistent: simulate + finalize; family grids: one grid per family
        # (Euler with local vol, Milstein, Heston) + finalize
        assert st["launches"] == (4 if cfg["units_per_thread"] == -1 else 2)
        plan.close()
    base.close()


def test_single_family_plan_persistent_equals_grid(qk):
    h = workloads.heston(40, paths=4096, steps=24, seed=3)
    model = np.full(40, QK_MC_HESTON, np.int32)
    grid = qk.plan(model=model, **h)
    pers = qk.plan(model=model, **h, flags=QK_PLAN_PERSISTENT)
    grid.execute()
    pers.execute()
    a, _ = grid.results()
    b, _ = pers.results()
    np.testing.assert_array_equal(a, b)
    plain, _ = qk.heston_monte_carlo_price_se_batch(**h)
    np.testing.assert_array_equal(a, plain)


def test_mixed_batch_with_invalid_and_constant_options(qk):
    b = _small_mixed(16, seed=11)
    b["spot"][3] = -1.0           # invalid -> NaN
    b["t"][5] = 1e-14             # intrinsic
    b["paths"][7] = 1             # invalid count -> NaN
    b["model"][9] = 42            # unknown model -> NaN
    p, se = qk.mixed_price_batch(**b)
    assert np.isnan(p[3]) and np.isnan(p[7]) and np.isnan(p[9])
    assert np.isfinite(p[5]) and np.isnan(se[5])
    ok = [i for i in range(16) if i not in (3, 5, 7, 9)]
    assert np.all(np.isfinite(p[ok])) and np.all(se[ok] > 0)


def test_timing_stats_and_device_results(qk):
    h = workloads.heston(16, paths=8192, steps=32, seed=4)
    plan = qk.plan(model=np.full(16, QK_MC_HESTON, np.int32), **h, flags=QK_PLAN_TIMING)
    plan.execute()
    p, _ = plan.results()
    st = plan.stats()
    assert st["simulate_ms"] > 0 and st["path_steps"] == 16 * 8192 * 32
    dp, ds = plan.device_results()
    assert dp and ds
    plan.close()


@pytest.mark.parametrize("model", [QK_MC_EULER, QK_MC_MILSTEIN, QK_MC_LOCAL_VOL, QK_MC_HESTON,
                                   QK_MC_HESTON_LR_DELTA])
@pytest.mark.parametrize("anti", [True, False])
def test_step_unrolling_gives_the_same_bits(qk, model, anti):
    """Two Philox step blocks per loop iteration (the autotuner's step
    unrolling) draw the same normals and do the same arithmetic: prices and
    standard errors equal the default kernel's bit for bit, for step counts
    that end inside a block, on a block boundary and at one step."""
    n = 24
    rng = np.random.default_rng(int(model) * 7 + int(anti))
    h = workloads.heston(n, paths=2048, steps=8, seed=int(model))
    h["steps"] = rng.choice([1, 2, 3, 5, 6, 7, 12, 13, 37, 200], n).astype(np.int32)
    h["paths"] = rng.choice([2, 3, 1001, 2048, 4097], n).astype(np.int32)
    h["vol"] = rng.uniform(0.1, 0.5, n)
    if model == QK_MC_HESTON_LR_DELTA:
        h["vol"] = np.full(n, 6.0)  # the mixed call's weight-clip column
    extra = 0 if anti else QK_PLAN_NO_ANTITHETIC
    base = qk.plan(model=np.full(n, model, np.int32), **h, flags=extra)
    base.execute()
    p0, s0 = base.results()
    for upt_flag in (0, QK_PLAN_GRAPH):
        plan = qk.plan(model=np.full(n, model, np.int32), **h,
                       flags=extra | upt_flag | QK_PLAN_STEP_UNROLL2)
        assert plan.config()["step_unroll"] == 2
        plan.execute()
        p, s = plan.results()
        np.testing.assert_array_equal(p, p0)
        np.testing.assert_array_equal(s, s0)
        plan.close()
    assert base.config()["step_unroll"] == 1
    base.close()


def test_autotuner_chooses_step_unrolling(qk):
    """The autotuner times block size x units per thread x step unrolling for
    a stepwise plan (and only block x units for a terminal one); whatever it
    picks, the prices stay those of the default shape to the last bits."""
    h = workloads.heston(64, paths=16384, steps=48, seed=21)
    model = np.full(64, QK_MC_HESTON, np.int32)
    base = qk.plan(model=model, **h)
    base.execute()
    p0, _ = base.results()
    tuned = qk.plan(model=model, **h, flags=QK_PLAN_AUTOTUNE)
    cfg = tuned.config()
    assert cfg["step_unroll"] in (1, 2) and cfg["units_per_thread"] in (1, 2, 4)
    assert cfg["step_unroll"] == 1 or cfg["units_per_thread"] <= 2
    tuned.execute()
    p, _ = tuned.results()
    np.testing.assert_allclose(p, p0, rtol=1e-13, atol=0)
    b = workloads.bsm_terminal(16, paths=65536, seed=2)
    term = qk.plan(model=np.full(16, QK_MC_STANDARD, np.int32), steps=np.ones(16, np.int32), **b,
                   flags=QK_PLAN_AUTOTUNE | QK_PLAN_STEP_UNROLL2)
    assert term.config()["step_unroll"] == 1
    for pl in (base, tuned, term):
        pl.close()


def test_mixed_workload_at_full_size_vs_reference_cpu_mc(qk):
    """The full uneven workload (4096 options, Euler / Milstein / local vol /
    Heston, paths 2^12..2^20, steps 16..511) priced by the autotuned plan in a
    CUDA graph, as the benchmark runs it; 256 of its options -- per model the
    ones with the most steps, paths and path-steps (the corner where FP32 path
    state drifts longest) and a seeded random rest -- against the reference's
    own CPU Monte Carlo on the same inputs (tests/golden/mixed_reference.json,
    produced by the oracle that equals the reference bit for bit):
    z = difference / combined SE, per model and over the whole subset."""
    import json
    import sys
    from pathlib import Path

    from stat_check import check_z, z_scores

    golden = Path(__file__).parent / "golden"
    sys.path.insert(0, str(golden))
    from make_mixed_reference import fingerprint

    doc = json.loads((golden / "mixed_reference.json").read_text())
    b = workloads.mixed()
    idx = np.array(doc["index"])
    assert fingerprint(b, idx) == doc["fingerprint"], "the mixed workload changed"
    ref_p = np.array([float.fromhex(x) for x in doc["price"]])
    ref_se = np.array([float.fromhex(x) for x in doc["stderr"]])
    plan = qk.plan(**b, flags=QK_PLAN_AUTOTUNE | QK_PLAN_GRAPH)
    plan.execute()
    p, se = plan.results()
    plan.close()
    # a deep out-of-the-money option may pay nothing on every path (SE 0);
    # z_scores then requires both sides to be exactly 0
    assert np.all(np.isfinite(p)) and np.all(se >= 0)
    z = z_scores(p[idx], ref_p, np.hypot(se[idx], ref_se))
    models = b["model"][idx]
    for m in np.unique(models):
        check_z(z[models == m], f"mixed workload model {int(m)} GPU vs reference CPU MC")
    check_z(z, "mixed workload (256 of 4096 options) GPU vs reference CPU MC")
    # the corner: at least one option per model with >= 500 steps and one with
    # >= 2^20 - 2^15 paths is in the checked set
    for m in np.unique(models):
        k = idx[models == m]
        assert b["steps"][k].max() >= 500 and b["paths"][k].max() >= (1 << 20) - (1 << 15)
