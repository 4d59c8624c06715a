"""The throughput probe behind the Monte Carlo rooflines' denominators
(qk_b200_pipe_probe, include/qk_diag.h): each measured width lies near the
B200's nominal per-SM-clock figure, so a roofline fraction computed from it
means what it says."""

import ctypes as ct

import pytest

pytestmark = pytest.mark.gpu

MUFU, FFMA, FFMA2, DFMA, MIX = 0, 1, 2, 3, 4


def _probe(qk, kind):
    v = ct.c_double(-1.0)
    rc = qk._lib.qk_b200_pipe_probe(0, kind, ct.byref(v))
    assert rc == 0
    return v.value


def test_measured_widths_near_nominal(qk):
    qk.set_device(0)
    xu, ffma, ffma2, dfma, mix = (_probe(qk, k) for k in (MUFU, FFMA, FFMA2, DFMA, MIX))
    print(f"lane-ops per SM per clock: MUFU {xu:.2f} FFMA {ffma:.1f} FFMA2 {ffma2:.1f} "
          f"DFMA {dfma:.1f} MUFU-in-mix {mix:.2f}")
    assert 14.0 <= xu <= 16.5          # 16 special-function lanes per SM
    assert 110.0 <= ffma <= 130.0      # 4 schedulers x 32 lanes
    assert 110.0 <= ffma2 <= 130.0     # packed pairs: half the instructions, same lanes
    assert 50.0 <= dfma <= 66.0        # 64 FP64 lanes per SM
    assert 0.0 < mix <= xu * 1.02      # a mix cannot beat the pure MUFU stream


def test_rejects_bad_arguments(qk):
    v = ct.c_double(0.0)
    assert qk._lib.qk_b200_pipe_probe(0, 99, ct.byref(v)) == -1
    assert qk._lib.qk_b200_pipe_probe(0, MUFU, None) == -1
