"""The benchmark's host-side pieces that need no GPU: the ncu figures its
roofline block reads from the committed profile summary."""

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_committed_ncu_figures_are_complete_and_plausible():
    figs = bench.ncu_figures()
    assert set(figs) == set(bench.NCU_FIGURES)
    # a compute-bound kernel: a few bytes of option records per path-step at most
    assert 0 < figs["dram_bytes_per_launch_full"] < 1e-3 * 1024 * 262144 * 200
    # below the reference formulas' count per path-step (6 XU, 50 ALU)
    assert 0 < figs["xu_per_path_step"] < bench.XU_PER_UNIT
    assert 0 < figs["thread_instructions_per_path_step"] < bench.ALU_PER_UNIT
    for key in ("issue_busy", "xu_pipe_busy"):
        assert 0 < figs[key] <= 1


def test_ncu_figures_read_only_the_listed_keys(tmp_path):
    p = tmp_path / "summary.md"
    p.write_text("| table | 1 |\nissue_busy: 0.5\nother_key: 3\nxu_per_path_step: 2.5\n")
    assert bench.ncu_figures(p) == {"issue_busy": 0.5, "xu_per_path_step": 2.5}
    assert bench.ncu_figures(tmp_path / "missing.md") == {}


class _FakeLib:
    """Stands in for the library: qk_b200_pipe_probe writes `rates[kind]`
    and returns `rc` (no GPU involved)."""

    def __init__(self, rates, rc=0):
        self.rates, self.rc = rates, rc

    def qk_b200_pipe_probe(self, device, kind, out):
        out._obj.value = self.rates[kind]
        return self.rc


class _FakeQK:
    def __init__(self, lib):
        self._lib = lib


def test_measured_pipe_widths_replace_the_nominal_ones(monkeypatch):
    monkeypatch.setattr(bench, "PIPES", dict(bench.PIPES))
    rates = {1: 125.8, 0: 15.97, 3: 63.8, 2: 127.5, 4: 14.8}
    got = bench.measure_pipes(_FakeQK(_FakeLib(rates)), 0)
    assert got == {"issue": 125.8, "xu": 15.97, "fp64": 63.8, "ffma2_lanes": 127.5,
                   "xu_in_heston_mix": 14.8}
    assert (bench.PIPES["issue"], bench.PIPES["xu"], bench.PIPES["fp64"]) == (125.8, 15.97, 63.8)
    assert bench.PIPES["source"].startswith("measured")


def test_nominal_pipe_widths_stay_when_the_probe_fails(monkeypatch):
    nominal = dict(bench.PIPES)
    monkeypatch.setattr(bench, "PIPES", dict(nominal))
    rates = {k: 1.0 for k in range(5)}
    assert bench.measure_pipes(_FakeQK(_FakeLib(rates, rc=-1)), 0) is None
    assert bench.measure_pipes(_FakeQK(_FakeLib({**rates, 0: 0.0})), 0) is None
    assert bench.measure_pipes(_FakeQK(object()), 0) is None  # an older library
    assert bench.PIPES == nominal
    assert (nominal["issue"], nominal["xu"], nominal["fp64"]) == (128.0, 16.0, 64.0)
