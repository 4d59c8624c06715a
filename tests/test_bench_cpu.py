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
