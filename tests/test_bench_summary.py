"""bench.py's host-side arithmetic (CPU): the algorithmic bytes per cell-step,
the roofline point of a timing, and the summary block that compares the
reduced precisions with the fp64 step timed the same way."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_algorithmic_bytes_per_cell_step():
    # 12 w per cell (state in and out, AREA, ZBC, FNC) and per unique edge two
    # cell ids, a code byte and three geometry values (SIDE, COSF, SINF)
    C, E = 207_234, 311_715
    assert bench.alg_bytes_per_cell_step(C, E, 8) == pytest.approx(12 * 8 + E / C * (8 + 1 + 3 * 8))
    assert bench.alg_bytes_per_cell_step(C, E, 4) == pytest.approx(12 * 4 + E / C * (8 + 1 + 3 * 4))


def test_summary_compares_reduced_precisions_with_the_warm_fp64_step():
    extras = {
        "split_207k": {"us_per_step": 11.0, "value": 1.0, "error_vs_fp64": {"rel_max": 3e-7}},
        "fp32_207k": {"us_per_step": 10.0, "value": 1.0, "error_vs_fp64": {"rel_max": 9e-7}},
        "persistent": {"c207k": {"us_per_step_two_kernel": 22.0, "us_per_step_persistent": 23.0,
                                 "bit_identical": True}},
        "ensemble": {"split_vs_fp64": 2.0, "split": {"value": 20e9, "error_vs_fp64": {}}},
        "refgpu": {"graph_us_per_step": 45.0},
        "halo": {"error": "no GPU"},
    }
    cells = 207_234
    s = bench.summarize(extras, us_step=24.0, cells=cells)
    assert s["fp64_207k_warm_us_per_step"] == 22.0
    assert s["split_207k"]["vs_fp64_step"] == pytest.approx(2.0)        # 22 / 11, not the timed 24 / 11
    assert s["fp32_207k"]["vs_fp64_step"] == pytest.approx(2.2)
    assert s["ensemble"]["split_vs_plain_fp64_step"] == pytest.approx(20e9 / (cells / 22e-6))
    assert s["reference_gpu"]["speedup_vs_reference_graph"] == pytest.approx(45.0 / 24.0)
    assert s["halo"] == {"error": "no GPU"}


def test_summary_without_the_persistent_leg_uses_the_headline_step():
    extras = {"split_207k": {"us_per_step": 12.0, "value": 1.0}}
    s = bench.summarize(extras, us_step=24.0, cells=1000)
    assert s["fp64_207k_warm_us_per_step"] == 24.0
    assert s["split_207k"]["vs_fp64_step"] == pytest.approx(2.0)


def test_hbm_point():
    p = bench.hbm_point("fp64", 207_234, 311_715, 22.0)
    b = bench.alg_bytes_per_cell_step(207_234, 311_715, 8)
    assert p["hbm_gbs_alg"] == pytest.approx(b * 207_234 / 22e-6 / 1e9)
