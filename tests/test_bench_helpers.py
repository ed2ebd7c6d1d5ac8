"""bench.py's counting and roofline helpers, on the host (no GPU): how many window
launches a timed region takes (whole and partial windows), the per-step byte models
the roofline divides by, and the roofline arithmetic itself."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


@pytest.mark.parametrize("first,n,launches", [
    (0, 10, 1), (0, 20, 2), (100, 1000, 100),   # whole windows
    (5, 20, 3),                                  # --warmup 5 --steps 20: 5 + 10 + 5 steps
    (3, 4, 1), (9, 2, 2), (0, 0, 0),
])
def test_timed_launches_counts_whole_and_partial_windows(first, n, launches):
    assert bench.timed_launches(first, n) == launches


def sizes(active=0):
    return {"n_exc": 8_000_000, "n_inh": 2_000_000, "n_astro": 2_000_000, "n_exc_edges": 800_024_855,
            "n_inh_edges": 199_983_518, "n_e2a_edges": 160_016_336, "n_sic_edges": 160_016_336,
            "active_astro": active}


def test_step_byte_models():
    s = sizes()
    g32, visits = bench.gather_step_bytes(s, "fp32")
    g64, _ = bench.gather_step_bytes(s, "fp64")
    assert visits == 1_320_041_045 and g64 > g32 > 4 * visits
    w32 = bench.window_step_bytes(s, "fp32", spikes_per_step=222.5)
    w64 = bench.window_step_bytes(s, "fp64", spikes_per_step=222.5)
    assert 0 < w32 < w64 < g32          # the window engine reads far less than the gather formulation
    assert bench.window_step_bytes(s, "fp32", 500.0) > w32                      # more spikes, more deposits
    assert bench.window_step_bytes(sizes(active=1000), "fp32", 222.5) > w32     # flagged a2n rows are read


def test_roofline_fractions():
    leg = {"bytes": 1.29e8, "gather_bytes": 6.1e9, "clocks": {"sm_mhz": 1965.0}}
    out = bench.roofline(leg, "fp32", achieved=974.0, peak=6650.0, peak_kind="fallback", ms_step=0.1324, device=0)
    assert out["bound"] == "issue" and out["frac"] == pytest.approx(974.0 / 6650.0)
    issue = out["issue"]
    assert issue["frac"] == pytest.approx(issue["achieved_warp_inst_per_s"] / issue["peak_warp_inst_per_s"])
    assert 0.0 < issue["frac"] < 1.5
    assert out["traffic"] == pytest.approx(bench.PROFILED_WINDOW["fp32"]["dram"] * 10.0 / 3.0)


def test_peak_source_is_named():
    peak, kind = bench.peaks()
    assert kind in ("measured", "fallback") and peak > 1000.0
