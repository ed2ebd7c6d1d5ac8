"""The windowed engine (one launch per 1 ms window, spikes pushed into inboxes, or
pulled from the previous window's spike words) gives bit-identical results to the
per-step path, which itself matches the oracle and the reference (test_gpu_parity,
test_gpu_reference_golden).  Both engines are forced through ASTROSIM_STEPPER and
the pull fallback through ASTROSIM_PUSH_LIMIT."""
import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg

pytestmark = pytest.mark.gpu

STATES = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic", "stp_x", "stp_u", "stp_t_last", "Ca", "IP3", "h",
          "sic_factor")


def run(monkeypatch, stepper, push_limit, chunks, **kw):
    monkeypatch.setenv("ASTROSIM_STEPPER", stepper)
    if push_limit is None:
        monkeypatch.delenv("ASTROSIM_PUSH_LIMIT", raising=False)
    else:
        monkeypatch.setenv("ASTROSIM_PUSH_LIMIT", str(push_limit))
    with asg.Simulation(**kw) as sim:
        for c in chunks:
            sim.step(c)
        out = {k: sim.state(k) for k in STATES}
        out["counts"] = sim.spike_counts()
        out["summary"] = {k: v for k, v in sim.summary().items() if k not in ("build_seconds", "run_seconds")}
        if kw.get("raster_steps"):
            out["raster"] = sim.raster()
    return out


@pytest.mark.parametrize("n_total,seed,precision", [(500, 1, "fp64"), (5000, 2, "fp64"), (2000, 3, "fp32"),
                                                    (20000, 7, "fp64"), (20000, 7, "fp32")])
def test_windowed_push_and_pull_match_per_step_path(monkeypatch, n_total, seed, precision):
    kw = dict(n_total=n_total, seed=seed, pre_ms=30, sim_ms=120, precision=precision, raster_steps=600)
    chunks = (3, 17, 100, 1117, 263)
    ref = run(monkeypatch, "plain", None, chunks, **kw)
    for push_limit in (None, 0):
        got = run(monkeypatch, "auto", push_limit, chunks, **kw)
        for k in STATES + ("counts", "raster"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{k} push_limit={push_limit}")
        assert got["summary"] == ref["summary"]
    assert ref["counts"].sum() > 0


def test_windowed_dt_quarter_ms(monkeypatch):
    kw = dict(n_total=3000, seed=4, pre_ms=10, sim_ms=90, dt=0.25)  # D = 4 steps
    ref = run(monkeypatch, "plain", None, (400,), **kw)
    got = run(monkeypatch, "auto", None, (7, 393), **kw)
    for k in STATES + ("counts",):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_every_launch_variant_is_bit_identical(monkeypatch, precision):
    """Every (block size, occupancy target) pair the autotuner may pick (block 0:
    nine variants over 64/128/256 threads), a fixed tuned size (64: its three
    variants) and block sizes outside the table (96, 512: the generic kernel) give
    the per-step path's results bit for bit."""
    kw = dict(n_total=4000, seed=5, pre_ms=20, sim_ms=60, precision=precision)
    ref = run(monkeypatch, "plain", None, (800,), **kw)
    cases = [(0, v) for v in range(9)] + [(64, v) for v in range(3)] + [(96, None), (512, None), (256, None)]
    for block, v in cases:
        if v is None:
            monkeypatch.delenv("ASTROSIM_WINDOW_VARIANT", raising=False)
        else:
            monkeypatch.setenv("ASTROSIM_WINDOW_VARIANT", str(v))
        got = run(monkeypatch, "auto", None, (13, 787), block=block, **kw)
        for k in STATES + ("counts",):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{k} block {block} variant {v}")
    monkeypatch.delenv("ASTROSIM_WINDOW_VARIANT", raising=False)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("sic_th,w_a2n,min_active", [(0.06, 3.0, 1000), (0.0705, 1.0, 100), (0.071, 1.0, 10)])
def test_active_astrocytes_windowed_matches_per_step(monkeypatch, precision, sic_th, w_a2n, min_active):
    """Lowered SIC thresholds make every astrocyte, a few hundred or a few tens of
    them active (the oracle at these settings: 1200, 140-310 and 16-48 of 1200
    active from 20 ms on).  The push flags the neurons whose a2n rows hold an active
    astrocyte and only those walk their rows; results equal the per-step path's,
    over irregular chunks (partial windows), with push and with pull delivery."""
    bio = {"SIC_th": sic_th, "w_a2n": w_a2n}
    kw = dict(n_total=6000, seed=13, pre_ms=10, sim_ms=90, precision=precision, raster_steps=1000)
    chunks = (7, 3, 120, 451, 419)
    monkeypatch.setenv("ASTROSIM_STEPPER", "plain")
    with asg.Simulation(biology=bio, **kw) as s:
        for c in chunks:
            s.step(c)
        ref = {k: s.state(k) for k in STATES}
        ref["counts"] = s.spike_counts()
        ref_active = int((s.state("sic_factor") > 0).sum())
    for push_limit in (None, 0):
        monkeypatch.setenv("ASTROSIM_STEPPER", "auto")
        if push_limit is None:
            monkeypatch.delenv("ASTROSIM_PUSH_LIMIT", raising=False)
        else:
            monkeypatch.setenv("ASTROSIM_PUSH_LIMIT", str(push_limit))
        with asg.Simulation(biology=bio, **kw) as s:
            for c in chunks:
                s.step(c)
            for k in STATES:
                np.testing.assert_array_equal(s.state(k), ref[k], err_msg=f"{k} push_limit={push_limit}")
            np.testing.assert_array_equal(s.spike_counts(), ref["counts"])
    monkeypatch.delenv("ASTROSIM_PUSH_LIMIT", raising=False)
    assert ref_active >= min_active, ref_active


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_every_variant_bit_identical_with_facilitation_and_active_astrocytes(monkeypatch, precision):
    """The regime where the launch-bounds instantiations once rounded the Tsodyks-
    Markram update differently (one fused step * dt - t_last): strong SIC input makes
    neurons fire often, and facilitation (U = 0.3, tau_fac = 150 ms) makes u vary.
    Every variant gives the per-step path's results bit for bit."""
    bio = {"SIC_th": 0.06, "w_a2n": 3.0, "stp_U": 0.3, "stp_tau_fac": 150.0}
    kw = dict(n_total=6000, seed=13, pre_ms=10, sim_ms=50, precision=precision)
    monkeypatch.setenv("ASTROSIM_STEPPER", "plain")
    with asg.Simulation(biology=bio, **kw) as s:
        s.step(600)
        ref = {k: s.state(k) for k in STATES}
        ref["counts"] = s.spike_counts()
    assert ref["counts"].sum() > 5000
    monkeypatch.setenv("ASTROSIM_STEPPER", "auto")
    for v in range(9):
        monkeypatch.setenv("ASTROSIM_WINDOW_VARIANT", str(v))
        with asg.Simulation(biology=bio, **kw) as s:
            for c in (7, 3, 290, 300):
                s.step(c)
            for k in STATES:
                np.testing.assert_array_equal(s.state(k), ref[k], err_msg=f"{k} variant {v}")
            np.testing.assert_array_equal(s.spike_counts(), ref["counts"], err_msg=f"variant {v}")
    monkeypatch.delenv("ASTROSIM_WINDOW_VARIANT", raising=False)
