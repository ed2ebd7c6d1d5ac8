"""Calcium recording into device memory (astrosim_record_calcium / astrosim_copy_calcium).

Each recorded sample must equal, bit for bit, the astrocyte calcium that
astrosim_get_state returns after the same step, on the windowed engine and on
the per-step engine, for recordings that start at step 0 and mid-run (mid-window),
and samples past the buffer must be dropped.
"""
import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg

pytestmark = pytest.mark.gpu


def reference_samples(sim, every, first, n, start, steps):
    """Ca after each step t in [start, start + steps) with (t + 1) % every == 0, via get_state."""
    out, t = [], start
    while t < start + steps:
        nxt = ((t // every) + 1) * every  # first t' + 1 multiple of every with t' >= t
        k = min(nxt, start + steps) - t
        sim.step(k)
        t += k
        if t % every == 0:
            out.append(sim.state("Ca")[first:first + n].copy())
    return np.array(out)


@pytest.mark.parametrize("stepper", ["windowed", "plain"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_recording_matches_state(monkeypatch, stepper, precision):
    if stepper == "plain":
        monkeypatch.setenv("ASTROSIM_STEPPER", "plain")
    cfg = dict(n_total=3000, seed=4, pre_ms=0.0, sim_ms=60.0, precision=precision)
    every, first, n = 7, 100, 300
    with asg.Simulation(**cfg) as rec, asg.Simulation(**cfg) as ref:
        rec.step(33)
        ref.step(33)  # start mid-window
        rec.record_calcium(every, first, n, max_samples=1000)
        rec.step(400)
        k, t0 = rec.calcium_samples()
        assert t0 == 34, t0  # (t0 + 1) % 7 == 0, first interval end after step 33
        got = rec.calcium()
        want = reference_samples(ref, every, first, n, 33, 400)
        assert k == len(want)
        np.testing.assert_array_equal(got, want)


def test_recording_drops_past_capacity():
    with asg.Simulation(n_total=2000, seed=2, pre_ms=0.0, sim_ms=50.0, precision="fp32") as sim:
        sim.record_calcium(10, 0, None, max_samples=5)
        sim.step(200)
        k, t0 = sim.calcium_samples()
        assert (k, t0) == (5, 9)
        a = sim.calcium()
        assert a.shape == (5, sim.n_astro)
        with asg.Simulation(n_total=2000, seed=2, pre_ms=0.0, sim_ms=50.0, precision="fp32") as ref:
            ref.step(50)
            np.testing.assert_array_equal(a[4], ref.state("Ca"))


def test_recording_rejects_bad_ranges():
    with asg.Simulation(n_total=1000, seed=1, pre_ms=0.0, sim_ms=10.0) as sim:
        with pytest.raises(asg.AstrosimError):
            sim.record_calcium(0)
        with pytest.raises(asg.AstrosimError):
            sim.record_calcium(5, first=sim.n_astro, n=1)
        with pytest.raises(asg.AstrosimError):
            sim.calcium_samples()
