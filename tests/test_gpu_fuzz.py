"""Randomised agreement sweep: 24 configurations drawn from a fixed seed (network
sizes from 1 to 8000 cells, both precisions, dt of 0.05-0.25 ms, substeps, pre-run
lengths and step chunks that start and stop inside windows, STP on and off,
coupling weights).  For each, the windowed engine equals the per-step engine bit
for bit (every state array, every per-step spike count, the summary), and a batch of
the windowed configurations stepped as one ensemble equals each run alone.
"""
import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg
from astrosimgpu_cuda_b200 import abi

pytestmark = pytest.mark.gpu

STATES = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic", "stp_x", "stp_u", "stp_t_last", "Ca", "IP3", "h",
          "sic_factor")
SIZES = (1, 2, 3, 5, 17, 40, 129, 256, 500, 1000, 3000, 8000)


def draw(rng, i):
    dt = float(rng.choice([0.05, 0.1, 0.1, 0.1, 0.2, 0.25]))
    return dict(n_total=int(rng.choice(SIZES)), seed=int(rng.integers(1, 1 << 30)), dt=dt,
                substeps=int(rng.choice([1, 1, 2])), pre_ms=float(rng.choice([0.0, 1.3, 5.0])),
                sim_ms=float(rng.choice([8.0, 20.0, 31.7])), precision=str(rng.choice(["fp64", "fp32"])),
                stp_enabled=int(rng.choice([1, 1, 0])), w_a2n=float(rng.choice([np.nan, 0.0, 1.5])),
                w_n2a=float(rng.choice([np.nan, 0.5])), neuron_drive_scale=float(rng.uniform(0.8, 3.0)))


def run(monkeypatch, stepper, kw, chunks):
    monkeypatch.setenv("ASTROSIM_STEPPER", stepper)
    with asg.Simulation(**kw) as sim:
        for c in chunks:
            sim.step(c)
        out = {k: sim.state(k) for k in STATES}
        out["counts"] = sim.spike_counts()
        out["summary"] = {k: v for k, v in sim.summary().items() if k not in ("build_seconds", "run_seconds")}
    return out


@pytest.mark.parametrize("i", range(24))
def test_engines_agree_on_random_configurations(monkeypatch, i):
    rng = np.random.default_rng(1000 + i)
    kw = draw(rng, i)
    total = int(kw["pre_ms"] / kw["dt"] + 0.5) + int(kw["sim_ms"] / kw["dt"] + 0.5)
    cuts = sorted(set(int(x) for x in rng.integers(1, max(2, total), size=3)))
    chunks = [b - a for a, b in zip([0] + cuts, cuts + [total]) if b > a]
    a = run(monkeypatch, "plain", kw, chunks)
    b = run(monkeypatch, "auto", kw, chunks)
    for k in STATES + ("counts",):
        np.testing.assert_array_equal(b[k], a[k], err_msg=f"{k} {kw}")
    assert b["summary"] == a["summary"], kw


def test_random_ensemble_equals_solo_runs():
    rng = np.random.default_rng(77)
    cfgs = []
    for i in range(12):
        kw = draw(rng, i)
        kw.update(dt=0.1, substeps=1, precision="fp32", sim_ms=20.0, pre_ms=float(rng.choice([0.0, 3.0])))
        cfgs.append(abi.default_config(**kw))
    with asg.Ensemble(cfgs) as ens:
        ens.step(230)  # whole windows; networks of 200 steps stop at their end
        got = [(ens.summary(i), ens.state(i, "V"), ens.state(i, "Ca")) for i in range(len(cfgs))]
    for i, c in enumerate(cfgs):
        with asg.Simulation(c) as sim:
            sim.step(sim.summary()["total_steps"])
            s = sim.summary()
            np.testing.assert_array_equal(got[i][1], sim.state("V"), err_msg=f"network {i} V")
            np.testing.assert_array_equal(got[i][2], sim.state("Ca"), err_msg=f"network {i} Ca")
        for k in ("spikes_total", "mean_ca", "active_astro", "engaged_astro", "steps_done"):
            assert got[i][0][k] == s[k], (i, k, got[i][0][k], s[k])
