"""The CUDA path reproduces the reference program's own GPU outputs.

tests/golden/reference_dynamics.json holds the summaries that the unmodified
reference binary (built from src/astrosim_fused.cu for sm_100a) printed on a B200,
recorded by tests/golden/make_reference_dynamics_golden.py.  For the FP64 cases
the spike counts, the final-step and engaged astrocyte counts, the windowed rates
and the printed mean calcium must match exactly.  The reference's FP32 build
(-DASTROSIM_USE_FLOAT) draws a different network, so FP32 cases are compared as
statistics (mean rate within 2 %).
"""
import json
import os

import pytest

import astrosimgpu_cuda_b200 as asg

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_dynamics.json")))


def windowed_rates(sim, s, dt=0.1):
    """The reference's checkpoint lines (src/astrosim_fused.cu:1081-1095) from per-step counts."""
    pre, sim_steps, total = s["pre_steps"], s["sim_steps"], s["total_steps"]
    every = max(1, sim_steps // 10)
    counts = sim.spike_counts(0, total)
    mark = 0 if pre == 0 else pre - 1
    last_cp, at_last, out = pre, int(counts[: mark + 1].sum()), []
    for step in range(pre + every, total, every):
        now = int(counts[: step + 1].sum())
        out.append(round((now - at_last) / (sim.n_neurons * (step - last_cp) * dt * 1e-3), 4))
        at_last, last_cp = now, step
    return out


@pytest.mark.parametrize("rec", [r for r in GOLDEN if r["precision"] == "fp64"],
                         ids=lambda r: f"n{r['n_total']}_pre{r['pre_ms']}_sim{r['sim_ms']}")
def test_fp64_matches_reference_gpu_run(rec):
    with asg.Simulation(n_total=rec["n_total"], seed=rec["seed"], pre_ms=rec["pre_ms"], sim_ms=rec["sim_ms"]) as sim:
        s = sim.summary()
        sim.step(s["total_steps"])
        s = sim.summary()
        assert f"connectivity: exc={s['n_exc_edges']} inh={s['n_inh_edges']} e2a={s['n_e2a_edges']} " \
               f"sic={s['n_sic_edges']}" == rec["connectivity"]
        assert s["spikes_measured"] == rec["spikes_measured"]
        assert f"{s['mean_rate_hz']:.4f}" == f"{rec['mean_rate_hz']:.4f}"
        assert f"{s['mean_ca']:.6g}" == rec["mean_ca_str"]
        assert s["active_astro"] == rec["active_astro"]
        assert s["engaged_astro"] == rec["engaged_astro"]
        assert windowed_rates(sim, s) == [round(x, 4) for x in rec["windowed_hz"]]


@pytest.mark.parametrize("rec", [r for r in GOLDEN if r["precision"] == "fp32"],
                         ids=lambda r: f"n{r['n_total']}")
def test_fp32_statistics_match_reference_fp32_build(rec):
    with asg.Simulation(n_total=rec["n_total"], seed=rec["seed"], pre_ms=rec["pre_ms"], sim_ms=rec["sim_ms"],
                        precision="fp32") as sim:
        sim.step(sim.summary()["total_steps"])
        s = sim.summary()
    assert abs(s["mean_rate_hz"] - rec["mean_rate_hz"]) <= 0.02 * rec["mean_rate_hz"]
