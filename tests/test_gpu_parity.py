"""GPU parity of the CUDA path (through the C ABI) against the reference's golden
connectivity and against the FP64 oracle (oracle/astrosim_oracle.cpp).

Tolerances:
  connectivity            bit-exact (SHA-256 of every CSR array)
  per-cell parameters     rtol 1e-14 (CUDA vs host libm in the Box-Muller normals)
  FP64 state, 100 steps   |gpu - oracle| <= 1e-12 * max(|oracle|, 1) elementwise
  FP64 spike raster       identical over the first 200 ms (2000 steps)
  FP32 spike raster       identical over the first 50 ms (500 steps)
  FP32 summary            mean rate within 2 % and SIC-threshold fraction within
                          0.02 of the FP64 oracle
"""
import hashlib

import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg
from oracle import oracle

pytestmark = pytest.mark.gpu

STATE_NEURON = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic", "stp_x", "stp_u", "stp_t_last")
STATE_ASTRO = ("Ca", "IP3", "h", "sic_factor")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def check_csrs(sim, rec):
    for k in ("exc", "inh", "sic", "e2a"):
        rs, src = sim.csr(k)
        assert src.size == rec["edges"][k], (rec["n_total"], rec["seed"], k)
        assert sha(rs) == rec["sha256"][k]["row_start"], (rec["n_total"], rec["seed"], k, "row_start")
        assert sha(src) == rec["sha256"][k]["src"], (rec["n_total"], rec["seed"], k, "src")


def test_connectivity_small_networks_bit_exact(golden_connectivity):
    n = 0
    for rec in golden_connectivity.values():
        if rec["n_total"] > 10000:
            continue
        with asg.Simulation(n_total=rec["n_total"], seed=rec["seed"], pre_ms=0, sim_ms=0) as sim:
            check_csrs(sim, rec)
        n += 1
    assert n >= 70


@pytest.mark.parametrize("n_total,seed", [(500, 1), (5000, 2), (4, 7)])
def test_parameters_match_oracle(n_total, seed):
    o = oracle.OracleSim(n_total=n_total, seed=seed, pre_ms=0, sim_ms=0)
    with asg.Simulation(n_total=n_total, seed=seed, pre_ms=0, sim_ms=0) as sim:
        for name in ("Ca_tot", "IP3_0", "tau_IP3", "delta_IP3", "V_reset", "b"):
            np.testing.assert_allclose(sim.state(name), o.state(name), rtol=1e-14, atol=0, err_msg=name)


def test_initial_state_matches_oracle():
    o = oracle.OracleSim(n_total=500, seed=1)
    with asg.Simulation(n_total=500, seed=1) as sim:
        for name in STATE_NEURON + STATE_ASTRO:
            np.testing.assert_array_equal(sim.state(name), o.state(name), err_msg=name)


def assert_state_close(sim, o, tag):
    for name in STATE_NEURON + STATE_ASTRO:
        a, b = sim.state(name), o.state(name)
        tol = 1e-12 * np.maximum(np.abs(b), 1.0)
        bad = np.abs(a - b) > tol
        assert not bad.any(), f"{tag} {name}: {bad.sum()} cells, max |d| {np.max(np.abs(a - b)):.3e}"


@pytest.mark.parametrize("n_total,seed", [(500, 1), (3000, 5)])
def test_fp64_state_matches_oracle_first_100_steps(n_total, seed):
    o = oracle.OracleSim(n_total=n_total, seed=seed, pre_ms=5, sim_ms=50)
    with asg.Simulation(n_total=n_total, seed=seed, pre_ms=5, sim_ms=50) as sim:
        done = 0
        for chunk in (1, 9, 40, 50):
            sim.step(chunk)
            o.step(chunk)
            done += chunk
            assert_state_close(sim, o, f"step {done}")
        np.testing.assert_array_equal(sim.spike_counts(), o.spike_counts())


@pytest.mark.parametrize("n_total,seed", [(500, 1), (2000, 3)])
def test_fp64_raster_identical_first_200ms(n_total, seed):
    o = oracle.OracleSim(n_total=n_total, seed=seed, pre_ms=100, sim_ms=100, raster_steps=2000)
    with asg.Simulation(n_total=n_total, seed=seed, pre_ms=100, sim_ms=100, raster_steps=2000) as sim:
        sim.step(2000)
        o.step(2000)
        r_gpu, r_cpu = sim.raster(), o.raster()
        assert r_cpu.sum() > 0
        diff = np.nonzero((r_gpu != r_cpu).any(axis=1))[0]
        assert diff.size == 0, f"raster differs first at step {diff[0]}"
        s1, s2 = sim.summary(), o.summary()
        for k in ("spikes_total", "spikes_measured", "active_astro", "engaged_astro"):
            assert s1[k] == s2[k], k


def test_fp64_full_config0_summary():
    """The reference's small CPU-sized case: N=500, seed 1, 1000 ms pre-run + 5000 ms recorded."""
    o = oracle.OracleSim(n_total=500, seed=1)
    with asg.Simulation(n_total=500, seed=1) as sim:
        total = sim.summary()["total_steps"]
        sim.step(total)
        o.step(total)
        a, b = sim.summary(), o.summary()
    assert a["total_steps"] == 60000
    assert abs(a["mean_rate_hz"] - b["mean_rate_hz"]) <= 0.02 * b["mean_rate_hz"]
    assert abs(a["active_astro"] - b["active_astro"]) / a["n_astro"] <= 0.02
    assert abs(a["engaged_astro"] - b["engaged_astro"]) / a["n_astro"] <= 0.02
    print("config0 gpu", {k: a[k] for k in ("spikes_measured", "mean_rate_hz", "mean_ca", "active_astro",
                                            "engaged_astro")})
    print("config0 oracle", {k: b[k] for k in ("spikes_measured", "mean_rate_hz", "mean_ca", "active_astro",
                                               "engaged_astro")})


def test_fp32_raster_first_50ms_matches_fp64_oracle():
    o = oracle.OracleSim(n_total=500, seed=1, pre_ms=20, sim_ms=30, raster_steps=500)
    with asg.Simulation(n_total=500, seed=1, pre_ms=20, sim_ms=30, raster_steps=500, precision="fp32") as sim:
        sim.step(500)
        o.step(500)
        r_gpu, r_cpu = sim.raster(), o.raster()
        assert r_cpu.sum() > 0
        diff = np.nonzero((r_gpu != r_cpu).any(axis=1))[0]
        assert diff.size == 0, f"fp32 raster differs first at step {diff[0]}"


def test_fp32_summary_within_tolerance_of_fp64_oracle():
    kw = dict(n_total=20000, seed=7, pre_ms=200, sim_ms=1000)
    o = oracle.OracleSim(**kw)
    with asg.Simulation(precision="fp32", **kw) as sim:
        total = sim.summary()["total_steps"]
        sim.step(total)
        o.step(total)
        a, b = sim.summary(), o.summary()
    assert abs(a["mean_rate_hz"] - b["mean_rate_hz"]) <= 0.02 * b["mean_rate_hz"], (a["mean_rate_hz"],
                                                                                    b["mean_rate_hz"])
    assert abs(a["active_astro"] - b["active_astro"]) / a["n_astro"] <= 0.02
    print("fp32 vs fp64 oracle rate", a["mean_rate_hz"], b["mean_rate_hz"], "active", a["active_astro"],
          b["active_astro"])


def test_stp_off_and_weight_overrides_match_oracle():
    kw = dict(n_total=800, seed=11, pre_ms=10, sim_ms=40, raster_steps=500, stp_enabled=0, w_a2n=0.0, w_n2a=0.5)
    o = oracle.OracleSim(**kw)
    with asg.Simulation(**kw) as sim:
        sim.step(500)
        o.step(500)
        np.testing.assert_array_equal(sim.raster(), o.raster())
        assert_state_close(sim, o, "no-stp")


def test_substeps_and_dt_variants_match_oracle():
    for kw in (dict(substeps=3), dict(dt=0.05), dict(dt=0.25)):
        args = dict(n_total=600, seed=2, pre_ms=5, sim_ms=20, **kw)
        o = oracle.OracleSim(**args)
        with asg.Simulation(**args) as sim:
            n = sim.summary()["total_steps"]
            sim.step(n)
            o.step(n)
            assert_state_close(sim, o, str(kw))
            np.testing.assert_array_equal(sim.spike_counts(), o.spike_counts())


def test_step_past_configured_length_and_zero_steps():
    with asg.Simulation(n_total=300, seed=1, pre_ms=1, sim_ms=1) as sim:
        sim.step(0)
        sim.step(50)
        s = sim.summary()
        assert s["steps_done"] == 50 and s["total_steps"] == 20
        with pytest.raises(asg.AstrosimError):
            sim.step(-1)
        with pytest.raises(asg.AstrosimError):
            sim.spike_counts(0, 51)
