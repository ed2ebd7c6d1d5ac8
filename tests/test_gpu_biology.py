"""Non-default biology on the GPU against the FP64 oracle given the same overrides.

The override sets exercise code paths the defaults leave idle: a refractory
period (t_ref > 0), SIC refresh every 3 steps, neuron noise every 5 steps,
facilitating STP (tau_fac > 0), Delta_T values that are not powers of two (the
exact constant division), longer equal delays (a 15-step window) and unequal
delays (the per-step engine).  Tolerances as in test_gpu_parity: FP64 state
within 1e-12 relative over the first 100 steps and an identical raster; the
batched and served forms must give the solo run's results bit for bit.
"""
import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg
from oracle import oracle

pytestmark = pytest.mark.gpu

STATE = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic", "stp_x", "stp_u", "stp_t_last",
         "Ca", "IP3", "h", "sic_factor")

CASES = {
    "refractory_interval_noise": {"e_t_ref": 0.5, "i_t_ref": 0.3, "sic_interval": 3, "noise_dt": 0.5,
                                  "stp_U": 0.4, "stp_tau_fac": 120.0, "exc_poiss_rate": 3300.0, "w_e": 6.0,
                                  "e_Delta_T": 2.5, "i_Delta_T": 1.5, "tau_IP3": 900.0, "i_C_m": 110.0},
    "long_equal_delays": {"d_e": 1.5, "d_i": 1.5, "d_a2n": 1.5, "astro_noise_std": 0.001, "w_n2a": 0.5},
    "unequal_delays": {"d_e": 1.0, "d_i": 0.7, "d_a2n": 2.0, "SIC_th": 0.15},
}


def assert_state_close(sim, o, tag):
    for name in STATE:
        a, b = sim.state(name), o.state(name)
        bad = np.abs(a - b) > 1e-12 * np.maximum(np.abs(b), 1.0)
        assert not bad.any(), f"{tag} {name}: {bad.sum()} cells, max |d| {np.max(np.abs(a - b)):.3e}"


@pytest.mark.parametrize("case", sorted(CASES))
def test_fp64_matches_oracle_with_overrides(case):
    bio = CASES[case]
    kw = dict(n_total=2000, seed=11, pre_ms=5.0, sim_ms=195.0, raster_steps=2000)
    o = oracle.OracleSim(biology=bio, **kw)
    with asg.Simulation(biology=bio, **kw) as sim:
        done = 0
        for chunk in (7, 33, 60):
            sim.step(chunk)
            o.step(chunk)
            done += chunk
            assert_state_close(sim, o, f"{case} step {done}")
        sim.step(1900)
        o.step(1900)
        r_gpu, r_cpu = sim.raster(), o.raster()
        assert r_cpu.sum() > 0
        diff = np.nonzero((r_gpu != r_cpu).any(axis=1))[0]
        assert diff.size == 0, f"{case}: raster differs first at step {diff[0]}"
        a, b = sim.summary(), o.summary()
        for k in ("spikes_total", "spikes_measured", "active_astro", "engaged_astro"):
            assert a[k] == b[k], (case, k)


def test_overrides_change_the_run_and_cfg_fields_apply_on_top():
    kw = dict(n_total=1000, seed=3, pre_ms=0.0, sim_ms=50.0)
    with asg.Simulation(**kw) as a, asg.Simulation(biology={"exc_poiss_rate": 5400.0}, **kw) as b, \
            asg.Simulation(biology={"exc_poiss_rate": 5400.0, "inh_poiss_rate": 5000.0}, neuron_drive_scale=0.5,
                           **kw) as c, \
            asg.Simulation(biology={"exc_poiss_rate": 2700.0}, **kw) as d:
        for s in (a, b, c, d):
            s.step(500)
        assert b.summary()["spikes_total"] > a.summary()["spikes_total"]
        # drive scale 0.5 applied after doubled rates gives the default rates back exactly
        np.testing.assert_array_equal(c.state("V"), a.state("V"))
        np.testing.assert_array_equal(d.state("V"), a.state("V"))


def test_ensemble_and_server_apply_per_network_overrides():
    from astrosimgpu_cuda_b200 import abi
    cfgs = [abi.default_config(n_total=n, seed=20 + i, pre_ms=0.0, sim_ms=100.0, precision="fp32")
            for i, n in enumerate((1200, 3000, 800))]
    bios = [{"exc_poiss_rate": 3100.0}, None, {"stp_U": 0.3, "sic_interval": 2}]
    with asg.Ensemble(cfgs, biology=bios) as ens:
        ens.step(1000)
        got = [ens.summary(i) for i in range(3)]
    with asg.Server(precision="fp32", builders=2) as srv:
        ids = [srv.submit(c, biology=b) for c, b in zip(cfgs, bios)]
        while srv.stats()["done"] < 3:
            srv.pump(10)
        served = [srv.result(r) for r in ids]
    for i, (c, b) in enumerate(zip(cfgs, bios)):
        with asg.Simulation(c, biology=b) as sim:
            sim.step(1000)
            want = sim.summary()
        for k in ("spikes_total", "spikes_measured", "mean_ca", "active_astro", "engaged_astro"):
            assert got[i][k] == want[k], (i, k)
            assert served[i][k] == want[k], (i, k)
