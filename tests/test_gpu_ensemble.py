"""The batched ensemble steps many uneven networks in shared launches (window
kernel over a tile table, CUDA-graph replay) and every network's result is
bit-identical to running it alone through astrosim_create/astrosim_step."""
import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg
from astrosimgpu_cuda_b200 import abi

pytestmark = pytest.mark.gpu

STATES = ("V", "w", "g_ex", "g_in", "I_sic", "stp_x", "Ca", "IP3", "h", "sic_factor")


def configs(precision, rng):
    sizes = [500, 800, 1500, 3000, 6000, 12000, 25000]
    cfgs = []
    for i, n in enumerate(sizes):
        cfgs.append(abi.default_config(
            n_total=n, seed=100 + i, pre_ms=20.0, sim_ms=(80.0 if i != 2 else 50.0), precision=precision,
            neuron_drive_scale=float(rng.uniform(0.8, 1.2)), w_a2n=float(rng.uniform(0.8, 1.2))))
    return cfgs


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_ensemble_matches_solo_runs(precision):
    cfgs = configs(precision, np.random.default_rng(3))
    with asg.Ensemble(cfgs) as ens:
        assert len(ens) == 7
        assert ens.shared_constants()  # only seeds, sizes, drive rates and w_a2n differ
        ens.step(500)
        ens.step(500)  # 1000 steps = 100 windows: tuning windows, graph replays and a remainder
        got = []
        for i in range(len(ens)):
            s = ens.summary(i)
            got.append(({k: ens.state(i, k) for k in STATES}, ens.spike_counts(i), s))
    for i, cfg in enumerate(cfgs):
        with asg.Simulation(cfg) as sim:
            total = sim.summary()["total_steps"]
            sim.step(total)
            states, counts, s = got[i]
            assert s["steps_done"] == total
            np.testing.assert_array_equal(counts, sim.spike_counts())
            for k in STATES:
                np.testing.assert_array_equal(states[k], sim.state(k), err_msg=f"net {i} {k}")
            solo = sim.summary()
            for k in ("spikes_total", "spikes_measured", "mean_ca", "active_astro", "engaged_astro"):
                assert s[k] == solo[k], (i, k)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_ensemble_with_differing_constants_matches_solo_runs(precision):
    """Networks whose biology differs beyond the per-network scalars take the
    staged-constants window kernel; their results are still each solo run's."""
    cfgs = [abi.default_config(n_total=n, seed=40 + i, pre_ms=10.0, sim_ms=60.0, precision=precision)
            for i, n in enumerate((900, 2500, 1700))]
    bios = [None, {"stp_U": 0.3, "SIC_th": 0.18}, {"exc_poiss_rate": 3100.0}]
    with asg.Ensemble(cfgs, biology=bios) as ens:
        assert not ens.shared_constants()
        ens.step(700)
        got = [({k: ens.state(i, k) for k in STATES}, ens.spike_counts(i)) for i in range(3)]
    for i, (c, b) in enumerate(zip(cfgs, bios)):
        with asg.Simulation(c, biology=b) as sim:
            sim.step(700)
            np.testing.assert_array_equal(got[i][1], sim.spike_counts())
            for k in STATES:
                np.testing.assert_array_equal(got[i][0][k], sim.state(k), err_msg=f"net {i} {k}")


def test_ensemble_shares_constants_when_only_scalars_differ():
    cfgs = [abi.default_config(n_total=n, seed=60 + i, pre_ms=0.0, sim_ms=20.0, precision="fp32")
            for i, n in enumerate((700, 1400))]
    with asg.Ensemble(cfgs, biology=[None, {"exc_poiss_rate": 3100.0, "inh_poiss_rate": 3100.0}]) as ens:
        assert ens.shared_constants()  # the rates enter only through the per-network drive scalars


def test_ensemble_rejects_mixed_precision_and_partial_windows():
    a = abi.default_config(n_total=500, seed=1, pre_ms=0, sim_ms=10)
    b = abi.default_config(n_total=500, seed=2, pre_ms=0, sim_ms=10, precision="fp32")
    with pytest.raises(asg.AstrosimError):
        asg.Ensemble([a, b])
    with asg.Ensemble([a, a]) as ens:
        with pytest.raises(asg.AstrosimError):
            ens.step(7)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_every_tile_shape_is_bit_identical(monkeypatch, precision):
    """The autotuner picks a (tile size, occupancy) pair: tiles of 64, 128 or 256 cells
    with three launch-bounds targets each.  Every pair gives each network the result
    of running it alone."""
    cfgs = [abi.default_config(n_total=n, seed=70 + i, pre_ms=5.0, sim_ms=35.0, precision=precision)
            for i, n in enumerate((700, 3300, 9000))]
    solo = []
    for cfg in cfgs:
        with asg.Simulation(cfg) as sim:
            sim.step(sim.summary()["total_steps"])
            solo.append(({k: sim.state(k) for k in STATES}, sim.spike_counts()))
    for v in range(9):
        monkeypatch.setenv("ASTROSIM_ENSEMBLE_VARIANT", str(v))
        with asg.Ensemble(cfgs) as ens:
            ens.step(400)
            for i in range(len(cfgs)):
                np.testing.assert_array_equal(ens.spike_counts(i), solo[i][1], err_msg=f"variant {v} net {i}")
                for k in STATES:
                    np.testing.assert_array_equal(ens.state(i, k), solo[i][0][k], err_msg=f"variant {v} net {i} {k}")
    monkeypatch.delenv("ASTROSIM_ENSEMBLE_VARIANT")
