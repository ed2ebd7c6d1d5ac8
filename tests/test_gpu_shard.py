"""One network split across ranks, against the single-GPU run.

The in-process group (astrosim_shard_group_*) runs every rank on this GPU, one
after another, with the same exchange a multi-GPU run does: each window the ranks
advance their own cells, all-gather the window's spikes and active SIC factors,
and deliver into their own cells.  Everything must be bit-identical to the
unsharded run: every state array, every per-step spike count, the raster and the
summary.  Cases cover 2 and 3 ranks, both precisions, ranks without astrocytes,
busy windows (pull delivery) and non-default biology.  The one-rank-per-process
path (astrosim_shard_*) is exercised with a world of one.
"""
import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg
from astrosimgpu_cuda_b200 import abi, shard

pytestmark = pytest.mark.gpu

STATES = [n for n in abi.STATE]


def compare(sharded, single, tag):
    for name in STATES:
        np.testing.assert_array_equal(sharded.state(name), single.state(name), err_msg=f"{tag} {name}")
    np.testing.assert_array_equal(sharded.spike_counts(), single.spike_counts(), err_msg=f"{tag} counts")
    a, b = sharded.summary(), single.summary()
    for k in ("spikes_total", "spikes_measured", "mean_rate_hz", "mean_ca", "active_astro", "engaged_astro",
              "steps_done"):
        assert a[k] == b[k], (tag, k, a[k], b[k])


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n_total", [500, 6000])
def test_group_matches_single_gpu(world, precision, n_total):
    kw = dict(n_total=n_total, seed=9, pre_ms=5.0, sim_ms=45.0, precision=precision)
    with shard.ShardGroup(world=world, **kw) as g, asg.Simulation(**kw) as s:
        for chunk in (10, 90, 400):
            g.step(chunk)
            s.step(chunk)
            compare(g, s, f"w{world} {precision} N{n_total} after {chunk}")


def test_group_busy_windows_and_raster():
    # a strong drive makes most windows busy (pull delivery) early on
    bio = {"exc_poiss_rate": 27000.0, "inh_poiss_rate": 25000.0}
    kw = dict(n_total=4000, seed=3, pre_ms=0.0, sim_ms=30.0, raster_steps=300)
    with shard.ShardGroup(world=3, biology=bio, **kw) as g, asg.Simulation(biology=bio, **kw) as s:
        g.step(300)
        s.step(300)
        per_window = s.spike_counts().reshape(-1, 10).sum(axis=1)
        assert (per_window > 1024).sum() >= 3, "expected busy windows (over the 1024-spike push limit)"
        compare(g, s, "busy")


def test_group_with_long_delays_and_biology():
    bio = {"d_e": 1.5, "d_i": 1.5, "d_a2n": 1.5, "sic_interval": 3, "noise_dt": 0.5, "w_n2a": 0.6}
    kw = dict(n_total=3000, seed=5, pre_ms=3.0, sim_ms=57.0)
    with shard.ShardGroup(world=2, biology=bio, **kw) as g, asg.Simulation(biology=bio, **kw) as s:
        g.step(600)
        s.step(600)
        compare(g, s, "delays")


def test_group_rejects_partial_windows_and_per_step_engine():
    with shard.ShardGroup(world=2, n_total=1000, seed=1, pre_ms=0.0, sim_ms=10.0) as g:
        with pytest.raises(asg.AstrosimError):
            g.step(15)
    with pytest.raises(asg.AstrosimError):
        shard.ShardGroup(world=2, n_total=1000, seed=1, biology={"d_i": 0.7})


def test_one_rank_per_process_world_of_one(tmp_path):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"file://{tmp_path}/pg", rank=0, world_size=1)
    try:
        kw = dict(n_total=3000, seed=4, pre_ms=5.0, sim_ms=45.0, precision="fp32")
        with shard.ShardedSimulation(**kw) as r, asg.Simulation(**kw) as s:
            r.step(500)
            s.step(500)
            compare(r, s, "rank")
            assert r.last_step_ms() > 0
    finally:
        dist.destroy_process_group()
