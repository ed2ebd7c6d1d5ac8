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


@pytest.mark.parametrize("n_total,builder", [(20000, None), (3000, "sequential")])
def test_each_rank_keeps_only_its_own_rows(monkeypatch, n_total, builder):
    """A rank builds and keeps the connectivity rows of its own cells only (the chunked
    builder emits just those edges; the one-thread walk for small networks slices its
    CSRs), about 1 / world of the network; every kept row is the whole network's row,
    and the summary still reports the whole network's edge counts."""
    if builder:
        monkeypatch.setenv("ASTROSIM_BUILDER", builder)
    world = 3
    kw = dict(n_total=n_total, seed=11, pre_ms=0.0, sim_ms=1.0)
    with shard.ShardGroup(world=world, **kw) as g, asg.Simulation(**kw) as s:
        for name in ("exc", "inh", "sic", "e2a"):
            rs_full, src_full = s.csr(name)
            held = 0
            next_row = 0
            for r in range(world):
                first, rs, src = g.csr(r, name)
                plan = shard.shard_plan(n_total, r, world)
                assert first == (plan[2] if name == "e2a" else plan[0])
                assert first == next_row
                lo, hi = first, first + rs.size - 1
                next_row = hi
                np.testing.assert_array_equal(rs, rs_full[lo:hi + 1] - rs_full[lo], err_msg=f"{name} rank {r}")
                np.testing.assert_array_equal(src, src_full[rs_full[lo]:rs_full[hi]], err_msg=f"{name} rank {r}")
                held += src.size
                # a rank's share of the edges follows its share of the cells (128-cell blocks)
                share = (hi - lo) / (rs_full.size - 1)
                assert src.size <= 1.25 * share * src_full.size + 64, (name, r, src.size, src_full.size, share)
            assert next_row == rs_full.size - 1
            assert held == src_full.size
        a, b = g.summary(), s.summary()
        for k in ("n_exc_edges", "n_inh_edges", "n_e2a_edges", "n_sic_edges"):
            assert a[k] == b[k], k


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


def test_group_at_full_size_keeps_half_the_rows_each():
    """N_total = 1e7 split over two ranks (both on this GPU, one after another): each
    rank keeps about half of the 1.32e9 connectivity rows, and 20 windows give the
    single-GPU run's results bit for bit."""
    kw = dict(n_total=10_000_000, seed=1, pre_ms=0.0, sim_ms=20.0, precision="fp32")
    with asg.Simulation(**kw) as s:
        s.step(200)
        want = {name: s.state(name) for name in ("V", "w", "g_ex", "Ca", "IP3", "h", "sic_factor")}
        want_counts = s.spike_counts()
        want_summary = s.summary()
    with shard.ShardGroup(world=2, **kw) as g:
        held = []
        for r in range(2):
            held.append(sum(g.csr(r, name)[2].size for name in ("exc", "inh", "sic", "e2a")))
        total = sum(want_summary[k] for k in ("n_exc_edges", "n_inh_edges", "n_e2a_edges", "n_sic_edges"))
        assert sum(held) == total
        for h in held:
            assert abs(h - total / 2) <= 0.02 * total, (h, total)
        g.step(200)
        np.testing.assert_array_equal(g.spike_counts(), want_counts)
        for name, v in want.items():
            np.testing.assert_array_equal(g.state(name), v, err_msg=name)
        assert want_counts.sum() > 0
