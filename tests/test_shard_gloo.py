"""Host side of the one-rank-per-process sharded network, on CPU with gloo
(world size 2): the ownership plans partition the cells, all ranks must describe
the same network, a failure on any rank stops every rank before the NCCL
communicator is joined, and rank 0's id reaches every rank.  No GPU is used; the
NCCL id is a stand-in made by the test.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, queue):
    import torch.distributed as dist

    from astrosimgpu_cuda_b200 import abi, shard
    os.environ["CUDA_VISIBLE_DEVICES"] = ""
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    out = {}
    try:
        # 1. the plans of all ranks partition the neurons and the astrocytes, in 128-cell blocks
        plans = [None] * world
        dist.all_gather_object(plans, shard.shard_plan(1_000_003, rank, world))
        out["plans"] = plans
        # 2. identical descriptions pass; a different seed on one rank fails on every rank
        cfg = abi.default_config(n_total=5000, seed=7)
        shard.agree_on_config(cfg, {"w_e": 4.0})
        bad = abi.default_config(n_total=5000, seed=7 + rank)
        try:
            shard.agree_on_config(bad, None)
            out["mismatch"] = "accepted"
        except ValueError as e:
            out["mismatch"] = str(e)
        # 3. one rank's failure reaches all ranks
        try:
            shard.all_ranks_ok(rank != 1, "rank one failed")
            out["ok"] = "passed"
        except RuntimeError as e:
            out["ok"] = str(e)
        # 4. rank 0's id on every rank
        out["id"] = shard.share_id(make_id=lambda: bytes(range(128)))
        # 5. without a GPU, creation fails on every rank before any communicator exists
        try:
            shard.ShardedSimulation(n_total=1000, seed=1)
            out["create"] = "created"
        except RuntimeError as e:
            out["create"] = str(e)
    finally:
        dist.destroy_process_group()
    queue.put((rank, out))


def test_sharded_host_logic_with_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(queue.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        out = results[r]
        plans = out["plans"]
        assert plans[0][0] == 0 and plans[0][2] == 0
        for a, b in zip(plans, plans[1:]):
            assert a[1] == b[0] and a[3] == b[2]
            assert a[1] % 128 == 0 and a[3] % 128 == 0
        from astrosimgpu_cuda_b200 import abi
        n_exc, n_inh, n_astro, _ = abi.scaling(1_000_003)
        assert plans[-1][1] == n_exc + n_inh and plans[-1][3] == n_astro
        sizes = [p[1] - p[0] for p in plans]
        assert max(sizes) - min(sizes) <= 128
        assert "different network: seed" in out["mismatch"]
        assert "rank 1: rank one failed" in out["ok"]
        assert out["id"] == bytes(range(128))
        assert "no CUDA device" in out["create"] and "rank 0" in out["create"] and "rank 1" in out["create"]
