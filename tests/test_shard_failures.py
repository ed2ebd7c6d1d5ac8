"""Failure handling of a sharded network, on CPU (no GPU is faulted, hung or used).

Every wait a rank makes on the others has a deadline (include/astrosim.h,
astrosim_shard_set_timeout): the exchange of each 1 ms window, the set-up of the
communicator and the gathers behind summary/get_state.  The deadline logic is
driven here through astrosim_shard_selftest_wait, which runs it against a stand-in
communicator: a rank that never completes an exchange (it died, or left between
windows) makes the wait return ASTROSIM_ERR_TIMEOUT within the deadline and abort
the communicator; a peer failure the communicator reports returns
ASTROSIM_ERR_PEER at once.  The host plumbing (torch.distributed, gloo, world
size 2) is checked the same way: a rank that leaves between windows makes the
other rank's next collective raise after the process group's short timeout
instead of waiting for ever.
"""
import datetime
import os
import socket
import time

import pytest
import torch.multiprocessing as mp

from astrosimgpu_cuda_b200 import abi, shard


@pytest.mark.parametrize("scenario,code,windows,aborted", [
    (0, abi.OK, 4, False),           # every exchange completes
    (1, abi.ERR_TIMEOUT, 0, True),   # the first exchange never completes
    (2, abi.ERR_PEER, 0, True),      # the communicator reports a failed peer
    (3, abi.ERR_TIMEOUT, 2, True),   # a rank left after window 1
])
def test_bounded_wait_on_stand_in_comm(scenario, code, windows, aborted):
    timeout = 0.25
    t0 = time.perf_counter()
    rc, done, was_aborted, waited = shard.selftest_wait(scenario, timeout)
    wall = time.perf_counter() - t0
    assert rc == code
    assert done == windows
    assert was_aborted == aborted
    if code == abi.ERR_TIMEOUT:
        assert timeout <= waited < timeout + 0.5  # the deadline fired, and soon after it passed
        assert b"no progress within" in shard._lib().astrosim_last_error()
    elif code == abi.ERR_PEER:
        assert waited < timeout  # reported by the communicator, before the deadline
        assert b"failure" in shard._lib().astrosim_last_error()
    else:
        assert waited < timeout
    assert wall < 5.0


def test_selftest_rejects_bad_arguments():
    assert shard.selftest_wait(7, 1.0)[0] == abi.ERR_INVALID_ARG
    assert shard.selftest_wait(0, 0.0)[0] == abi.ERR_INVALID_ARG


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, queue):
    import torch.distributed as dist

    os.environ["CUDA_VISIBLE_DEVICES"] = ""
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=4))
    out = {}
    # window 0: both ranks take part in the host-side agreement
    out["w0"] = shard.all_ranks_ok(True, "")
    if rank == 1:
        queue.put((rank, {"left": True}))
        queue.close()
        queue.join_thread()  # the result is sent before the process vanishes
        os._exit(0)  # leaves between windows, with nothing in flight
    t0 = time.perf_counter()
    try:
        shard.all_ranks_ok(True, "")  # window 1: rank 1 is gone
        out["w1"] = "completed"
    except Exception as e:  # gloo reports the closed peer or the timeout
        out["w1"] = type(e).__name__
    out["seconds"] = time.perf_counter() - t0
    queue.put((rank, out))
    queue.close()
    queue.join_thread()
    os._exit(0)


def test_rank_that_leaves_between_windows_stops_the_other():
    world = 2
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert results[1] == {"left": True}
    r0 = results[0]
    assert r0["w0"] is True
    assert r0["w1"] != "completed"
    assert r0["seconds"] < 30.0
