"""Serving: requests admitted by HBM footprint, built while the batch runs, joined
and retired between windows (continuous batching).  Each result is the same alone
and in the mix: exactly equal summaries (same arithmetic, shared launches)."""
import time

import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg
from astrosimgpu_cuda_b200 import abi

pytestmark = pytest.mark.gpu

KEYS = ("steps_done", "spikes_total", "spikes_measured", "mean_rate_hz", "mean_ca", "active_astro", "engaged_astro",
        "n_exc_edges", "n_e2a_edges")


def request_configs(precision, n, rng):
    cfgs = []
    for i in range(n):
        cfgs.append(abi.default_config(
            n_total=int(np.exp(rng.uniform(np.log(500), np.log(20000)))), seed=int(rng.integers(1, 1 << 30)),
            pre_ms=float(rng.choice([0.0, 10.0])), sim_ms=float(rng.integers(2, 12) * 10.0), precision=precision,
            neuron_drive_scale=float(rng.uniform(0.8, 1.2))))
    return cfgs


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_results_same_alone_and_in_the_mix(precision):
    rng = np.random.default_rng(11 if precision == "fp32" else 12)
    cfgs = request_configs(precision, 12, rng)
    # a budget for about three requests at a time forces queueing and slot reuse
    budget = 3 * int(max(c.n_total for c in cfgs) * 3200 + (64 << 20))
    results, max_running, queued = {}, 0, 0
    with asg.Server(precision=precision, budget_bytes=budget, builders=4) as srv:
        ids = [srv.submit(c) for c in cfgs[:6]]
        pumps = 0
        while len(results) < len(cfgs):
            srv.pump(5)
            pumps += 1
            if pumps == 3:
                ids += [srv.submit(c) for c in cfgs[6:]]  # arrivals while others are on the GPU
            st = srv.stats()
            max_running = max(max_running, st["running"])
            for i, rid in enumerate(ids):
                if i not in results:
                    r = srv.result(rid)
                    if r is not None:
                        results[i] = r
                        queued += r["queue_s"] > 0.0
            assert pumps < 20000
            if st["running"] == 0 and st["building"] > 0:
                time.sleep(0.001)
        assert srv.stats()["done"] == len(cfgs)
    assert max_running >= 2
    for i, cfg in enumerate(cfgs):
        with asg.Simulation(cfg) as sim:
            sim.step(sim.summary()["total_steps"])
            solo = sim.summary()
        for k in KEYS:
            assert results[i][k] == solo[k], (i, k, results[i][k], solo[k])


def test_server_rejects_requests_it_cannot_hold():
    with asg.Server(precision="fp32", budget_bytes=200 << 20, builders=1) as srv:
        with pytest.raises(asg.AstrosimError):
            srv.submit(abi.default_config(n_total=5_000_000, precision="fp32"))
        with pytest.raises(asg.AstrosimError):
            srv.submit(abi.default_config(n_total=500, precision="fp64"))
