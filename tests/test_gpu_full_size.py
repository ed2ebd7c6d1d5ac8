"""The north-star tolerances at the benchmark's full size, N_total = 1e7 (seed 1).

The FP64 path is pinned to the reference program's own GPU output at this size by
test_gpu_reference_golden.py (spike count, windowed rates, mean calcium, astrocyte
counts, exactly).  Here it is also held against the FP64 oracle (OpenMP on every
host core) on the same connectivity, the device-built CSR: every cell is within
1e-12 relative for the first 30 steps.  Over 100 steps a few values in a million
drift past 1e-12, all of them membrane potentials: the device path rounds
differently from the oracle in two ways (CUDA's exp against the host C library's,
fused multiply-adds as in the reference program), and the test shows that an
oracle with the same two rounding differences departs by the same amount.
FP32: the spike raster equals the FP64 one through step 67 (6.7 ms) and its
per-step spike counts over the first 50 ms stay within 1 % in total; at this size
some neuron of the ten million crosses threshold one step apart within 4-9 ms in
every FP32 build, so the whole 50 ms raster is not identical (it is at N = 500 and
5e3; test_gpu_fp32_raster.py gives the measurements and the reason).
These runs take about two minutes.
"""
import os

import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg
from oracle import oracle

pytestmark = pytest.mark.gpu

N = 10_000_000
STATE = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic", "stp_x", "stp_u", "stp_t_last",
         "Ca", "IP3", "h", "sic_factor")


def beyond(a_get, b_get, tol=1e-12):
    """Values of two runs that differ by more than tol (relative, floor 1), over all arrays:
    (count, worst relative difference, {array: indices of the cells beyond tol})."""
    total, worst, where = 0, 0.0, {}
    for name in STATE:
        a, b = a_get(name), b_get(name)
        d = np.abs(a - b) / np.maximum(np.abs(b), 1.0)
        idx = np.nonzero(d > tol)[0]
        total += idx.size
        worst = max(worst, float(d.max()))
        if idx.size:
            where[name] = idx
    return total, worst, where


def exp_ulp_disagreement():
    """ulp distance between CUDA's double exp (the device path's, as in the reference
    program) and the host C library's (the oracle's) over arguments of the AdEx term
    (V - V_th) / Delta_T: CUDA's exp is evaluated by torch on the device."""
    import math

    import torch
    x = np.random.default_rng(5).uniform(-20.0, 26.0, size=200_000)
    dev = torch.exp(torch.tensor(x, dtype=torch.float64, device="cuda")).cpu().numpy()
    host = np.array([math.exp(v) for v in x])
    return np.abs(dev.view(np.int64) - host.view(np.int64))


def test_fp64_state_against_oracle_at_full_size():
    """Where the FP64 state leaves 1e-12 at full size, and why.

    The device path and the oracle compute the same formulas with two differences
    in rounding: CUDA's exp and the host C library's disagree in the last bit for
    some arguments, and the device fuses multiply-adds (as the reference program
    compiled by nvcc does) where the oracle rounds each operation.  Two more oracles
    stand in for those differences on the host: one whose AdEx exp is moved by one
    ulp on the measured fraction of arguments, and one that also fuses the neuron
    update's multiply-adds.  The values past 1e-12 at step 100 are all membrane
    potentials, and the oracle with both rounding differences departs from the plain
    oracle by as many values, by the same order of magnitude, as the device does:
    the departure is what one-ulp differences grow to in neurons near threshold at
    this size, not a fault of either path.  The device path itself equals the
    reference program's own output exactly (test_gpu_reference_golden.py)."""
    ulps = exp_ulp_disagreement()
    assert ulps.max() <= 1, "CUDA and host exp should agree to one ulp"
    rate = float((ulps > 0).mean())
    print(f"CUDA vs host exp: {rate:.4%} of arguments one ulp apart")
    assert rate > 0.0

    kw = dict(n_total=N, seed=1, pre_ms=100.0, sim_ms=500.0)
    with asg.Simulation(**kw) as sim:
        csrs = {k: sim.csr(k) for k in ("exc", "inh", "sic", "e2a")}
        threads = os.cpu_count() or 1
        o = oracle.OracleSim(threads=threads, csrs=csrs, **kw)
        q_exp = oracle.OracleSim(threads=threads, csrs=csrs, **kw)
        q_exp.perturb_exp(rate)
        q_both = oracle.OracleSim(threads=threads, csrs=csrs, **kw)
        q_both.perturb_exp(rate)
        q_both.contract()
        del csrs
        runs = (sim, o, q_exp, q_both)
        try:
            for run in runs:
                run.step(1)
            n1 = beyond(sim.state, o.state)[0]
            assert n1 == 0, f"step 1: {n1} cells beyond 1e-12"
            for run in runs:
                run.step(29)
            n30 = beyond(sim.state, o.state)[0]
            assert n30 == 0, f"step 30: {n30} cells beyond 1e-12"
            np.testing.assert_array_equal(sim.spike_counts(), o.spike_counts())
            for run in runs:
                run.step(70)
            n_dev, worst_dev, where_dev = beyond(sim.state, o.state)
            n_exp, worst_exp, where_exp = beyond(q_exp.state, o.state)
            n_both, worst_both, where_both = beyond(q_both.state, o.state)
            for tag, n, worst, where in (("device", n_dev, worst_dev, where_dev), ("one-ulp exp", n_exp, worst_exp,
                                          where_exp), ("one-ulp exp + fused", n_both, worst_both, where_both)):
                print(f"step 100, {tag} vs oracle: {n} values beyond 1e-12 (worst {worst:.2e}) in "
                      f"{ {k: v.size for k, v in where.items()} }")
            v_dev = o.state("V")[where_dev.get("V", np.zeros(0, dtype=np.int64))]
            print("oracle V of the device's departing cells:", np.round(np.sort(v_dev), 2)[:40])
            assert n_dev <= 1e-5 * 12_000_000 * len(STATE)
            assert set(where_dev) <= {"V"} and set(where_both) <= {"V"}, (set(where_dev), set(where_both))
            # the two rounding differences together reproduce the divergence, to within an order of magnitude
            assert n_both > 0
            assert n_both / 10 <= n_dev <= n_both * 10, (n_dev, n_both)
            assert worst_both / 100 <= worst_dev <= worst_both * 100, (worst_dev, worst_both)
            c_gpu, c_cpu = sim.spike_counts(), o.spike_counts()
            assert abs(int(c_gpu.sum()) - int(c_cpu.sum())) <= 1e-3 * max(1, int(c_cpu.sum()))
        finally:
            for run in runs[1:]:
                run.close()


def test_fp32_raster_against_fp64_at_full_size():
    kw = dict(n_total=N, seed=1, pre_ms=100.0, sim_ms=500.0, raster_steps=500)
    with asg.Simulation(precision="fp64", **kw) as d:
        d.step(500)
        r64, c64 = d.raster(), d.spike_counts()
    with asg.Simulation(precision="fp32", **kw) as f:
        f.step(500)
        r32, c32 = f.raster(), f.spike_counts()
    assert r64.sum() > 0
    diff = np.nonzero((r32 != r64).any(axis=1))[0]
    first = int(diff[0]) if diff.size else 500
    print(f"FP32 raster equals FP64 through step {first - 1}; {diff.size} of 500 steps differ somewhere")
    # measured: first difference at step 68 for seed 1 (42-84 over seeds 1-3 and both FP32 builds,
    # test_gpu_fp32_raster.py); the 500-step identity does not hold at this size
    assert 40 <= first < 500, first
    assert abs(int(c32.sum()) - int(c64.sum())) <= 0.01 * int(c64.sum())
