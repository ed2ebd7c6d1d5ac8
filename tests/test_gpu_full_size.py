"""The north-star tolerances at the benchmark's full size, N_total = 1e7 (seed 1).

The FP64 path is pinned to the reference program's own GPU output at this size by
test_gpu_reference_golden.py (spike count, windowed rates, mean calcium, astrocyte
counts, exactly).  Here it is also held against the FP64 oracle (OpenMP on every
host core) on the same connectivity, the device-built CSR: every cell is within
1e-12 relative for the first 30 steps.  Over 100 steps a few values in a million
drift past 1e-12: the oracle evaluates exp with the host C library and the device
path with CUDA's (as the reference program does), and the test shows that a
one-ulp exp difference on the measured fraction of arguments, alone, produces the
same divergence.
FP32: the spike raster equals the FP64 one for the first 5 ms (50 steps) and its
per-step spike counts over the first 50 ms stay within 1 % in total; at this size
some neuron of the ten million crosses threshold one step apart within about 7 ms,
so the whole 50 ms raster is not identical (it is at N = 500, test_gpu_parity.py).
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

    The device path and the oracle compute the same operations, except that CUDA's
    exp and the host C library's disagree in the last bit for some arguments (and
    the device fuses some multiply-adds, as the reference program compiled by nvcc
    does).  A second oracle whose AdEx exp is moved by one ulp on the same fraction
    of arguments stands in for that disagreement alone: it departs from the plain
    oracle by the same number of values, by the same order of magnitude, as the
    device does.  So the values past 1e-12 at step 100 are what a one-ulp exp
    difference grows to at this size, not a fault of either path; the device path
    itself equals the reference program's own output exactly
    (test_gpu_reference_golden.py)."""
    ulps = exp_ulp_disagreement()
    assert ulps.max() <= 1, "CUDA and host exp should agree to one ulp"
    rate = float((ulps > 0).mean())
    print(f"CUDA vs host exp: {rate:.4%} of arguments one ulp apart")
    assert rate > 0.0

    kw = dict(n_total=N, seed=1, pre_ms=100.0, sim_ms=500.0)
    with asg.Simulation(**kw) as sim:
        csrs = {k: sim.csr(k) for k in ("exc", "inh", "sic", "e2a")}
        o = oracle.OracleSim(threads=os.cpu_count() or 1, csrs=csrs, **kw)
        q = oracle.OracleSim(threads=os.cpu_count() or 1, csrs=csrs, **kw)
        q.perturb_exp(rate)
        del csrs
        try:
            for run in (sim, o, q):
                run.step(1)
            n1 = beyond(sim.state, o.state)[0]
            assert n1 == 0, f"step 1: {n1} cells beyond 1e-12"
            for run in (sim, o, q):
                run.step(29)
            n30 = beyond(sim.state, o.state)[0]
            assert n30 == 0, f"step 30: {n30} cells beyond 1e-12"
            np.testing.assert_array_equal(sim.spike_counts(), o.spike_counts())
            for run in (sim, o, q):
                run.step(70)
            n_dev, worst_dev, where_dev = beyond(sim.state, o.state)
            n_exp, worst_exp, where_exp = beyond(q.state, o.state)
            print(f"step 100, device vs oracle: {n_dev} values beyond 1e-12 (worst {worst_dev:.2e}) in "
                  f"{ {k: v.size for k, v in where_dev.items()} }")
            print(f"step 100, one-ulp exp oracle vs oracle: {n_exp} values beyond 1e-12 (worst {worst_exp:.2e}) in "
                  f"{ {k: v.size for k, v in where_exp.items()} }")
            assert n_dev <= 1e-5 * 12_000_000 * len(STATE)
            # the one-ulp exp difference alone reproduces the divergence, to within an order of magnitude
            assert n_exp > 0
            assert n_exp / 10 <= n_dev <= n_exp * 10, (n_dev, n_exp)
            assert worst_exp / 100 <= worst_dev <= worst_exp * 100, (worst_dev, worst_exp)
            c_gpu, c_cpu = sim.spike_counts(), o.spike_counts()
            assert abs(int(c_gpu.sum()) - int(c_cpu.sum())) <= 1e-3 * max(1, int(c_cpu.sum()))
        finally:
            o.close()
            q.close()


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
    assert first >= 50
    assert abs(int(c32.sum()) - int(c64.sum())) <= 0.01 * int(c64.sum())
