"""astrosim_astro_totals_noalloc, the summary reduction that allocates nothing.

It exists for callers that cannot allocate device memory where they need the
totals (their memory is all handed to their own pool or a fixed budget, or they
must not enter the CUDA allocator, whose cudaMalloc/cudaFree may synchronize the
device).  This test calls it through the C ABI on device arrays the caller owns
and checks that two calls in a row give the same totals as astrosim_summary,
which reduces the same state with cudaMalloc'd scratch.  The tolerance is exact:
both run the same fixed-order reduction on the same values.
"""
import ctypes as C

import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg
from astrosimgpu_cuda_b200 import abi

pytestmark = pytest.mark.gpu

NOALLOC_MAX_ASTRO = 8388608


class Totals(C.Structure):
    _fields_ = [("sum_ca", C.c_double), ("mean_ca", C.c_double), ("active", C.c_uint32), ("engaged", C.c_uint32)]


def entry():
    L = asg.lib()
    f = L.astrosim_astro_totals_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return L, f


def test_noalloc_totals_match_summary_twice():
    import torch

    L, f = entry()
    # N=500, seed 1, 1000 ms pre-run + 5000 ms recorded: 5 astrocytes end above the
    # SIC threshold and 8 cross it during the recorded window.  The engaged flags
    # are rebuilt on the host from the SIC factor after every recorded step.
    with asg.Simulation(n_total=500, seed=1, pre_ms=1000, sim_ms=5000) as sim:
        s0 = sim.summary()
        pre, total = s0["pre_steps"], s0["total_steps"]
        sim.step(pre)
        engaged = np.zeros(sim.n_astro, dtype=np.uint8)
        for _ in range(total - pre):
            sim.step(1)
            engaged |= (sim.state("sic_factor") > 0).astype(np.uint8)
        s = sim.summary()
        ca = sim.state("Ca")
        n_astro = sim.n_astro
    assert int(engaged.sum()) == s["engaged_astro"] > 0
    assert s["active_astro"] > 0

    d_ca = torch.tensor(ca, dtype=torch.float64, device="cuda")
    d_eng = torch.tensor(engaged, dtype=torch.uint8, device="cuda")
    d_out = torch.empty(C.sizeof(Totals), dtype=torch.uint8, device="cuda")
    for _ in range(2):
        d_out.fill_(0xAB)  # stale bytes must not survive into the result
        torch.cuda.synchronize()
        rc = f(d_ca.data_ptr(), d_eng.data_ptr(), n_astro, s["sic_th"], d_out.data_ptr(), None)
        assert rc == abi.OK, L.astrosim_last_error()
        torch.cuda.synchronize()
        t = Totals.from_buffer_copy(bytes(d_out.cpu().numpy()))
        assert t.mean_ca == s["mean_ca"]
        assert t.sum_ca == pytest.approx(float(ca.sum()), rel=1e-13)
        assert t.active == s["active_astro"]
        assert t.engaged == s["engaged_astro"]


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    L, f = entry()
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = f(d.data_ptr(), d.data_ptr(), NOALLOC_MAX_ASTRO + 1, 0.2, d.data_ptr(), None)
    assert rc == abi.ERR_INVALID_ARG
    assert b"ASTROSIM_NOALLOC_MAX_ASTRO" in L.astrosim_last_error()


@pytest.mark.parametrize("n_astro", [0, 1, 2049, 2048 * 37 + 1, 2048 * 4095 + 1, NOALLOC_MAX_ASTRO])
def test_noalloc_totals_match_host_counts(n_astro):
    """Random device data at sizes that cover the empty input, one and many partial
    blocks, a last block with one astrocyte, and the full capacity of the scratch.
    Counts must equal the host's exactly; the calcium sum agrees with an exactly
    rounded host sum to 1e-13 relative (the device adds in a fixed tree order)."""
    import math

    import torch

    L, f = entry()
    rng = np.random.default_rng(n_astro + 11)
    sic_th = 0.19669
    ca = rng.uniform(0.0, 0.4, size=n_astro)
    engaged = (rng.integers(0, 4, size=n_astro) * 85).astype(np.uint8)  # 0, 85, 170, 255
    want_active = int(np.count_nonzero((ca - sic_th) * 1000.0 > 1.0))
    want_engaged = int(np.count_nonzero(engaged))
    want_sum = math.fsum(ca.tolist()) if n_astro else 0.0

    d_ca = torch.tensor(ca, dtype=torch.float64, device="cuda") if n_astro else torch.zeros(1, dtype=torch.float64,
                                                                                           device="cuda")
    d_eng = torch.tensor(engaged, dtype=torch.uint8, device="cuda") if n_astro else torch.zeros(1, dtype=torch.uint8,
                                                                                               device="cuda")
    d_out = torch.empty(C.sizeof(Totals), dtype=torch.uint8, device="cuda")
    results = []
    for _ in range(2):
        d_out.fill_(0xAB)
        torch.cuda.synchronize()
        rc = f(d_ca.data_ptr(), d_eng.data_ptr(), n_astro, sic_th, d_out.data_ptr(), None)
        assert rc == abi.OK, L.astrosim_last_error()
        torch.cuda.synchronize()
        t = Totals.from_buffer_copy(bytes(d_out.cpu().numpy()))
        assert t.active == want_active
        assert t.engaged == want_engaged
        if n_astro:
            assert t.sum_ca == pytest.approx(want_sum, rel=1e-13)
            assert t.mean_ca == t.sum_ca / n_astro
        else:
            assert t.sum_ca == 0.0 and t.mean_ca == 0.0
        results.append((t.sum_ca, t.mean_ca, t.active, t.engaged))
    assert results[0] == results[1]  # same fixed order, bit-identical on repeat
