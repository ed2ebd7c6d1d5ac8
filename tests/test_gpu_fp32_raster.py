"""How long the FP32 form keeps the FP64 spike raster, and why it cannot keep it
for 50 ms in large networks.

The FP32 form runs the RK4 stages in float (V, w, Ca and IP3 accumulate in double,
and the threshold test runs in double).  Its rounding, about 1e-7 of each stage
value, reaches the membrane potential; in a neuron that is running away towards
threshold the AdEx exponential amplifies it, and with enough spikes one of them
falls a step earlier or later than in FP64.  Measured first differing step, from
t = 0 (seeds 1, 2, 3; 1000 steps):

    N_total   FP32 (product)   IEEE FP32 build    FP64, constants moved 1 ulp
    5e3       329, 561, -      -, 561, -          -
    1e5       78, 212, 290     291, 212, 190      -
    1e6       89, 78, 95       160, 147, 132      -
    1e7       63, 48, 42       84, 48, 57         -

So the 50 ms (500-step) identity holds at N = 500 (test_gpu_parity.py) and for
two of three seeds at N = 5e3, and not from N = 1e5 on.  The IEEE build
(lib/libastrosim_b200_fp32ieee.so: CUDA's correctly rounded float functions and
divisions, the term-by-term formulas and 53-bit noise uniforms instead of the
hardware approximations and the refolded formulas) moves the first difference
only a little, so neither the approximations nor the refolding are the cause:
float stages are.  FP64 with constants moved by one ulp keeps
the raster for 100 ms at every size, so the flips are FP32's precision, not a
sensitivity any correct FP64 arithmetic would show.  The statistics the FP32 form
is held to instead (mean rate and SIC-threshold fraction within 2 % / 0.02 of FP64)
are checked at the C2 configuration below and at N = 1e7 in bench.py (seeds 1-3).
"""
import json
import math
import os
import subprocess
import sys

import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def raster(n, seed, steps, precision, biology=None):
    with asg.Simulation(n_total=n, seed=seed, pre_ms=0.0, sim_ms=steps * 0.1, precision=precision,
                        raster_steps=steps, biology=biology) as sim:
        sim.step(steps)
        return sim.raster()


def first_diff(a, b):
    d = np.nonzero(np.any(a != b, axis=1))[0]
    return int(d[0]) if d.size else None


def test_small_network_keeps_the_raster_for_tens_of_ms():
    """N_total = 5e3: the raster holds at least 30 ms for seeds 1-3 (measured 32.9,
    56.1 and over 100 ms), against 4-9 ms at N_total = 1e7."""
    firsts = {}
    for seed in (1, 2, 3):
        firsts[seed] = first_diff(raster(5000, seed, 1000, "fp64"), raster(5000, seed, 1000, "fp32"))
    print("N=5e3 FP32 first differing step, seeds 1-3:", firsts)
    for seed, f in firsts.items():
        assert f is None or f >= 300, (seed, f)


def test_fp64_with_one_ulp_constants_keeps_the_raster_at_full_size():
    base = raster(10_000_000, 1, 1000, "fp64")
    bio = {"e_C_m": math.nextafter(130.0, math.inf), "i_C_m": math.nextafter(104.0, math.inf)}
    moved = raster(10_000_000, 1, 1000, "fp64", biology=bio)
    assert first_diff(base, moved) is None


def test_c2_configuration_fp32_against_fp64():
    """N_total = 1e6, seed 7, 200 ms pre-run + 1000 ms recorded: the raster over the
    first 50 ms differs (as measured for seeds 1-3 at this size); the mean rate and
    the SIC-threshold fraction are within 2 % and 0.02 of FP64."""
    kw = dict(n_total=1_000_000, seed=7, pre_ms=200.0, sim_ms=1000.0, raster_steps=500)
    out = {}
    for prec in ("fp64", "fp32"):
        with asg.Simulation(precision=prec, **kw) as sim:
            sim.step(sim.summary()["total_steps"])
            s = sim.summary()
            out[prec] = (sim.raster(), s["mean_rate_hz"], s["active_astro"] / s["n_astro"])
    f = first_diff(out["fp64"][0], out["fp32"][0])
    print(f"C2 FP32 raster equals FP64 through step {None if f is None else f - 1}; "
          f"rate {out['fp32'][1]:.5f} vs {out['fp64'][1]:.5f} Hz, SIC fraction {out['fp32'][2]:.5f} vs "
          f"{out['fp64'][2]:.5f}")
    assert out["fp64"][0].sum() > 0
    assert f is not None and 30 <= f < 500, f
    assert abs(out["fp32"][1] - out["fp64"][1]) <= 0.02 * out["fp64"][1]
    assert abs(out["fp32"][2] - out["fp64"][2]) <= 0.02


IEEE_SCRIPT = r"""
import json, sys
import numpy as np
import astrosimgpu_cuda_b200 as asg
res = {}
for seed in (1, 2, 3):
    r = {}
    for prec in ("fp64", "fp32"):
        with asg.Simulation(n_total=1_000_000, seed=seed, pre_ms=0.0, sim_ms=100.0, precision=prec,
                            raster_steps=1000) as sim:
            sim.step(1000)
            r[prec] = sim.raster()
    d = np.nonzero(np.any(r["fp64"] != r["fp32"], axis=1))[0]
    res[seed] = int(d[0]) if d.size else None
print(json.dumps(res))
"""


def test_ieee_float_build_does_not_keep_the_raster_either():
    """The measurement build with IEEE float functions, divisions and 53-bit noise
    uniforms also leaves the FP64 raster within 50 ms at N_total = 1e6."""
    lib = os.path.join(REPO, "astrosimgpu_cuda_b200", "lib", "libastrosim_b200_fp32ieee.so")
    env = dict(os.environ, ASTROSIM_LIBRARY=lib, PYTHONPATH=REPO)
    r = subprocess.run([sys.executable, "-c", IEEE_SCRIPT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    firsts = json.loads(r.stdout.strip().splitlines()[-1])
    print("IEEE FP32 build, first differing step at N=1e6, seeds 1-3:", firsts)
    for seed, f in firsts.items():
        assert f is not None and f < 500, (seed, f)
