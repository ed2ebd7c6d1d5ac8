"""CPU checks of the FP64 oracle (oracle/astrosim_oracle.cpp) against the
reference's own outputs: the golden connectivity fixtures come from the reference
binary's --dump-edges path (tests/golden/make_connectivity_golden.py)."""
import hashlib

import numpy as np
import pytest

from oracle import oracle

MASK = (1 << 64) - 1


def splitmix(seed, stream, counter):
    """Pure-Python restatement of src/astrosim_fused.cu:127-135."""
    z = (seed + stream * 0x9E3779B97F4A7C15 + counter * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


@pytest.mark.parametrize("seed,stream,counter", [(1, 0x5EED, 0), (7, 0x5EED, 123456789), (2**63 + 5, 3, 2**40),
                                                 (1 ^ 0xC2B2AE3D27D4EB4F, 1000003 * 17 + 5, 2)])
def test_rng_bits_matches_restatement(seed, stream, counter):
    assert oracle.rng_bits(seed, stream, counter) == splitmix(seed, stream, counter)
    assert oracle.rng_uniform(seed, stream, counter) == (splitmix(seed, stream, counter) >> 11) * 2.0 ** -53


def test_poisson_counts_follow_knuth():
    lam = 2700 * 0.1 * 1e-3
    lim = np.exp(-lam)
    for stream in range(200):
        c, prod = 0, oracle.rng_uniform(99, stream, 0)
        k = 0
        while prod > lim:
            k += 1
            c += 1
            prod *= oracle.rng_uniform(99, stream, c)
        assert oracle.rng_poisson(99, stream, lam) == k


def test_seq_normals_pairs_share_uniforms():
    z = oracle.seq_normals(3, 0x5EED, 6)
    u1, u2 = oracle.rng_uniform(3, 0x5EED, 0), oracle.rng_uniform(3, 0x5EED, 1)
    r, th = np.sqrt(-2 * np.log(u1)), 2 * np.pi * u2
    assert z[0] == pytest.approx(r * np.cos(th), rel=1e-15)
    assert z[1] == pytest.approx(r * np.sin(th), rel=1e-15)


def test_oracle_connectivity_matches_reference_golden(golden_connectivity):
    checked = 0
    for rec in golden_connectivity.values():
        if rec["n_total"] > 100000:
            continue
        s = oracle.OracleSim(n_total=rec["n_total"], seed=rec["seed"], pre_ms=0, sim_ms=0)
        for k in ("exc", "inh", "sic", "e2a"):
            rs, src = s.csr(k)
            assert src.size == rec["edges"][k], (rec["n_total"], rec["seed"], k)
            assert sha(rs) == rec["sha256"][k]["row_start"], (rec["n_total"], rec["seed"], k)
            assert sha(src) == rec["sha256"][k]["src"], (rec["n_total"], rec["seed"], k)
        s.close()
        checked += 1
    assert checked >= 90


def test_oracle_full_csr_n500(golden_connectivity):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "csr_n500_s1.npz"))
    s = oracle.OracleSim(n_total=500, seed=1)
    for k in ("exc", "inh", "sic", "e2a"):
        rs, src = s.csr(k)
        np.testing.assert_array_equal(rs, z[f"{k}_rs"])
        np.testing.assert_array_equal(src, z[f"{k}_src"])
    # row invariants: exc/inh rows ascending (one edge per pre/post pair)
    rs, src = s.csr("exc")
    for t in range(500):
        row = src[rs[t]:rs[t + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0)
        assert t not in row  # no autapses


def test_oracle_parameters_in_bounds():
    s = oracle.OracleSim(n_total=2000, seed=4)
    ca_tot = s.state("Ca_tot")
    assert np.all(ca_tot >= 1.8958264782990153 * 0.9) and np.all(ca_tot <= 1.8958264782990153 * 1.05)
    vr = s.state("V_reset")
    assert np.all(vr[:1600] >= -55.0) and np.all(vr[:1600] <= -45.0)
    assert np.all(vr[1600:] >= -66.0) and np.all(vr[1600:] <= -54.0)


def test_oracle_deterministic_and_thread_independent():
    a = oracle.OracleSim(n_total=500, seed=1, pre_ms=5, sim_ms=20, threads=1)
    b = oracle.OracleSim(n_total=500, seed=1, pre_ms=5, sim_ms=20, threads=4)
    a.step(250)
    b.step(250)
    for name in ("V", "w", "Ca", "IP3", "g_ex", "I_sic"):
        np.testing.assert_array_equal(a.state(name), b.state(name))
    sa, sb = a.summary(), b.summary()
    for k in ("build_seconds", "run_seconds"):
        sa.pop(k), sb.pop(k)
    assert sa == sb


def test_oracle_pre_run_zero_quirk():
    # With pre_ms = 0 the reference reads its counter after step 0 and clears the
    # engaged flags there (src/astrosim_fused.cu:1066), so step 0's spikes are not recorded.
    s = oracle.OracleSim(n_total=500, seed=1, pre_ms=0, sim_ms=30)
    s.step(300)
    c = s.spike_counts()
    sm = s.summary()
    assert sm["spikes_measured"] == int(c[1:].sum())
    assert sm["spikes_total"] == int(c.sum())
