"""The CLI keeps the reference's flags and printed lines (src/astrosim_fused.cu:853-871, 1131-1141)."""
import os
import re
import subprocess

import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg

pytestmark = pytest.mark.gpu


def run_cli(*args):
    r = subprocess.run([asg.CLI_PATH, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout


def test_cli_summary_lines_match_library():
    out = run_cli("--n", "500", "--seed", "1", "--pre-ms", "20", "--sim-ms", "100")
    assert "connectivity: exc=40073 inh=9957 e2a=8019 sic=8019 edges" in out
    assert re.search(r"wall time\s+: [0-9.]+ s for 1200 steps \([0-9.]+ us/step", out)
    spikes = int(re.search(r"spikes \(recorded win\): (\d+)", out).group(1))
    rate = float(re.search(r"mean firing rate\s+: ([0-9.]+) Hz", out).group(1))
    with asg.Simulation(n_total=500, seed=1, pre_ms=20, sim_ms=100) as sim:
        sim.step(1200)
        s = sim.summary()
    assert spikes == s["spikes_measured"]
    assert abs(rate - s["mean_rate_hz"]) < 1e-4
    assert len(re.findall(r"windowed rate: [0-9.]+ Hz", out)) == 9


def test_cli_dump_edges_round_trips(tmp_path, golden_connectivity):
    import hashlib
    path = tmp_path / "e.csv"
    run_cli("--n", "500", "--seed", "1", "--dump-edges", str(path))
    rows = path.read_text().splitlines()
    assert rows[0] == "type,source,target"
    rec = golden_connectivity["500:1"]
    exc = [r for r in rows[1:] if r.startswith("exc_primary,")]
    assert len(exc) == rec["edges"]["exc"]
    src = np.array([int(r.split(",")[1]) for r in exc], dtype="<u4")
    assert hashlib.sha256(src.tobytes()).hexdigest() == rec["sha256"]["exc"]["src"]
    a2n = [r for r in rows[1:] if r.startswith("a2n,")]
    assert all(r.split(",")[1].startswith("A") for r in a2n)
    inh = [int(r.split(",")[1]) for r in rows[1:] if r.startswith("inh_primary,")]
    assert min(inh) >= 400  # inhibitory sources are printed with the +n_exc offset


def test_cli_fp32_runs():
    out = run_cli("--n", "1000", "--pre-ms", "0", "--sim-ms", "20", "--precision", "fp32")
    assert "precision=float" in out and "mean firing rate" in out
