"""The warp swarms' chunk-table bookkeeping against plain walks, on the host (no GPU).

tests/swarm_tables_check.cpp models a warp's lanes in lockstep (claims in a random
order each round, refill, hand-off, continuation, resolve) over random tapes shaped
like the builder's three sections, and checks every candidate's resolved exit and
pre count against a plain walk from it.  The GPU tests compare the device kernels
with the one-CTA tables and the reference's connectivity (test_gpu_builder.py)."""
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_swarm_tables_equal_plain_walks(tmp_path):
    exe = tmp_path / "swarm_tables_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), os.path.join(HERE, "swarm_tables_check.cpp")],
                   check=True)
    r = subprocess.run([str(exe), "6"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"candidates (\d+) mismatches (\d+)", r.stdout)
    assert m and int(m.group(1)) == 6 * (384 + 192 + 192 + 384 + 192 + 192) and int(m.group(2)) == 0
