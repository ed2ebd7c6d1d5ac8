"""The builder's re-merge walk against its plain walk, on the host (no GPU).

tests/walk_equivalence.cpp includes the device walk code (csrc/walk_chunked.cuh)
with host stand-ins for the two device intrinsics it uses and compares the walks'
end positions and error flags over random skip caches; the device tests then pin
the plain walk's output to the reference's connectivity (test_gpu_builder.py)."""
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_remerge_walk_draws_what_the_plain_walk_draws(tmp_path):
    exe = tmp_path / "walk_equivalence"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), os.path.join(HERE, "walk_equivalence.cpp")],
                   check=True)
    r = subprocess.run([str(exe), "2000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"walks (\d+) mismatches (\d+) cache_overruns (\d+)", r.stdout)
    assert m and int(m.group(1)) == 80000 and int(m.group(2)) == 0
    assert int(m.group(3)) > 0  # walks that run off the cache are compared too
