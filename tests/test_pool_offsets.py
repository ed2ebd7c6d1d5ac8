"""The builder's pool-offset scan against a sequential walk of the pools, on the host
(no GPU).  tests/pool_offsets_check.cpp draws the pools with the model's counter RNG
and compares the scan's per-post offsets with the sequential ones; the device tests
then pin the built connectivity to the reference's (test_gpu_builder.py)."""
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_pool_offset_scan_matches_the_sequential_pools(tmp_path):
    exe = tmp_path / "pool_offsets_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), os.path.join(HERE, "pool_offsets_check.cpp")],
                   check=True)
    r = subprocess.run([str(exe), "200"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"trials (\d+) mismatches (\d+) redrawing_posts (\d+)", r.stdout)
    assert m and int(m.group(1)) == 200 and int(m.group(2)) == 0
    assert int(m.group(3)) > 1000  # the scan had redraws to find
