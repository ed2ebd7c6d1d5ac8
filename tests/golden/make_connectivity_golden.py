#!/usr/bin/env python3
"""Generates the connectivity golden fixtures from the reference program itself.

Runs the unmodified reference binary (built by ``make -C oracle ref`` from the
reference's own source file into ``oracle/_ref/astrosim_fused_ref``) with
``--dump-edges``, which builds the network with the reference's host code
(src/astrosim_fused.cu:631-735) and writes it as CSV (src/astrosim_fused.cu:873-902)
without touching a GPU.  The CSV rows come out target by target in CSR order, so
the four target-keyed CSRs are recovered exactly and recorded as:

  connectivity.json      per (n_total, seed): edge counts and the SHA-256 of each
                         CSR's row_start and src arrays (little-endian uint32)
  csr_n{N}_s{S}.npz      the full CSRs for a few small networks

Usage:  python tests/golden/make_connectivity_golden.py [--big]
(--big adds N=1e6 seed 7, whose dump is about 3 GB and takes a minute.)
"""
import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pyarrow.csv as pacsv

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(REPO, "oracle", "_ref", "astrosim_fused_ref")

SMALL_N = [1, 2, 3, 4, 5, 8, 10, 13, 20, 30, 50, 64, 80, 99, 100, 101, 102, 103, 104, 105,
           110, 125, 150, 200, 333, 500, 1000, 2000, 5000, 10000, 50000, 100000]
SEEDS = [1, 2, 7]
FULL = [(500, 1), (100, 2)]


def scaling(n_total):
    """src/astrosim_fused.cu:606-614 (lround = round half away from zero)."""
    def lround(x):
        return int(np.floor(x + 0.5)) if x >= 0 else -int(np.floor(-x + 0.5))
    n_exc = max(1, lround(n_total * 0.8))
    n_inh = max(1, n_total - n_exc)
    n_astro = max(1, lround(n_total / 5.0))
    return n_exc, n_inh, n_astro


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def dump_to_csrs(n_total, seed, tmpdir):
    path = os.path.join(tmpdir, f"e_{n_total}_{seed}.csv")
    out = subprocess.run([REF_BIN, "--n", str(n_total), "--seed", str(seed), "--dump-edges", path],
                         check=True, capture_output=True, text=True).stdout
    line = [l for l in out.splitlines() if l.startswith("connectivity:")][0]
    counts = {}
    for tok in line.split(":", 1)[1].split("edges")[0].split():
        k, v = tok.split("=")
        counts[k] = int(v)
    tbl = pacsv.read_csv(path, convert_options=pacsv.ConvertOptions(
        column_types={"type": pa.string(), "source": pa.string(), "target": pa.string()}))
    os.remove(path)
    n_exc, n_inh, n_astro = scaling(n_total)
    n_neurons = n_exc + n_inh
    src_col, tgt_col = tbl.column("source"), tbl.column("target")
    blocks = [("exc", counts["exc"], n_neurons, 0, False, False),
              ("inh", counts["inh"], n_neurons, n_exc, False, False),
              ("e2a", counts["e2a"], n_astro, 0, False, True),
              ("sic", counts["sic"], n_neurons, 0, True, False)]
    csrs, start = {}, 0
    for name, n_edges, n_targets, src_off, src_a, tgt_a in blocks:
        s = src_col.slice(start, n_edges)
        t = tgt_col.slice(start, n_edges)
        start += n_edges
        if src_a:
            s = pc.utf8_slice_codeunits(s, 1)
        if tgt_a:
            t = pc.utf8_slice_codeunits(t, 1)
        s = pc.cast(s, pa.int64()).to_numpy() - src_off
        t = pc.cast(t, pa.int64()).to_numpy()
        assert np.all(np.diff(t) >= 0), "dump rows are not target-ordered"
        rs = np.zeros(n_targets + 1, dtype=np.int64)
        np.cumsum(np.bincount(t, minlength=n_targets), out=rs[1:])
        csrs[name] = (rs.astype(np.uint32), s.astype(np.uint32))
    assert start == tbl.num_rows
    return counts, csrs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true")
    args = ap.parse_args()
    if not os.path.exists(REF_BIN):
        sys.exit(f"missing {REF_BIN}: run `make -C oracle ref` first")
    out_json = os.path.join(HERE, "connectivity.json")
    golden = json.load(open(out_json)) if os.path.exists(out_json) else {}
    cases = [(n, s) for n in SMALL_N for s in SEEDS]
    if args.big:
        cases.append((1000000, 7))
    with tempfile.TemporaryDirectory() as td:
        for n, s in cases:
            counts, csrs = dump_to_csrs(n, s, td)
            golden[f"{n}:{s}"] = {
                "n_total": n, "seed": s,
                "edges": {k: int(csrs[k][1].size) for k in csrs},
                "sha256": {k: {"row_start": sha(csrs[k][0]), "src": sha(csrs[k][1])} for k in csrs},
            }
            if (n, s) in FULL:
                np.savez_compressed(os.path.join(HERE, f"csr_n{n}_s{s}.npz"),
                                    **{f"{k}_{p}": csrs[k][i] for k in csrs for i, p in enumerate(("rs", "src"))})
            print(n, s, golden[f"{n}:{s}"]["edges"], flush=True)
    with open(out_json, "w") as f:
        json.dump(dict(sorted(golden.items(), key=lambda kv: (kv[1]["n_total"], kv[1]["seed"]))), f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
