#!/usr/bin/env python3
"""Records the reference program's own summaries on a GPU, as dynamics golden data.

Runs the unmodified reference binaries built by ``make -C oracle ref`` from the
reference's source file (oracle/_ref/astrosim_fused_ref, FP64, and
oracle/_ref/astrosim_fused_ref_f32, the -DASTROSIM_USE_FLOAT build) for a set of
short configurations and parses the lines the reference prints at the end of a
run (src/astrosim_fused.cu:1131-1141).  Needs a CUDA device; writes JSON.

Usage:  python tests/golden/make_reference_dynamics_golden.py --out reference_dynamics.json
        (--min-n / --max-n select cases; --merge FILE keeps FILE's other records)
"""
import argparse
import json
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
BIN = {"fp64": os.path.join(REPO, "oracle", "_ref", "astrosim_fused_ref"),
       "fp32": os.path.join(REPO, "oracle", "_ref", "astrosim_fused_ref_f32")}

CASES = [("fp64", 500, 1, 0, t) for t in (1, 5, 10, 20, 50, 100, 200, 500)] + [
    ("fp64", 500, 1, 1000, 5000),
    ("fp64", 5000, 2, 0, 100),
    ("fp64", 2000, 3, 50, 150),
    ("fp64", 1000000, 7, 200, 1000),
    ("fp64", 10000000, 1, 100, 500),
    ("fp32", 500, 1, 1000, 5000),
    ("fp32", 1000000, 7, 200, 1000),
]


def parse(out):
    def grab(pat, cast=float):
        m = re.search(pat, out)
        return cast(m.group(1)) if m else None
    return {
        "connectivity": grab(r"(connectivity: exc=\d+ inh=\d+ e2a=\d+ sic=\d+) edges", str),
        "build_s": grab(r"edges, built in ([0-9.]+) s"),
        "wall_s": grab(r"wall time\s+: ([0-9.]+) s"),
        "us_per_step": grab(r"\(([0-9.]+) us/step"),
        "spikes_measured": grab(r"spikes \(recorded win\): (\d+)", int),
        "mean_rate_hz": grab(r"mean firing rate\s+: ([0-9.]+) Hz"),
        "mean_ca_str": grab(r"mean calcium \(final\) : (\S+) uM", str),
        "active_astro": grab(r"astrocytes active\s+: (\d+) /", int),
        "engaged_astro": grab(r"astrocytes engaged\s+: (\d+) /", int),
        "windowed_hz": [float(x) for x in re.findall(r"windowed rate: ([0-9.]+) Hz", out)],
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--max-n", type=int, default=10**7)
    ap.add_argument("--min-n", type=int, default=0)
    ap.add_argument("--merge", default=None, help="existing golden file: keep its other records")
    args = ap.parse_args()
    res = json.load(open(args.merge)) if args.merge else []
    for prec, n, seed, pre, sim in CASES:
        if n > args.max_n or n < args.min_n:
            continue
        cmd = [BIN[prec], "--n", str(n), "--seed", str(seed), "--pre-ms", str(pre), "--sim-ms", str(sim)]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
        rec = {"precision": prec, "n_total": n, "seed": seed, "pre_ms": pre, "sim_ms": sim,
               "returncode": r.returncode, **parse(r.stdout)}
        key = (prec, n, seed, pre, sim)
        res = [x for x in res if (x["precision"], x["n_total"], x["seed"], x["pre_ms"], x["sim_ms"]) != key]
        res.append(rec)
        print(json.dumps(rec), flush=True)
    with open(args.out, "w") as f:
        json.dump(res, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
