#!/usr/bin/env python3
"""Benchmark of the tripartite network simulator on B200.

Workload (the N=1e7 configuration): one network of N_total = 1e7 (8M excitatory,
2M inhibitory AdEx neurons, 2M Li-Rinzel astrocytes, about 1.32e9 synapses),
seed 1, dt = 0.1 ms, built on the device from (N, seed) exactly as the reference
builds it.  One bench step = one network time step (dt).  `value` is net-steps/s
of the FP32 form (FP64 accumulators) with the network resident in HBM; the plain
FP64 path is measured beside it under "fp64".  `e2e` is the whole job through the
C ABI: astrosim_create (device build) + the 100 ms pre-run and 500 ms recorded
window (6000 steps) + astrosim_summary, timed on the host wall clock.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun with N > 1 every rank simulates its own replica network (seed 1 +
rank); value = all ranks' net-steps / max-over-ranks device time.
`--impl reference` runs the reference program itself (built from its own source
for sm_100a into oracle/_ref) on the same configuration.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "net-steps/s & syn-events/s at N=1e7 FP32 vs FP64; ensemble sims/s, p50/p99"
N_TOTAL = 10_000_000
SEED = 1
DT = 0.1
PRE_MS, SIM_MS = 100.0, 500.0


# One steady-state window_kernel launch measured by ncu (profiles/), at
# N_total = 3e6, where the state streamed per launch is several times the L2:
# DRAM bytes read + written, warp instructions issued and the fraction of issue
# slots busy.  Bytes and instructions grow with the cell count, so a launch at N
# carries about N / 3e6 times these.
PROFILED_WINDOW = {
    "fp32": {"n": 3_000_000, "dram": 353.47e6, "warp_inst": 376.78e6, "issue_busy": 0.844},
    "fp64": {"n": 3_000_000, "dram": 506.90e6, "warp_inst": 838.86e6, "issue_busy": 0.736},
}
PROFILED_SOURCE = "ncu, one steady-state window_kernel launch at N_total=3e6 (profiles/), scaled to N_total"
SCHEDULERS_PER_SM = 4  # warp schedulers per B200 SM: one warp instruction each per cycle at most


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                     f[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
        finally:
            try:
                os.remove(self.path)
            except OSError:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def dist_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def gather_step_bytes(s, precision):
    """Bytes one time step moves in the reference's per-step gather formulation.

    Every CSR source id is read once per step (4 B per edge visit, the a2n rows on
    every refresh step) and every cell's state is read and written once: neurons
    124 B (FP64) / 72 B (FP32), astrocytes 92 B / 48 B, plus one spike bit per neuron.
    """
    e_visit = s["n_exc_edges"] + s["n_inh_edges"] + s["n_e2a_edges"] + s["n_sic_edges"]
    nn = s["n_exc"] + s["n_inh"]
    sn, sa = (124, 92) if precision == "fp64" else (72, 48)
    return 4 * e_visit + nn * sn + s["n_astro"] * sa + nn / 8, e_visit


def window_step_bytes(s, precision, spikes_per_step, window=10):
    """Algorithmic bytes per time step of the windowed engine (one launch per window).

    Per window each neuron reads V, w, V_reset, b (32 B), five conductance/SIC
    values, its refractory counter and inbox count (8 B) and its a2n flag bit, and
    writes V, w, the five values, the counter and its spike word; a neuron whose a2n
    row holds an active astrocyte also reads the row (8 B of row_start + 4 B per
    entry; estimated from the active astrocytes at the last step times their a2n
    fan-out).  Each astrocyte reads Ca, IP3, h, four parameters, its inbox count and
    flag, and writes Ca, IP3, h, `window` SIC factors, its flag and last factor.
    Each spike delivers one deposit (key, step, value: 12 B FP32 / 16 B FP64, plus a
    4 B count update) per outgoing edge.
    """
    r = 8 if precision == "fp64" else 4
    nn = s["n_exc"] + s["n_inh"]
    na = s["n_astro"]
    a2n_fanout = s["n_sic_edges"] / max(1, na)
    flagged = min(nn, s.get("active_astro", 0) * a2n_fanout)
    row = s["n_sic_edges"] / max(1, nn)
    neuron = nn * (32 + 5 * r + 8 + 1 / 8 + 16 + 5 * r + 8) + flagged * (8 + 4 * row)
    astro = na * (16 + r + 32 + 5 + 16 + r + window * r + 1 + r)
    fanout = (s["n_exc_edges"] + s["n_inh_edges"] + s["n_e2a_edges"]) / max(1, nn)
    deposits = spikes_per_step * window * fanout * ((16 if r == 8 else 12) + 4)
    return (neuron + astro + deposits) / window


def sm_count(device):
    try:
        import torch
        return torch.cuda.get_device_properties(device).multi_processor_count
    except Exception:
        return 148


def roofline(leg, prec, achieved, peak, peak_kind, ms_step, device):
    """The window kernel's roofline: HBM bytes against the measured copy bandwidth,
    and, since the kernel is bound by instruction issue, warp instructions issued
    against one per scheduler per cycle at the SM clock sampled during the run."""
    prof = PROFILED_WINDOW[prec]
    scale = N_TOTAL / prof["n"]
    out = {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "traffic": prof["dram"] * scale if prof["dram"] else None,
           "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum, " + PROFILED_SOURCE,
           "peak_source": peak_kind,
           "kernel": f"window_kernel<{'float' if prec == 'fp32' else 'double'}> (one launch = one 10-step window, "
                     f"its push_kernel inside the timed duration)",
           "algorithmic_bytes_per_step": leg["bytes"],
           "gather_formulation_bytes_per_step": leg["gather_bytes"],
           "gather_formulation_equivalent_gbs": leg["gather_bytes"] / (ms_step * 1e-3) / 1e9}
    mhz = (leg.get("clocks") or {}).get("sm_mhz")
    if prof["warp_inst"] and mhz:
        inst_per_step = prof["warp_inst"] * scale / 10
        achieved_ips = inst_per_step / (ms_step * 1e-3)
        peak_ips = sm_count(device) * SCHEDULERS_PER_SM * mhz * 1e6
        out["issue"] = {"achieved_warp_inst_per_s": achieved_ips, "peak_warp_inst_per_s": peak_ips,
                        "frac": achieved_ips / peak_ips, "sm_mhz": mhz,
                        "warp_inst_per_step": inst_per_step,
                        "issue_slots_busy_ncu": prof["issue_busy"], "source": PROFILED_SOURCE}
    return out


def timed_launches(first, n, window=10):
    """Window-kernel launches that stepping [first, first + n) takes (whole or partial windows)."""
    launches, t = 0, first
    while t < first + n:
        t = min((t // window + 1) * window, first + n)
        launches += 1
    return launches


def run_ours(args, ws, rank, local):
    import astrosimgpu_cuda_b200 as asg

    out = {}
    seed = SEED + rank
    # One-time process set-up (CUDA context, lazy module loading) happens on a
    # 30000-neuron network first (large enough for the parallel builder), as in a
    # long-running process; the e2e timer then covers the job itself.
    for prec in ("fp32", "fp64"):
        with asg.Simulation(n_total=30000, seed=seed, pre_ms=0, sim_ms=2, precision=prec, device=local) as warm:
            warm.step(20)
    # ---- e2e: config -> device build -> 6000 steps -> summary, through the C ABI
    dist_barrier(ws)
    t0 = time.perf_counter()
    sim = asg.Simulation(n_total=N_TOTAL, seed=seed, pre_ms=PRE_MS, sim_ms=SIM_MS, precision="fp32", device=local)
    t_created = time.perf_counter()
    total = sim.summary()["total_steps"]
    if args.no_e2e:
        total = 0
    sim.step(total)
    t_stepped = time.perf_counter()
    summ = sim.summary()
    counts = sim.spike_counts(0, total)
    t_end = time.perf_counter()
    e2e_s = dist_max(t_end - t0, ws)
    out["e2e"] = {"value": ws * total / e2e_s, "unit": "net-steps/s", "seconds": e2e_s, "steps": total,
                  "h2d_bytes_per_step": 120 / max(total, 1),
                  "d2h_bytes_per_step": (counts.nbytes + 8 * summ["n_astro"] + 200) / max(total, 1),
                  "includes": "astrosim_create (device connectivity + parameters) + astrosim_step x6000 + "
                              "astrosim_summary + per-step spike counts",
                  "seconds_create": t_created - t0, "seconds_steps": t_stepped - t_created,
                  "seconds_readback": t_end - t_stepped}
    out["summary_fp32"] = {k: summ[k] for k in ("spikes_measured", "mean_rate_hz", "mean_ca", "active_astro",
                                                "engaged_astro", "build_seconds", "n_exc_edges", "n_inh_edges",
                                                "n_e2a_edges", "n_sic_edges")}

    # ---- device-resident stepping, FP32 (the headline) then FP64
    res = {}
    for prec in args.precisions:
        if prec == "fp64":
            sim.close()
            sim = asg.Simulation(n_total=N_TOTAL, seed=seed, pre_ms=PRE_MS, sim_ms=SIM_MS, precision="fp64",
                                 device=local)
            sim.step(total)  # same state point as the FP32 measurement
        sim.step(args.warmup)
        dist_barrier(ws)
        with ClockSampler(local) as clk:
            sim.step(args.steps)
            ms = sim.last_step_ms()
        ms = dist_max(ms, ws)
        s = sim.summary()
        counts = sim.spike_counts(s["steps_done"] - args.steps, args.steps)
        spikes_per_step = float(counts.mean()) if counts.size else 0.0
        gb, e_visit = gather_step_bytes(s, prec)
        res[prec] = {"ms": ms, "clocks": clk.summary(), "bytes": window_step_bytes(s, prec, spikes_per_step),
                     "gather_bytes": gb, "e_visit": e_visit, "spikes_per_step": spikes_per_step, "summary": s}
    sim.close()
    return out, res


def run_sharded(args, ws, rank, local):
    """One N_total network split across the ranks (strong scaling), one rank per GPU over NCCL."""
    from astrosimgpu_cuda_b200 import shard

    W = 10
    steps = -(-args.steps // W) * W
    warm = -(-args.warmup // W) * W
    dist_barrier(ws)
    t0 = time.perf_counter()
    sim = shard.ShardedSimulation(n_total=N_TOTAL, seed=SEED, pre_ms=PRE_MS, sim_ms=SIM_MS, precision="fp32",
                                  device=local)
    total = sim.summary()["total_steps"]
    sim.step(total)
    summ = sim.summary()
    counts = sim.spike_counts(0, total)
    e2e_s = dist_max(time.perf_counter() - t0, ws)
    sim.step(warm)
    dist_barrier(ws)
    with ClockSampler(local) as clk:
        sim.step(steps)
        ms = sim.last_step_ms()
    ms = dist_max(ms, ws)
    s = sim.summary()
    spikes_per_step = float(sim.spike_counts(s["steps_done"] - steps, steps).mean())
    sim.close()
    if rank != 0:
        return None
    peak, peak_kind = peaks()
    value = steps / (ms * 1e-3)
    bytes_step = window_step_bytes(s, "fp32", spikes_per_step)
    achieved = bytes_step * value / 1e9
    return {
        "metric": METRIC, "value": value, "unit": "net-steps/s", "n_gpus": ws, "steps": steps, "warmup": warm,
        "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic: the network is generated on the device from (N_total, seed)",
        "config": {"workload": f"one network N_total={N_TOTAL} split across {ws} GPUs by cell ranges; spikes and "
                               f"active SIC factors all-gathered over NCCL once per 10-step window",
                   "n_total": N_TOTAL, "seed": SEED, "dt_ms": DT, "parallelism": f"shard{ws}",
                   "l2": "no flush: per-step working set far larger than L2"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak * ws, "unit": "GB/s",
                     "frac": achieved / (peak * ws), "traffic": None, "peak_source": f"{peak_kind} x {ws} GPUs",
                     "kernel": "window kernel of every rank (aggregate)", "algorithmic_bytes_per_step": bytes_step},
        "e2e": {"value": total / e2e_s, "unit": "net-steps/s", "seconds": e2e_s, "steps": total,
                "h2d_bytes_per_step": 120 / total, "d2h_bytes_per_step": (counts.nbytes + 200) / total},
        "gpu_launches": (steps // W) * (4 + 2 * (ws - 1)),
        "spikes_per_step": spikes_per_step, "clocks": clk.summary(),
        "summary": {k: summ[k] for k in ("spikes_measured", "mean_rate_hz", "mean_ca", "active_astro",
                                         "engaged_astro")},
    }


def cpu_baseline(args):
    """The FP64 oracle (OpenMP, every host core) stepping the same N=1e7 network."""
    import numpy as np

    import astrosimgpu_cuda_b200 as asg
    from oracle import oracle

    threads = os.cpu_count() or 1
    with asg.Simulation(n_total=N_TOTAL, seed=SEED, pre_ms=PRE_MS, sim_ms=SIM_MS) as sim:
        csrs = {k: sim.csr(k) for k in ("exc", "inh", "sic", "e2a")}
    o = oracle.OracleSim(oracle_cfg(), threads=threads, csrs=csrs)
    del csrs
    o.step(1)
    n = max(1, args.cpu_steps)
    t = time.perf_counter()
    o.step(n)
    dt_s = time.perf_counter() - t
    o.close()
    return {"value": n / dt_s, "unit": "net-steps/s", "cores": threads, "kind": "port",
            "sample": f"FP64 oracle, the N=1e7 seed-1 network (device-built CSR, identical to the reference's), "
                      f"{n} time steps after 1 warm-up step, {dt_s:.1f} s",
            "seconds": dt_s}


def oracle_cfg():
    from astrosimgpu_cuda_b200 import abi
    return abi.default_config(n_total=N_TOTAL, seed=SEED, pre_ms=PRE_MS, sim_ms=SIM_MS)


def run_reference(args, ws, rank):
    if rank != 0:
        return None
    binary = os.path.join(REPO, "oracle", "_ref", "astrosim_fused_ref_f32")
    if not os.path.exists(binary):
        return {"impl": "reference", "unavailable": "oracle/_ref/astrosim_fused_ref_f32 not built"}
    steps = args.warmup + args.steps
    cmd = [binary, "--n", str(N_TOTAL), "--seed", str(SEED), "--pre-ms", "0", "--sim-ms", f"{steps * DT:g}"]
    t = time.perf_counter()
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=3600)
    wall = time.perf_counter() - t
    if r.returncode != 0:
        return {"impl": "reference", "unavailable": f"reference exited {r.returncode}: {r.stderr.strip()[-200:]}"}
    us = float(re.search(r"\(([0-9.]+) us/step", r.stdout).group(1))
    build = float(re.search(r"built in ([0-9.]+) s", r.stdout).group(1))
    value = 1e6 / us
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "net-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": us / 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "single network N_total=1e7 seed 1, dt 0.1 ms; the reference's -DASTROSIM_USE_FLOAT "
                               "build (its FP32 network differs from the FP64 one)",
                   "n_total": N_TOTAL, "seed": SEED, "steps_run": steps},
        "cpu_baseline": {"value": value, "unit": "net-steps/s", "cores": 1, "kind": "reference",
                         "sample": f"unmodified reference program built for sm_100a: serial host connectivity build "
                                   f"({build:.1f} s) then {steps} steps on the B200; value from its printed us/step"},
        "e2e": {"value": value, "unit": "net-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_host_build_s": build, "reference_process_wall_s": wall,
        "reference_e2e_steps_per_s_incl_build": steps / wall,
    }


def reference_sequential(cfgs, sample):
    """Wall time per network of the reference program run once per network (its FP32 build)."""
    binary = os.path.join(REPO, "oracle", "_ref", "astrosim_fused_ref_f32")
    if not os.path.exists(binary):
        return None
    times = []
    for i in sample:
        c = cfgs[i]
        cmd = [binary, "--n", str(c.n_total), "--seed", str(c.seed), "--pre-ms", f"{c.pre_ms:g}",
               "--sim-ms", f"{c.sim_ms:g}", "--w-a2n", f"{c.w_a2n:g}"]
        t = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            return None
        times.append(time.perf_counter() - t)
    return sum(times) / len(times)


def ours_sequential(cfgs, sample):
    import astrosimgpu_cuda_b200 as asg
    times = []
    for i in sample:
        t = time.perf_counter()
        with asg.Simulation(cfgs[i]) as sim:
            sim.step(sim.summary()["total_steps"])
            sim.summary()
        times.append(time.perf_counter() - t)
    return sum(times) / len(times)


def run_seed_sweep(args, local):
    """Config C3's seeds 1-3 at N=1e7: FP32 against FP64 on the same network (mean rate, SIC fraction)."""
    import astrosimgpu_cuda_b200 as asg

    out = []
    for seed in (1, 2, 3):
        row = {"seed": seed}
        for prec in ("fp32", "fp64"):
            with asg.Simulation(n_total=N_TOTAL, seed=seed, pre_ms=PRE_MS, sim_ms=SIM_MS, precision=prec,
                                device=local) as sim:
                sim.step(sim.summary()["total_steps"])
                sm = sim.summary()
            row[prec] = {"mean_rate_hz": sm["mean_rate_hz"], "sic_fraction": sm["active_astro"] / sm["n_astro"],
                         "engaged_fraction": sm["engaged_astro"] / sm["n_astro"], "mean_ca": sm["mean_ca"],
                         "spikes_measured": sm["spikes_measured"]}
        a, b = row["fp32"], row["fp64"]
        row["fp32_rate_rel_err"] = abs(a["mean_rate_hz"] - b["mean_rate_hz"]) / max(b["mean_rate_hz"], 1e-300)
        row["fp32_sic_fraction_abs_err"] = abs(a["sic_fraction"] - b["sic_fraction"])
        out.append(row)
    return out


def run_ensemble(args):
    """256 networks, N_total log-uniform in [500, 50000], 2000 ms each, FP32 (the batched configuration)."""
    import numpy as np

    import astrosimgpu_cuda_b200 as asg
    from astrosimgpu_cuda_b200 import abi

    rng = np.random.default_rng(2026)
    n = args.ens_networks
    cfgs = [abi.default_config(n_total=int(np.exp(rng.uniform(np.log(500), np.log(50000)))), seed=1000 + i,
                               pre_ms=0.0, sim_ms=2000.0, precision="fp32",
                               neuron_drive_scale=float(rng.uniform(0.8, 1.2)), w_a2n=float(rng.uniform(0.8, 1.2)))
            for i in range(n)]
    t0 = time.perf_counter()
    with asg.Ensemble(cfgs) as ens:
        build_s = ens.build_seconds()
        ens.step(20000)
        step_ms = ens.last_step_ms()
        rates = [ens.summary(i)["mean_rate_hz"] for i in range(n)]
    wall = time.perf_counter() - t0
    sample = [int(x) for x in rng.choice(n, size=min(n, args.baseline_sample), replace=False)]
    ours = ours_sequential(cfgs, sample) if sample else None
    ref = reference_sequential(cfgs, sample) if sample else None
    out = {"networks": n, "n_total_sum": int(sum(c.n_total for c in cfgs)), "sim_ms": 2000.0, "dtype": "f32",
           "sims_per_s": n / wall, "sims_per_s_stepping_only": n / (step_ms * 1e-3),
           "build_s": build_s, "stepping_s": step_ms * 1e-3, "wall_s": wall,
           "mean_rate_hz": float(np.mean(rates))}
    if ours:
        out.update({"plain_path_sequential_sims_per_s": 1.0 / ours,
                    "baseline_sample": f"{len(sample)} of the {n} networks, run one after another",
                    "speedup_vs_plain_path_sequential": (n / wall) * ours})
    if ref:
        out["reference_sequential_sims_per_s"] = 1.0 / ref
        out["speedup_vs_reference_sequential"] = (n / wall) * ref
        out["reference_note"] = "unmodified reference FP32 build, one process per network (its host build, " \
                                "default drive rate: it has no drive flag)"
    return out


def serving_configs(n, seed):
    """Serving requests: N log-uniform in [1e3, 2e5], 200-2000 ms, drive within +-20 %, FP32."""
    import numpy as np

    from astrosimgpu_cuda_b200 import abi

    rng = np.random.default_rng(seed)
    return [abi.default_config(n_total=int(np.exp(rng.uniform(np.log(1e3), np.log(2e5)))),
                               seed=int(rng.integers(1, 1 << 40)), pre_ms=0.0,
                               sim_ms=float(int(rng.uniform(200, 2000))), precision="fp32",
                               neuron_drive_scale=float(rng.uniform(0.8, 1.2))) for _ in range(n)]


def run_serving(args, rate):
    """Open-loop Poisson arrivals at `rate` req/s; min(serve_requests, rate x serve_window) requests."""
    import numpy as np

    import astrosimgpu_cuda_b200 as asg

    n = args.serve_requests if args.serve_full else \
        int(min(args.serve_requests, max(1, np.ceil(rate * args.serve_window))))
    cfgs = serving_configs(n, 7 + int(rate))
    rng = np.random.default_rng(1000 + int(rate))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    submit_t = np.zeros(n)
    ids = []
    deadline = args.serve_timeout
    with asg.Server(precision="fp32", builders=12) as srv:
        t0 = time.perf_counter()
        i = 0
        while True:
            now = time.perf_counter() - t0
            while i < n and arrivals[i] <= now:
                ids.append(srv.submit(cfgs[i]))
                submit_t[i] = time.perf_counter() - t0
                i += 1
            st = srv.stats()
            if i == n and st["done"] == n:
                break
            if now > deadline:
                break
            if st["running"] == 0 and st["building"] == 0 and st["pending"] == 0 and i < n:
                time.sleep(max(0.0, min(0.01, arrivals[i] - now)))
                continue
            srv.pump(args.serve_pump_windows)
            if st["running"] == 0:
                time.sleep(0.0005)
        res = [srv.result(r) for r in ids]
        stats = srv.stats()
    done = [(k, r) for k, r in enumerate(res) if r is not None]
    lat = np.array([r["latency_s"] for _, r in done]) if done else np.array([np.nan])
    finish = max(submit_t[k] + r["latency_s"] for k, r in done) if done else float("nan")
    return {"arrival_rate_per_s": rate, "requests": n, "completed": len(done),
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_queue_s": float(np.mean([r["queue_s"] for _, r in done])) if done else None,
            "mean_build_s": float(np.mean([r["build_s"] for _, r in done])) if done else None,
            "mean_run_s": float(np.mean([r["run_s"] for _, r in done])) if done else None,
            "sims_per_s": len(done) / finish if done else 0.0, "makespan_s": finish,
            "budget_bytes": stats["budget_bytes"]}


def serving_sweep(args):
    """The rate sweep plus sequential baselines on a sample of the same request distribution."""
    rates = [float(r) for r in args.serve_rates.split(",")]
    out = {"dtype": "f32", "workload": "open-loop Poisson arrivals; N_total log-uniform in [1e3, 2e5], "
                                      "200-2000 ms, drive within +-20 %, seeds random",
           "requests_per_rate": (f"{args.serve_requests} at every rate (--serve-full)" if args.serve_full else
                                 f"min({args.serve_requests}, ceil(rate x {args.serve_window:g} s)): the full "
                                 f"{args.serve_requests}-request stream needs {args.serve_requests / 5:.0f} s of "
                                 f"arrivals at 5 req/s, too long for the default run; --serve-full runs it"),
           "rates": [run_serving(args, r) for r in rates]}
    if args.baseline_sample <= 0:
        return out
    cfgs = serving_configs(args.baseline_sample, 99)
    sample = list(range(len(cfgs)))
    ours = ours_sequential(cfgs, sample)
    out["plain_path_sequential_sims_per_s"] = 1.0 / ours
    out["baseline_sample"] = f"{len(sample)} requests of the same distribution, run one after another"
    ref = reference_sequential(cfgs, sample)
    if ref:
        out["reference_sequential_sims_per_s"] = 1.0 / ref
        best = max(r["sims_per_s"] for r in out["rates"])
        out["best_speedup_vs_reference_sequential"] = best * ref
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the whole-job run (profiling captures)")
    ap.add_argument("--n", type=int, default=N_TOTAL, help="network size (the benchmark is N=1e7)")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-seed-sweep", action="store_true", help="skip the seeds 1-3 FP32 vs FP64 comparison")
    ap.add_argument("--leg", choices=("ensemble", "serving"), default=None,
                    help="run only the batched ensemble or the serving sweep (profiling captures)")
    ap.add_argument("--ens-networks", type=int, default=256)
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-rates", default="5,20,50,200", help="comma-separated arrival rates (req/s)")
    ap.add_argument("--serve-window", type=float, default=30.0, help="seconds of arrivals per rate at most")
    ap.add_argument("--serve-full", action="store_true",
                    help="the full --serve-requests stream at every rate (about 10 minutes for 5,20,50,200 req/s)")
    ap.add_argument("--serve-pump-windows", type=int, default=10)
    ap.add_argument("--serve-timeout", type=float, default=120.0)
    ap.add_argument("--baseline-sample", type=int, default=8)
    ap.add_argument("--shard", action="store_true",
                    help="with N > 1 GPUs: split one N_total network across the ranks (strong scaling) "
                         "instead of one replica network per rank (weak scaling, the default)")
    ap.add_argument("--precision", default="both", choices=("both", "fp32", "fp64"),
                    help="device-resident legs to time (profiling captures use one)")
    args = ap.parse_args()
    args.precisions = ("fp32", "fp64") if args.precision == "both" else (args.precision,)
    globals()["N_TOTAL"] = args.n
    args.warmup = max(3, args.warmup)
    ws, rank, local = dist_init()

    if args.impl == "reference":
        line = run_reference(args, ws, rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return

    if args.leg:  # one form alone, for profiling captures
        if ws == 1:
            # The process set-up the full run does first (CUDA context, first use of the
            # kernels), so that the leg times its own work as it does inside the full run;
            # otherwise it counts about 1.2 s of context creation as network builds.
            import astrosimgpu_cuda_b200 as asg
            with asg.Simulation(n_total=30000, seed=SEED, pre_ms=0, sim_ms=2, precision="fp32") as warm:
                warm.step(20)
            leg = run_ensemble(args) if args.leg == "ensemble" else serving_sweep(args)
            print(json.dumps({"leg": args.leg, args.leg: leg}), flush=True)
        return

    if args.shard:
        line = run_sharded(args, ws, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return

    extra, res = run_ours(args, ws, rank, local)
    if rank != 0:
        return
    peak, peak_kind = peaks()
    # the headline is FP32; a capture run of one precision reports that one
    f32 = res.get("fp32") or res["fp64"]
    f64 = res.get("fp64")
    ms_step = f32["ms"] / args.steps
    value = ws * args.steps / (f32["ms"] * 1e-3)
    achieved = f32["bytes"] / (ms_step * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "net-steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if "fp32" in res else "f64",
        "data": "synthetic: the network is generated on the device from (N_total, seed) by the reference's "
                "construction; no dataset",
        "config": {"workload": "single network N_total=1e7 (8M exc, 2M inh AdEx, 2M Li-Rinzel astrocytes), seed 1, "
                               "dt 0.1 ms; FP32 RK4 stages with FP64 V/w/Ca/IP3 accumulators; one step = one dt",
                   "n_total": N_TOTAL, "seed": SEED, "dt_ms": DT,
                   "timed_after": "the 6000-step e2e run plus the warm-up steps",
                   "window_alignment": "the engine advances every cell through 10-step windows, one launch per "
                                       "window; a call that starts or ends inside a window runs that part as its "
                                       "own launch, which reads and writes all cell state once more (e.g. "
                                       "--warmup 5 --steps 20 times three launches of 5 + 10 + 5 steps)",
                   "timed_window_launches": timed_launches(f32["summary"]["steps_done"] - args.steps, args.steps),
                   "l2": "no flush: per-step working set (CSR 5.3 GB + state) is far larger than the 126 MB L2"},
        "syn_events_per_s": f32["e_visit"] * value,
        "syn_events_definition": "edge visits of the reference's per-step gather formulation (every CSR entry "
                                 "once per step: E_visit x steps/s); the windowed push engine reads only the "
                                 "edges of sources that spiked, so this is equivalent work, not work done",
        "roofline": roofline(f32, "fp32" if "fp32" in res else "fp64", achieved, peak, peak_kind, ms_step, local),
        "spikes_per_step": f32["spikes_per_step"],
        "e2e": extra["e2e"],
        "gpu_launches": timed_launches(f32["summary"]["steps_done"] - args.steps, args.steps) +
                        (f32["summary"]["steps_done"] // 10 - (f32["summary"]["steps_done"] - args.steps) // 10),
        "clocks": f32["clocks"],
        "summary_fp32": extra["summary_fp32"],
    }
    if f64 is not None and f64 is not f32:
        line["fp64"] = {"value": ws * args.steps / (f64["ms"] * 1e-3), "unit": "net-steps/s",
                        "ms_per_step": f64["ms"] / args.steps,
                        "syn_events_per_s": f64["e_visit"] * ws * args.steps / (f64["ms"] * 1e-3),
                        "clocks": f64["clocks"]}
        line["fp32_over_fp64"] = f64["ms"] / f32["ms"]
    if args.precision == "both" and ws == 1 and args.n == 10_000_000 and not args.no_seed_sweep:
        line["fp32_vs_fp64_seeds"] = run_seed_sweep(args, local)
    if not args.no_ensemble and ws == 1 and args.n == 10_000_000:
        line["ensemble"] = run_ensemble(args)
    if not args.no_serving and ws == 1 and args.n == 10_000_000:
        line["serving"] = serving_sweep(args)
    if not args.no_cpu_baseline and ws == 1:
        try:
            line["cpu_baseline"] = cpu_baseline(args)
        except Exception as e:  # the baseline is reported, not required
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)[:200]}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
