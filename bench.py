#!/usr/bin/env python
"""Benchmark: bit-vectorised SCA (SCABit) on a 16384^2 lattice, attempted site updates per ns.

Workload (one GPU): two resident 16384x16384 periodic lattices (2^28 sites, 64 MiB packed
each, ENC_CBBIT), flat start, one at (p,q) = (1,0) and one at (0.5,0.5), counter-based
random bits from seed 42.  A step advances each lattice by --mcs-per-step Monte-Carlo
steps (default 200, so 50 steps cover the 10^4 MCS of the configuration).  Inputs are
resident in HBM when the timed region starts; L2 is flushed between steps (untimed).

value  = whole-job attempted updates / ns, device time (CUDA events on the lattices' stream),
         max over ranks; --gpus N runs N independent replicas (weak scaling).
e2e    = the same metric through the public API with host buffers: every step pushes both
         lattices from pinned host memory, runs the MCS, pops both lattices and reads W^2.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

LX = LY = 14
SEED = 42
PQS = [(1.0, 0.0), (0.5, 0.5)]
METRIC = "site updates/ns (SCA, DT, batched) vs plain loop; exact correlator TOPS"
UNIT = "attempted site updates/ns"

# Per-launch DRAM traffic of scabit_fused_kernel measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum), summarised in profiles/scabit_fused_16384.md; None until captured.
NCU_TRAFFIC_PER_LAUNCH = None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mcs-per-step", type=int, default=200)
    ap.add_argument("--fusion", type=int, default=0, help="MCS per HBM pass (0 = library default)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def dist_setup(n):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(torch, buf):
    buf.add_(1)


def run_ours(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    import cudakpz_b200 as kpzb

    dev_stream = torch.cuda.Stream()
    scheds = []
    for (p, q) in PQS:
        s = kpzb.Scheduler(LX, LY, scheduler="scaBit", device=local)
        s.setPQ(p, q)
        s.supplySeed(SEED, rank)
        s.setFusion(args.fusion)
        s.setStream(dev_stream.cuda_stream)
        scheds.append(s)
    N = 1 << (LX + LY)
    M = args.mcs_per_step
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")  # 256 MiB > L2

    def step():
        for s in scheds:
            s.mcsPQSyncRngAsync(M)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    barrier(world)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t_wall0 = time.perf_counter()
    for i in range(args.steps):
        with torch.cuda.stream(dev_stream):
            flush_l2(torch, flush)
            starts[i].record(dev_stream)
        step()
        with torch.cuda.stream(dev_stream):
            ends[i].record(dev_stream)
    torch.cuda.synchronize()
    barrier(world)
    wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    ms = max_over_ranks(ms, world)
    updates = float(N) * M * len(scheds) * args.steps * world
    value = updates / (ms * 1e6)

    # launches: the library runs k-MCS fused passes (k = its resolved choice) plus a
    # one-launch-per-half-step remainder
    k = scheds[0].fusion()
    fused_launches = (M // k) if k > 1 else 0
    half_launches = 2 * (M - fused_launches * k)
    launches_per_step = (fused_launches + half_launches) * len(scheds)
    dominant = "scabit_fused_kernel" if k > 1 else "scabit_half_kernel"
    if k > 1:
        per_launch_ms = ms / (args.steps * launches_per_step)
        bytes_per_launch = float(N) * k  # 1 B per attempted update, N*k attempts per pass
    else:
        per_launch_ms = ms / (args.steps * launches_per_step)
        bytes_per_launch = float(N) / 2  # one half-step: N/2 attempts
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1),
                "peak": peak, "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": NCU_TRAFFIC_PER_LAUNCH, "algorithmic_bytes_per_launch": bytes_per_launch,
                "launch_ms": round(per_launch_ms, 4), "mcs_per_launch": k if k > 1 else 0.5}

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, torch, kpzb, scheds, N, M, world)
    for s in scheds:
        s.setStream(0)
        s.close()
    return value, ms, wall, clk, roofline, e2e, launches_per_step * args.steps, k


def run_e2e(args, torch, kpzb, scheds, N, M, world):
    """Public API with host buffers: push (pinned H2D) -> mcs -> pop (D2H) -> roughness."""
    import numpy as np
    nw = scheds[0].size_words()
    host = [torch.empty(nw, dtype=torch.int32).pin_memory() for _ in scheds]
    outs = [torch.empty(nw, dtype=torch.int32).pin_memory() for _ in scheds]
    for h, s in zip(host, scheds):
        s.setStream(0)
        s.initHomogeneous()
        s.popSystem(h.numpy().view(np.uint32))
    steps = max(3, args.steps // 4)
    for s in scheds:
        s.mcsPQSyncRng(M)  # warm-up through the same path
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        for h, o, s in zip(host, outs, scheds):
            s.pushSystem(h.numpy().view(np.uint32))
            s.mcsPQSyncRng(M)
            s.popSystem(o.numpy().view(np.uint32))
            s.roughness()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    dt = max_over_ranks(dt, world)
    updates = float(N) * M * len(scheds) * steps * world
    return {"value": round(updates / (dt * 1e9), 3), "unit": UNIT,
            "h2d_bytes_per_step": nw * 4 * len(scheds),
            "d2h_bytes_per_step": (nw * 4 + 64) * len(scheds), "steps": steps}


def cpu_sample(nthreads=1):
    """Oracle SCABit per-site restatement on a 2048^2 sample, (1,0) and (0.5,0.5), 1 MCS each."""
    from oracle import oracle as o
    lx = ly = 11
    t0 = time.perf_counter()
    upd = 0
    for (p, q) in PQS:
        w = o.homogeneous(lx, ly, o.ENC_CBBIT)
        o.sca_mcs(w, lx, ly, o.ENC_CBBIT, SEED, 0, 0, 1, p, q)
        upd += 1 << (lx + ly)
    dt = time.perf_counter() - t0
    return upd / (dt * 1e9), dt


def run_reference(args, world, rank):
    """Reference arm: the CPU implementation of the path on the host cores (rank 0 only)."""
    if rank != 0:
        return None
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    vals = []
    for _ in range(args.warmup):
        pass
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        for _ in range(args.steps):
            res = pool.map(_ref_worker, range(cores))
            vals.append(sum(r[0] for r in res))
    wall = time.perf_counter() - t0
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": round(value, 6), "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(wall * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "SCABit 16384^2 (p,q)=(1,0),(0.5,0.5); CPU sample 2048^2, 1 MCS "
                                   "per (p,q) per core"},
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "2048^2 lattice, 1 MCS at (1,0) and 1 MCS at (0.5,0.5), per core"},
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    return line


def _ref_worker(i):
    sys.path.insert(0, str(ROOT))
    return cpu_sample()


def main():
    args = parse()
    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        line = run_reference(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    value, ms, wall, clk, roofline, e2e, launches, k = run_ours(args, world, rank, local)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, dt = cpu_sample()
        cpu = {"value": round(v, 6), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"oracle per-site SCABit, 2048^2, 1 MCS at (1,0) + 1 MCS at (0.5,0.5), {dt:.1f} s"}
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic",
                "config": {"workload": "SCABit 16384^2 periodic, flat start, (p,q)=(1,0) and (0.5,0.5), "
                                       "seed 42, counter-based random bits",
                           "lattice": "16384x16384", "mcs_per_step": args.mcs_per_step,
                           "lattices_per_gpu": len(PQS), "mcs_per_pass": k,
                           "l2": "flushed between steps (256 MiB write, untimed)",
                           "parallelism": f"replicas x{world}"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
                "gpu_launches": launches, "wall_s": round(wall, 3)}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
