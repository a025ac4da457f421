#!/usr/bin/env python
"""Benchmark: bit-vectorised SCA (SCABit) on a 16384^2 lattice, attempted site updates per ns.

Workload (one GPU): two resident 16384x16384 periodic lattices (2^28 sites, 64 MiB packed
each, ENC_CBBIT), flat start, one at (p,q) = (1,0) and one at (0.5,0.5), counter-based
random bits from seed 42.  A step advances each lattice by --mcs-per-step Monte-Carlo
steps (default 200; the default 50 steps are the 10^4 MCS of the configuration).  Inputs are
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

# Per-launch DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of the pass kernels
# at 16384^2, from one ncu capture per (p, q, pass kernel, MCS per pass, CTAs per SM or tile
# rows): the first pass after an L2 flush, so an upper bound for passes that follow one another
DT_NCU_BYTES_32768 = 103.849e6 + 36.303e6
NCU_TRAFFIC_PER_LAUNCH = {(1.0, 0.0, "band", 7, 0): 67.324e6 + 23.171e6,
                          (0.5, 0.5, "band", 4, 1): 67.218e6 + 17.975e6,
                          (1.0, 0.0, "wave", 6, 2): 89.707e6 + 19.618e6,
                          (1.0, 0.0, "strip", 8, 128): 85.564e6 + 22.054e6,
                          (0.5, 0.5, "strip", 4, 56): 71.193e6 + 19.824e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mcs-per-step", type=int, default=200)
    ap.add_argument("--fusion", type=int, default=0, help="MCS per HBM pass (0 = library default)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--only-pq", type=int, default=-1,
                    help="run only lattice i of the headline pair (profiling a single rate)")
    ap.add_argument("--lx", type=int, default=0,
                    help="override the workload's log2 lattice side (small cases for ncu)")
    ap.add_argument("--dt-inner", choices=["dt", "dbsh", "db", "dtdbsh", "dbshrep"], default=None,
                    help="--workload dt / c3curve: the DT kernel's inner decomposition (default dbsh, the "
                         "reference's default)")
    ap.add_argument("--reference-gpu", action="store_true",
                    help="with --impl reference: time the reference's own CUDA scheduler on this GPU "
                         "(oracle/_ref/kpz_ref_gpu) instead of its CPU scheduler")
    ap.add_argument("--dry-run", action="store_true",
                    help="launcher check: form the process group (gloo, CPU), barrier, max over ranks, print")
    ap.add_argument("--lattice-streams", type=int, default=2,
                    help="1: the lattices of a step run one after the other on one stream; 2: each "
                         "lattice on its own stream, concurrently (per-lattice figures then come from "
                         "a short sequential run after the timed one)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the configs / reference_gpu blocks measured after the headline")
    ap.add_argument("--seeds", type=int, default=16, help="--workload c3curve: independent runs")
    ap.add_argument("--t-end", type=int, default=2000, help="--workload c3curve: MCS per run")
    ap.add_argument("--workload", choices=["scabit", "dt", "db4", "batch", "gram", "measure", "c3curve"],
                    default="scabit",
                    help="scabit: the headline 16384^2 SCA runs; dt / batch / gram: the other configs; "
                         "db4: the C3 lattice under the DB4 scheduler")
    return ap.parse_args()


def dist_setup(args):
    """One process per GPU: RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the environment
    (torchrun, or spawn_ranks below).  NCCL carries only the barriers and the max-over-ranks of
    the timings (the replicas exchange nothing); --dry-run uses gloo on the CPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo" if args.dry_run else "nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def spawn_ranks(args):
    """--gpus N without torchrun: start N rank processes of this script on this host, one per
    GPU (LOCAL_RANK = i), rendezvous on 127.0.0.1, and return the worst exit code.  Refuses
    N larger than the number of visible GPUs (except for --dry-run, which runs on the CPU)."""
    import socket
    if not args.dry_run:
        import torch
        nvis = torch.cuda.device_count()
        if args.gpus > nvis:
            print(json.dumps({"error": f"--gpus {args.gpus} but {nvis} GPU(s) visible"}), flush=True)
            return 2
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(args.gpus):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(args.gpus),
                   LOCAL_WORLD_SIZE=str(args.gpus), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(Path(__file__).resolve()), *sys.argv[1:]], env=env))
    rcs = [pr.wait() for pr in procs]
    return max(rcs)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device="cuda"):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_dry(args, world, rank):
    """--dry-run: the launcher and rank plumbing without GPU work -- every rank joins the
    group, passes a barrier and contributes its rank to a max-over-ranks (gloo, CPU)."""
    barrier(world)
    top = max_over_ranks(float(rank), world, device="cpu")
    if rank != 0:
        return None
    return {"metric": METRIC, "dry_run": True, "impl": args.impl, "n_gpus": world, "max_rank": int(top),
            "scaling": "weak", "config": {"parallelism": f"replicas x{world}"}}


class ClockSampler:
    """SM clocks and throttle reasons sampled every 10 ms during the timed region (NVML via
    nvidia-ml-py, read only; nvidia-smi at its 100 ms minimum when NVML is unavailable)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.thread = None
        self.samples = []
        self.reasons = set()
        self.smax = None

    def _nvml_loop(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self.stop_flag:
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for nm, b in bits.items():
                    if r & b:
                        self.reasons.add(nm)
            except Exception:  # pragma: no cover - depends on the driver
                pass
            time.sleep(0.01)

    def start(self):
        import threading
        self.stop_flag = False
        try:
            import pynvml as nv
            nv.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.gpu]) if vis and vis.split(",")[0].isdigit() else self.gpu
            h = nv.nvmlDeviceGetHandleByIndex(idx)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag = True
            self.thread.join(timeout=5)
            sm = self.samples
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(self.reasons), "samples": len(sm), "source": "nvml 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi 100 ms"}


def flush_l2(torch, buf):
    buf.add_(1)


def run_ours(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    import cudakpz_b200 as kpzb

    dev_stream = torch.cuda.Stream()
    scheds = []
    pqs = PQS if args.only_pq < 0 else [PQS[args.only_pq]]
    LX = LY = args.lx or globals()["LX"]
    for (p, q) in pqs:
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
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(scheds) + 1)] for _ in range(args.steps)]
    t_wall0 = time.perf_counter()
    for i in range(args.steps):
        with torch.cuda.stream(dev_stream):
            flush_l2(torch, flush)
        ev[i][0].record(dev_stream)
        for j, s in enumerate(scheds):
            s.mcsPQSyncRngAsync(M)
            ev[i][j + 1].record(dev_stream)
    torch.cuda.synchronize()
    barrier(world)
    wall = time.perf_counter() - t_wall0
    per_lat = [sum(ev[i][j].elapsed_time(ev[i][j + 1]) for i in range(args.steps)) for j in range(len(scheds))]
    step_ms = sum(per_lat)
    conc = args.lattice_streams > 1 and len(scheds) > 1
    if conc:
        # the same steps with each lattice on its own stream: both start after the L2 flush and
        # the step ends when both are done (their launches fill each other's idle SM slots)
        lat_st = [torch.cuda.Stream() for _ in scheds]
        for s, st in zip(scheds, lat_st):
            s.setStream(st.cuda_stream)
        ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        torch.cuda.synchronize()
        barrier(world)
        t_wall0 = time.perf_counter()
        for i in range(args.steps):
            with torch.cuda.stream(dev_stream):
                flush_l2(torch, flush)
            ev0[i].record(dev_stream)
            done = []
            for s, st in zip(scheds, lat_st):
                st.wait_event(ev0[i])
                s.mcsPQSyncRngAsync(M)
                e = torch.cuda.Event()
                e.record(st)
                done.append(e)
            for e in done:
                dev_stream.wait_event(e)
            ev1[i].record(dev_stream)
        torch.cuda.synchronize()
        barrier(world)
        wall = time.perf_counter() - t_wall0
        step_ms = sum(ev0[i].elapsed_time(ev1[i]) for i in range(args.steps))
        for s in scheds:
            s.setStream(dev_stream.cuda_stream)
    clk = clocks.stop()
    ms = max_over_ranks(step_ms, world)
    updates = float(N) * M * len(scheds) * args.steps * world
    value = updates / (ms * 1e6)

    # launches: each lattice runs k-MCS passes of its pass kernel (the tuner's choice for its
    # rates) plus a one-launch-per-half-step remainder
    plans = [s.plan() for s in scheds]
    ks = [pl[0] for pl in plans]
    launches_per_step = 0
    for k in ks:
        fused = (M // k) if k > 1 else 0
        launches_per_step += fused + 2 * (M - fused * k)
    kinds = sorted({pl[2] for pl in plans if pl[0] > 1})
    kernel_names = {"stream": "scabit_stream_kernel", "band": "scabit_fused_kernel", "wave": "scabit_wave_kernel",
                    "strip": "scabit_strip_kernel"}
    dominant = "+".join(kernel_names[k] for k in kinds) if kinds else "scabit_half_kernel"
    # HBM: algorithmic bytes, 1 B per attempted update, over the device time of the launches
    # (fused passes carry more than 95 % of it); with temporal blocking this exceeds the copy
    # peak -- reported as the fusion gain, not as a roofline fraction
    per_launch_ms = sum(per_lat) / (args.steps * launches_per_step)
    bytes_per_launch = float(N) * M * len(scheds) / launches_per_step
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    hbm = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
           "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback",
           "unit": "GB/s", "frac": round(achieved / peak, 4),
           "algorithmic_bytes_per_launch": bytes_per_launch, "launch_ms": round(per_launch_ms, 4)}

    # INT roofline, the binding one: the bitwise update's algorithmic ALU operations against the
    # LOP3 throughput of this GPU measured live (probe kernel, a few ms, after the timed region)
    lop3, iadd3 = kpzb.probe_alu_peak(local)
    opw = [alu_ops_per_word(p, q) for (p, q) in pqs]
    traffic = fused_traffic(pqs, plans, M, LX)
    roofline = {"bound": "int-alu", "kernel": dominant, "achieved": None, "peak": round(lop3 / 1e12, 3),
                "unit": "Tops/s (algorithmic integer ops)", "frac": None, "traffic": traffic,
                "traffic_note": "dram bytes per pass launch from an ncu capture of the same plan (first pass "
                                "after an L2 flush), launch-weighted" if traffic else "no capture of this plan",
                "peak_source": "measured live (kpzb_probe_alu_peak, 3-input LOP3 chains); of measured",
                "iadd3_peak": round(iadd3 / 1e12, 3), "mcs_per_pass": ks,
                "plans": [{"mcs_per_pass": a, "ctas_per_sm_or_tile_rows": b, "kernel": c} for a, b, c in plans],
                "hbm": hbm, "fusion_gain": hbm["frac"]}
    if None not in opw:
        ops_step = sum(float(N) * M * o / 32.0 for o in opw)
        int_ach = ops_step * args.steps / (step_ms * 1e-3)
        upd_per_op = float(N) * M * len(scheds) / ops_step  # attempts per algorithmic ALU op
        int_roof_upd = lop3 * upd_per_op / 1e9
        hbm_roof_upd = peak  # 1 B per attempt: GB/s == attempts/ns
        roofline.update({"achieved": round(int_ach / 1e12, 3), "frac": round(int_ach / lop3, 4),
                         "alu_ops_per_word": {f"{p},{q}": o for (p, q), o in zip(pqs, opw)},
                         "roofline_upd_per_ns": round(int_roof_upd, 1),
                         "per_lattice_frac": {f"{p},{q}": round(float(N) * M * args.steps * o / 32.0
                                                                 / (t * 1e-3) / lop3, 4)
                                              for (p, q), o, t in zip(pqs, opw, per_lat)}})
        # the slower of the two rooflines bounds the update rate; with temporal blocking the HBM
        # one (1 B per attempt) is the faster, so the binding fraction is the INT one
        roofline["slower_roofline"] = "hbm" if hbm_roof_upd <= int_roof_upd else "int-alu"
        roofline["frac_of_slower_roofline"] = round(value / min(hbm_roof_upd, int_roof_upd), 4)
        if achieved > peak:
            roofline["frac_of_slower_roofline"] = roofline["frac"]
            roofline["slower_roofline"] = "int-alu (HBM exceeded by temporal blocking: see fusion_gain)"

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, torch, kpzb, scheds, N, M, world)
    for s in scheds:
        s.setStream(0)
        s.close()
    per_lattice = [{"p": p, "q": q, "mcs_per_pass": kk, "kernel": pl[2],
                    "upd_per_ns": round(float(N) * M * args.steps / (t * 1e6), 1)}
                   for (p, q), kk, pl, t in zip(pqs, ks, plans, per_lat)]
    return value, ms, wall, clk, roofline, e2e, launches_per_step * args.steps, ks, per_lattice


def fused_traffic(pqs, plans, M, lx):
    """Launch-weighted mean DRAM bytes per pass from the ncu captures, when every lattice ran a
    captured (p, q, pass kernel, k) at 16384^2; None otherwise."""
    if lx != 14:
        return None
    tot, n = 0.0, 0
    for (p, q), (k, c, kind) in zip(pqs, plans):
        t = NCU_TRAFFIC_PER_LAUNCH.get((p, q, kind, k, c))
        if t is None or k < 2:
            return None
        tot += t * (M // k)
        n += M // k
    return round(tot / n) if n else None


# Algorithmic integer-ALU operations of one random-sequential attempt (DT, DB4), counted as
# alu_ops_per_word counts the SCABit rule: the acceptance word (Philox4x32-10's 20 three-way
# XORs per call / 4 words = 5; its multiplies run on the FMA pipe), the 4-bit position (5/8,
# rounded to 1), extracting the site's 2 slope bits and its neighbours' 2 bits (2 each: shift
# and mask), classifying the 4-bit configuration as 12 or 3 (2), the threshold compare (1)
# and the 3 XOR flips -- the kpz/kpzSimulationPrimitivesTemplates.cu:229-268 rule.
DT_ALU_OPS_PER_ATTEMPT = 5 + 1 + 6 + 2 + 1 + 3


def alu_ops_per_word(p, q):
    """Algorithmic integer-ALU operations per 32-site word per half-step of the SCABit rule
    (kpz/kpzSCABitCores.cu:69-74,139-145), counted as 3-input LOP3 / funnel-shift steps:
    minimum candidates 2 (when p > 0), maximum candidates 2 (when q > 0), their union 1 (when
    both), XOR of the flip mask into the four words 4, the one-bit x-shift of every other row 1
    (2 shifts on half the rows), and per random plane 1 to apply it plus the ALU part of
    Philox4x32-10 per word (10 rounds x 2 three-way XORs / 4 words = 5; its multiplies run on
    the FMA pipe).  p, q in {0, 1} need no plane, 1/2 one; other rates are not counted here."""
    ops = 4 + 1
    ops += 2 if p > 0 else 0
    ops += 2 if q > 0 else 0
    ops += 1 if (p > 0 and q > 0) else 0
    planes = sum(1 for r in (p, q) if 0 < r < 1) and 1
    if any(0 < r < 1 and r != 0.5 for r in (p, q)):
        return None
    ops += planes * (1 + 5)
    return ops


def run_e2e(args, torch, kpzb, scheds, N, M, world):
    """Public API with host buffers: push (pinned H2D) -> mcs -> pop (D2H) -> roughness, every
    step, both lattices, through the asynchronous entry points.  Each lattice runs on its own
    stream and its MCS waits for the other lattice's MCS to finish, so the lattices take turns
    on the SMs and one lattice's copies and W^2 read overlap the other's MCS (two MCS passes
    sharing the SMs would finish together and leave the copies exposed).  A step's roughness
    is enqueued behind its pop, then the next step's input is pushed: kpzb_push_async copies it
    into the handle's stage buffer on a copy stream while the current step is still queued, and
    each step's W^2 is read while the other lattice's step runs."""
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
    streams = [torch.cuda.Stream() for _ in scheds]
    for s, st in zip(scheds, streams):
        s.setStream(st.cuda_stream)
    # one untimed pass through the whole pipeline, so that one-time work (the stage buffer and
    # copy stream of the first asynchronous push, first launches of the analysis kernels) stays
    # out of the timed region
    for h, o, s in zip(host, outs, scheds):
        s.pushSystemAsync(h.numpy().view(np.uint32))
        s.mcsPQSyncRngAsync(M)
        s.popSystemAsync(o.numpy().view(np.uint32))
        s.roughnessAsync()
        s.joinRoughness()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    L = len(scheds)
    unread = [False] * L
    mcs_done = [None] * L
    for h, s in zip(host, scheds):
        s.pushSystemAsync(h.numpy().view(np.uint32))
    for step in range(steps):
        for j, (h, o, s) in enumerate(zip(host, outs, scheds)):
            prev = (j - 1) % L  # with one lattice: itself
            if mcs_done[prev] is not None and prev != j:
                streams[j].wait_event(mcs_done[prev])
            s.mcsPQSyncRngAsync(M)
            ev = torch.cuda.Event()
            ev.record(streams[j])
            mcs_done[j] = ev
            s.popSystemAsync(o.numpy().view(np.uint32))
            s.roughnessAsync()
            if step + 1 < steps:
                s.pushSystemAsync(h.numpy().view(np.uint32))
            unread[j] = True
            if unread[prev]:
                scheds[prev].joinRoughness()
                unread[prev] = False
    for j, s in enumerate(scheds):  # every step's result is read before the clock stops
        if unread[j]:
            s.joinRoughness()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    dt = max_over_ranks(dt, world)
    for s in scheds:
        s.setStream(0)
    updates = float(N) * M * len(scheds) * steps * world
    return {"value": round(updates / (dt * 1e9), 3), "unit": UNIT,
            "h2d_bytes_per_step": nw * 4 * len(scheds),
            "d2h_bytes_per_step": (nw * 4 + 128) * len(scheds), "steps": steps}  # words + the W^2 record


REF_BIN = ROOT / "oracle" / "_ref" / "kpz_ref"
REF_LX = 14  # CPU sample on the benchmark lattice itself (16384^2)
REF_MCS = 12  # MCS per (p,q) per sample: about 10 s of CPU work on 16 cores


def ref_sample(threads):
    """The reference's own SchedulerCPUCBBit (kpz/schedulerCPUCBBit_nested.inl), compiled from
    its sources into oracle/_ref/kpz_ref: REF_MCS MCS at (1,0) and at (0.5,0.5) on the 16384^2
    lattice with `threads` threads; returns (updates/ns, seconds of timed work)."""
    upd, secs = 0.0, 0.0
    for (p, q) in PQS:
        r = subprocess.run([str(REF_BIN), "bench-cbbit", str(REF_LX), str(p), str(q), str(REF_MCS), str(threads)],
                           capture_output=True, text=True, check=True)
        line = [ln for ln in r.stdout.splitlines() if ln and not ln.startswith("#")][0].split()
        secs += float(line[1])
        upd += float(1 << (2 * REF_LX)) * REF_MCS
    return upd / (secs * 1e9), secs


def port_sample():
    """Fallback when the reference binary was not built: the oracle's per-site SCABit."""
    from oracle import oracle as o
    lx = 11
    t0 = time.perf_counter()
    upd = 0
    for (p, q) in PQS:
        w = o.homogeneous(lx, lx, o.ENC_CBBIT)
        o.sca_mcs(w, lx, lx, o.ENC_CBBIT, SEED, 0, 0, 1, p, q)
        upd += 1 << (2 * lx)
    dt = time.perf_counter() - t0
    return upd / (dt * 1e9), dt


def dtr_sample(threads):
    """The reference's own CPU double-tiling scheduler SchedulerCPUDTr<TinyMT32>
    (kpz/schedulerCPUDTr.cpp), compiled from its sources into oracle/_ref/kpz_ref: REF_MCS MCS
    at p = 0.95, q = 0.05 on the 16384^2 lattice with `threads` threads (the C3 rates; the CPU
    side of C3 runs at 2^14, where the growth regime is that of the 65536^2 run)."""
    if not REF_BIN.exists():
        return None
    r = subprocess.run([str(REF_BIN), "bench-dtr", str(REF_LX), "0.95", "0.05", str(REF_MCS), str(threads)],
                       capture_output=True, text=True, check=True)
    line = [ln for ln in r.stdout.splitlines() if ln and not ln.startswith("#")][0].split()
    secs = float(line[1])
    v = float(1 << (2 * REF_LX)) * REF_MCS / (secs * 1e9)
    return {"value": round(v, 6), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"reference SchedulerCPUDTr<TinyMT32> (oracle/_ref), 16384^2, {REF_MCS} MCS at "
                      f"p=0.95 q=0.05, {threads} threads, {secs:.2f} s timed"}


def batch_cpu_sample(threads):
    """C4's CPU side: the reference's SchedulerCPUCBBit (the per-replica loop's rate) at the
    three replica rates, 1 MCS each on an 8192^2 lattice, `threads` threads."""
    if not REF_BIN.exists():
        return None
    upd, secs = 0.0, 0.0
    for (p, q) in [(1.0, 0.0), (0.9, 0.1), (0.75, 0.25)]:
        r = subprocess.run([str(REF_BIN), "bench-cbbit", "13", str(p), str(q), "1", str(threads)],
                           capture_output=True, text=True, check=True)
        line = [ln for ln in r.stdout.splitlines() if ln and not ln.startswith("#")][0].split()
        secs += float(line[1])
        upd += float(1 << 26)
    return {"value": round(upd / (secs * 1e9), 6), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"reference SchedulerCPUCBBit (oracle/_ref), 8192^2, 1 MCS at each of (1,0), (0.9,0.1), "
                      f"(0.75,0.25), {threads} threads, {secs:.2f} s timed; a loop over the replicas runs at "
                      "this rate"}


def gram_cpu_sample(threads, N):
    """C5's CPU side: one pair of the reference's Correlator::correlate (kpz/correlator.cpp) at
    16384^2 with `threads` threads, scaled to the 64 x 65 / 2 = 2080 pairs of the Gram, in the
    metric's unit (2*64*64*N height-product ops / s)."""
    if not REF_BIN.exists():
        return None
    r = subprocess.run([str(REF_BIN), "bench-corr", "14", str(threads)], capture_output=True, text=True,
                       check=True)
    secs = float([ln for ln in r.stdout.splitlines() if ln and not ln.startswith("#")][0].split()[0])
    return {"value": round(2.0 * 64 * 64 * N / (2080 * secs) / 1e12, 9), "unit": "TOPS (2*64*64*N height-product ops / s)",
            "cores": threads, "kind": "reference",
            "sample": f"reference Correlator::correlate (oracle/_ref), one pair at 16384^2, {threads} threads, "
                      f"{secs:.2f} s; x 2080 pairs = {2080 * secs / 3600:.1f} h for the Gram"}


def cpu_baseline_sample(threads):
    if REF_BIN.exists():
        v, secs = ref_sample(threads)
        return {"value": round(v, 6), "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"reference SchedulerCPUCBBit (oracle/_ref), 16384^2, {REF_MCS} MCS at (1,0) + "
                          f"{REF_MCS} MCS at (0.5,0.5), {threads} threads, {secs:.2f} s timed"}
    v, secs = port_sample()
    return {"value": round(v, 6), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"oracle per-site SCABit, 2048^2, 1 MCS at (1,0) + 1 MCS at (0.5,0.5), {secs:.1f} s"}


def run_reference(args, world, rank):
    """Reference arm: the reference's CPU implementation of the path on all host cores
    (rank 0 only); each step a bounded sample of the workload (see cpu_baseline_sample)."""
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    rs = args.workload in ("dt", "db4") and REF_BIN.exists()
    sample = (lambda: dtr_sample(cores)) if rs else (lambda: cpu_baseline_sample(cores))
    for _ in range(min(args.warmup, 1)):  # a CPU sample needs no more than one warm-up
        sample()
    vals = []
    t0 = time.perf_counter()
    last = None
    for _ in range(args.steps):
        last = sample()
        vals.append(last["value"])
    wall = time.perf_counter() - t0
    value = statistics.median(vals)
    last["value"] = round(value, 6)
    return {"metric": METRIC, "value": round(value, 6), "unit": UNIT, "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(wall * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": ("random-sequential double tiling (SchedulerCPUDTr), p=0.95 q=0.05; each CPU "
                                    f"step {REF_MCS} MCS on the 16384^2 lattice") if rs else
                                   ("SCABit 16384^2 periodic, flat start, (p,q)=(1,0) and (0.5,0.5); "
                                    f"each CPU step {REF_MCS} MCS per (p,q) on the 16384^2 lattice"),
                       "value": "median over the steps"},
            "cpu_baseline": last,
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


REF_GPU_BIN = ROOT / "oracle" / "_ref" / "kpz_ref_gpu"
# the reference's DT built with each KPZ_INNER_DD (kpz_ref_gpu itself: the default DBSH)
REF_GPU_DT_BIN = {"dt": "kpz_ref_gpu_innerdt", "dbsh": "kpz_ref_gpu", "db": "kpz_ref_gpu_innerdb",
                  "dtdbsh": "kpz_ref_gpu_innerdtdbsh", "dbshrep": "kpz_ref_gpu_innerdbshrep"}


def run_reference_gpu(args, world, rank, local):
    """The reference's own CUDA schedulers on this GPU (rank 0 only): SchedulerSCABit<SLCG64>
    (kpz/schedulerSCABit.cu, kpz/kpzSCABit.cu) for the headline workload, SchedulerDT<SLCG64,
    dis> with its default DBSH inner decomposition (kpz/schedulerDT.cu, kpz/kpz.cu) for
    --workload dt, built from the CudaKpz sources into oracle/_ref/kpz_ref_gpu and driven
    through their public mcsPQSyncRng (host wall time around the synchronous call)."""
    if rank != 0:
        return None
    if not REF_GPU_BIN.exists():
        return {"impl": "reference", "device": "gpu",
                "unavailable": "oracle/_ref/kpz_ref_gpu not built (needs the CudaKpz sources and nvcc)"}
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
    clocks = ClockSampler(local)
    runs = []
    binary = REF_GPU_BIN
    if args.workload in ("dt", "db4"):
        lx = args.lx or 16
        m = args.steps * max(1, args.mcs_per_step // 100)
        jobs = [(args.workload, lx, 0.95, 0.05, max(1, args.warmup // 3), m)]
        if args.workload == "dt":
            inner = args.dt_inner or "dbsh"
            binary = REF_GPU_BIN.parent / REF_GPU_DT_BIN[inner]
            name = f"SchedulerDT<SLCG64, dis> ({inner.upper()})"
        else:
            name = "Scheduler<SLCG64, LocalLayoutDB4> (db4)"
        config = {"workload": f"reference {name}, {1 << lx}^2, p=0.95 q=0.05", "mcs_timed": m}
    else:
        lx = args.lx or LX
        m = args.steps * args.mcs_per_step
        jobs = [("scabit", lx, p, q, max(2, args.warmup), m) for (p, q) in PQS]
        config = {"workload": f"reference SchedulerSCABit<SLCG64>, {1 << lx}^2, flat start, (p,q)=(1,0) and "
                              "(0.5,0.5)", "mcs_timed_per_lattice": m}
    clocks.start()
    for (cmd, lxx, p, q, warm, n) in jobs:
        if not binary.exists():
            clocks.stop()
            return {"impl": "reference", "device": "gpu", "unavailable": f"{binary.name} not built"}
        r = subprocess.run([str(binary), cmd, str(lxx), str(p), str(q), str(warm), str(n)],
                           capture_output=True, text=True, env=env, timeout=1200)
        if r.returncode != 0:
            clocks.stop()
            return {"impl": "reference", "device": "gpu",
                    "unavailable": f"kpz_ref_gpu {cmd} exited {r.returncode}: {r.stderr.strip()[-200:]}"}
        f = [ln for ln in r.stdout.splitlines() if ln and not ln.startswith("#")][-1].split()
        runs.append({"p": p, "q": q, "upd_per_ns": round(float(f[0]), 1), "seconds": round(float(f[1]), 4),
                     "w2": float(f[2]), "mcs": n, "lattice": f"{1 << lxx}x{1 << lxx}", "sites": 1 << (2 * lxx)})
    clk = clocks.stop()
    upd = sum(float(x["sites"]) * x["mcs"] for x in runs)
    secs = sum(x["seconds"] for x in runs)
    value = upd / (secs * 1e9)
    return {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "impl": "reference", "device": "gpu",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(secs * 1e3 / args.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic", "config": config, "per_lattice": runs,
            "timing": "host wall clock around the reference's synchronous mcsPQSyncRng", "clocks": clk}


def _line(metric_value, ms_step, args, world, config, **extra):
    d = {"metric": METRIC, "value": round(metric_value, 4), "unit": extra.pop("unit", UNIT),
         "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
         "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
         "dtype": extra.pop("dtype", "u32"), "data": "synthetic", "config": config}
    d.update(extra)
    return d


def _timed(torch, stream, fn, steps):
    """Device time of `steps` calls of fn on `stream` (CUDA events), ms total."""
    a = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    b = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for i in range(steps):
        a[i].record(stream)
        fn()
        b[i].record(stream)
    torch.cuda.synchronize()
    return sum(x.elapsed_time(y) for x, y in zip(a, b))


def run_dt(args, world, rank, local):
    """Config C3: DT random-sequential, 65536^2 (1 GiB ENC_LOCAL), p=0.95 q=0.05 (--workload
    db4: the same lattice and rates under the DB4 scheduler)."""
    import torch
    torch.cuda.set_device(local)
    import cudakpz_b200 as kpzb
    lx = args.lx or 16
    st = torch.cuda.Stream()
    db4 = args.workload == "db4"
    s = kpzb.Scheduler(lx, lx, scheduler="db4" if db4 else "dt", device=local)
    if not db4:
        s.setDtInner(args.dt_inner or "dbsh")
    s.setPQ(0.95, 0.05)
    s.supplySeed(1 + rank)
    s.setStream(st.cuda_stream)
    m = max(1, args.mcs_per_step // 100)
    for _ in range(args.warmup):
        s.mcsPQSyncRngAsync(m)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ms = _timed(torch, st, lambda: s.mcsPQSyncRngAsync(m), args.steps)
    clk = clocks.stop()
    ms = max_over_ranks(ms, world)
    N = 1 << (2 * lx)
    value = float(N) * m * args.steps * world / (ms * 1e6)
    launches = (2 if db4 else 4) * m * args.steps
    per_launch = ms / launches
    # DT: one domain set per launch, N/4 attempts reading and writing their blocks and halos
    # (~0.52 B each); DB4: every block per launch, N/2 attempts reading and writing the whole
    # lattice (1 B each)
    alg_launch = 0.5 * N if db4 else 0.52 * N / 4
    peak = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()).get("hbm_gbs", 6650.0) if (
        ROOT / "MEASURED_PEAKS.json").exists() else 6650.0
    ach = alg_launch / (per_launch * 1e-3) / 1e9
    # DRAM bytes of one DT launch from an ncu capture of dt_kernel at 32768^2 (103.8 MB read +
    # 36.3 MB written for 2^28 attempts), scaled by the lattice's sites: every launch reads and
    # writes its domain set's blocks and halos once, so the traffic grows with N
    traffic = round(DT_NCU_BYTES_32768 * N / (1 << 30)) if (not db4 and args.dt_inner == "dt") else None
    inner = args.dt_inner or "dbsh"
    s.setStream(0)
    ok, rep = s.consitencyCheck()
    s.close()
    lop3, _ = kpzb.probe_alu_peak(local)
    opa = DT_ALU_OPS_PER_ATTEMPT
    cpu = dtr_sample(os.cpu_count() or 1) if (rank == 0 and world == 1 and not args.no_cpu) else None
    int_roofline = {"bound": "int-alu", "achieved": round(value / world * opa / 1e3, 3),
                    "peak": round(lop3 / 1e12, 3), "unit": "Tops/s",
                    "frac": round(value / world * opa * 1e9 / lop3, 4),
                    "peak_source": "measured live (kpzb_probe_alu_peak, 3-input LOP3 chains)",
                    "alu_ops_per_attempt": opa, "roofline_upd_per_ns": round(lop3 / opa / 1e9, 1)}
    return _line(value, ms / args.steps, args, world,
                 {"workload": (f"DB4 random-sequential {1 << lx}^2 periodic ({N // 4 >> 20} MiB ENC_LOCAL), "
                               "flat start, p=0.95 q=0.05, 2 launches per MCS over all 256x128 blocks, "
                               "5-site dead border") if db4 else
                              (f"DT random-sequential {1 << lx}^2 periodic ({N // 4 >> 20} MiB ENC_LOCAL), "
                               f"flat start, p=0.95 q=0.05, random origin + shuffled domain sets per MCS, "
                               f"inner scheme {inner.upper()}"),
                  "mcs_per_step": m, "lattice": f"{1 << lx}x{1 << lx}", "parallelism": f"replicas x{world}"},
                 roofline={"bound": "int-alu", "kernel": "dt_kernel", "achieved": int_roofline["achieved"],
                           "peak": int_roofline["peak"], "unit": "Tops/s (algorithmic integer ops)",
                           "frac": int_roofline["frac"], "traffic": traffic,
                           "peak_source": int_roofline["peak_source"] + "; of measured",
                           "alu_ops_per_attempt": opa, "roofline_upd_per_ns": int_roofline["roofline_upd_per_ns"],
                           "hbm": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                                   "frac": round(ach / peak, 4),
                                   "note": ("1 B" if db4 else "0.52 B") + "/attempt algorithmic"},
                           "note": "integer/barrier bound" + ("; traffic scaled from a 32768^2 ncu capture"
                                                              if traffic else ""),
                           "slower_roofline": "int-alu", "frac_of_slower_roofline": int_roofline["frac"]},
                 clocks=clk, gpu_launches=launches, invariants_ok=ok, cpu_baseline=cpu)


def run_batch(args, world, rank, local):
    """Config C4: 512 replicas (256x256^2, 128x1024^2, 64x2048^2, 64x4096^2), rates from
    {(1,0),(0.9,0.1),(0.75,0.25)} drawn with seed 0, replica seeds 1000+i; one batched pass
    kernel per k MCS vs the plain per-lattice launch loop (one launch per half-step)."""
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    import cudakpz_b200 as kpzb
    lxs = [8] * 256 + [10] * 128 + [11] * 64 + [12] * 64
    rng = np.random.default_rng(0)
    rates = [(1.0, 0.0), (0.9, 0.1), (0.75, 0.25)]
    pq = [rates[i] for i in rng.integers(0, 3, size=len(lxs))]
    seeds = [1000 + i for i in range(len(lxs))]
    sites = float(sum(1 << (2 * lx) for lx in lxs))
    b = kpzb.Batch(lxs, [a for a, _ in pq], [c for _, c in pq], seeds, device=local)
    m = 64
    b.mcs(m * max(1, args.warmup))  # the first MCS tunes the pass shape (replicas restored after)
    plan = b.plan()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        b.mcs(m)
    dt_b = time.perf_counter() - t0
    clk = clocks.stop()
    dt_b = max_over_ranks(dt_b, world)
    value = sites * m * args.steps * world / (dt_b * 1e9)
    # plain per-lattice launch loop on the same replicas (one step, same MCS)
    hs = []
    for i, lx in enumerate(lxs):
        s = kpzb.Scheduler(lx, lx, device=local)
        s.setPQ(*pq[i])
        s.supplySeed(seeds[i])
        s.setFusion(1)
        hs.append(s)
    for s in hs:
        s.mcsPQSyncRngAsync(2)
    for s in hs:
        s.join()
    t0 = time.perf_counter()
    for s in hs:
        s.mcsPQSyncRngAsync(m)
    for s in hs:
        s.join()
    dt_plain = time.perf_counter() - t0
    plain = sites * m / (dt_plain * 1e9)
    # the same loop with each lattice at its tuned pass plan (temporal blocking per lattice)
    for s in hs:
        s.setFusion(0)
    for s in hs:
        s.mcsPQSyncRngAsync(8)  # resolves (and tunes, once per size and rate class) the plans
    for s in hs:
        s.join()
    t0 = time.perf_counter()
    for s in hs:
        s.mcsPQSyncRngAsync(m)
    for s in hs:
        s.join()
    dt_tuned = time.perf_counter() - t0
    tuned = sites * m / (dt_tuned * 1e9)
    # identical per-replica lattices: compare a sample of replicas after equal MCS
    same = True
    for i in (0, 300, 400, 500):
        ref = kpzb.Scheduler(lxs[i], lxs[i], device=local)
        ref.setPQ(*pq[i])
        ref.supplySeed(seeds[i])
        ref.mcsPQSyncRng(m * (args.warmup + args.steps))
        same &= bool(np.array_equal(ref.popSystem(), b.pop(i)))
        ref.close()
    for s in hs:
        s.close()
    b.close()

    # where the time goes: the same kind of batch restricted to one size class or one rate class
    def sub_rate(sel):
        idx = [i for i in range(len(lxs)) if sel(i)]
        sb = kpzb.Batch([lxs[i] for i in idx], [pq[i][0] for i in idx], [pq[i][1] for i in idx],
                        [seeds[i] for i in idx], device=local)
        sb.mcs(m)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        sb.mcs(m)
        d = time.perf_counter() - t1
        out = {"replicas": len(idx), "upd_per_ns": round(sum(1 << (2 * lxs[i]) for i in idx) * m / (d * 1e9), 1),
               "plan": {"mcs_per_pass": sb.plan()[0], "ctas_per_sm": sb.plan()[1]}}
        sb.close()
        return out
    breakdown = {"256^2 replicas (resident in shared memory)": sub_rate(lambda i: lxs[i] == 8),
                 "1024^2-4096^2 replicas (banded)": sub_rate(lambda i: lxs[i] > 8),
                 "rate (1,0): no random plane": sub_rate(lambda i: pq[i] == (1.0, 0.0)),
                 "rates (0.9,0.1) and (0.75,0.25): bit-serial planes": sub_rate(lambda i: pq[i] != (1.0, 0.0))}
    return _line(value, dt_b * 1e3 / args.steps, args, world,
                 {"workload": "512 SCABit replicas (256x256^2,128x1024^2,64x2048^2,64x4096^2), mixed (p,q)",
                  "mcs_per_step": m, "parallelism": f"replicas x{world}"},
                 plan={"mcs_per_pass": plan[0], "ctas_per_sm": plan[1], "source": "kpzb_batch_autotune"},
                 breakdown=breakdown,
                 plain_loop_value=round(plain, 3), speedup_vs_plain_loop=round(value / plain, 2),
                 tuned_loop_value=round(tuned, 3), speedup_vs_tuned_loop=round(value / tuned, 2),
                 replicas_bit_identical_to_single_runs=same, clocks=clk,
                 timing="host wall clock around synchronous batch calls",
                 cpu_baseline=batch_cpu_sample(os.cpu_count() or 1) if (rank == 0 and world == 1 and not args.no_cpu)
                 else None)


def c3_times(t_end):
    ts = [2 ** k for k in range(20) if 2 ** k < t_end]
    return ts + [t_end]


def curve_stats(w2, ts):
    """Seed-averaged W^2(t) with standard errors, and beta from a fit of log W^2 against log t
    over t >= 32 with a jackknife error over the seeds."""
    import numpy as np
    w2 = np.asarray(w2, dtype=float)
    n = len(w2)
    t = np.asarray(ts, dtype=float)
    sel = t >= 32

    def beta(rows):
        return float(np.polyfit(np.log(t[sel]), np.log(rows.mean(0)[sel]), 1)[0] / 2)
    b = beta(w2)
    jk = [beta(np.delete(w2, i, axis=0)) for i in range(n)] if n > 2 else [b]
    bj = float(np.mean(jk))
    err = float(np.sqrt((n - 1) / n * np.sum((np.array(jk) - bj) ** 2))) if n > 2 else None
    return {"t": list(ts), "w2_mean": [round(float(v), 6) for v in w2.mean(0)],
            "w2_stderr": [round(float(v), 6) for v in (w2.std(0, ddof=1) / np.sqrt(n) if n > 1 else 0 * w2[0])],
            "beta": round(b, 5), "beta_jackknife_err": None if err is None else round(err, 5), "seeds": n}


def run_c3curve(args, world, rank, local):
    """Config C3 as a curve: DT random-sequential on the 65536^2 lattice (--lx), p=0.95 q=0.05,
    flat start, --seeds independent runs to --t-end MCS (default 16 x 2000), inner scheme
    --dt-inner (the reference's default DBSH unless given); W^2 at t = 2^k and t_end, the
    interface velocity from the deposition/desorption counters, beta from W^2(t)."""
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    import cudakpz_b200 as kpzb
    lx = args.lx or 16
    N = float(1 << (2 * lx))
    ts = c3_times(args.t_end)
    inner = args.dt_inner or "dbsh"
    w2, vel = [], []
    t0 = time.perf_counter()
    for sd in range(1 + rank * args.seeds, 1 + (rank + 1) * args.seeds):
        s = kpzb.Scheduler(lx, lx, scheduler="dt", device=local)
        s.setDtInner(inner)
        s.setPQ(0.95, 0.05)
        s.supplySeed(sd)
        s.enableCounters(True)
        t, row = 0, []
        for T in ts:
            s.mcsPQSyncRng(T - t)
            t = T
            row.append(s.roughness().w2)
        dep, des = s.counters()
        vel.append(2.0 * (dep - des) / N / ts[-1])
        w2.append(row)
        s.close()
    secs = time.perf_counter() - t0
    st = curve_stats(w2, ts)
    v = np.array(vel)
    return _line(N * ts[-1] * len(w2) * world / (secs * 1e9), secs * 1e3, args, world,
                 {"workload": f"DT {1 << lx}^2, p=0.95 q=0.05, flat start, inner scheme {inner.upper()}, "
                              f"{len(w2)} seeds x {ts[-1]} MCS", "lattice": f"{1 << lx}x{1 << lx}"},
                 curve=st, velocity={"mean": round(float(v.mean()), 6),
                                     "stderr": round(float(v.std(ddof=1) / np.sqrt(len(v))), 6) if len(v) > 1 else None},
                 timing="host wall clock around the whole curve (includes the roughness reductions)")


def run_reference_c3curve(args, rank, local):
    """The reference's own SchedulerDT<SLCG64, dis> build with the chosen inner scheme on the same
    curve (kpz_ref_gpu dtcurve, supplySeed(1, seed)): W^2 at the same times, beta."""
    if rank != 0:
        return None
    binary = REF_GPU_BIN.parent / REF_GPU_DT_BIN[args.dt_inner or "dbsh"]
    if not binary.exists():
        return {"impl": "reference", "unavailable": f"{binary.name} not built"}
    lx = args.lx or 16
    ts = c3_times(args.t_end)
    w2 = []
    t0 = time.perf_counter()
    for sd in range(1, args.seeds + 1):
        r = subprocess.run([str(binary), "dtcurve", str(lx), "0.95", "0.05", str(sd)] + [str(t) for t in ts],
                           capture_output=True, text=True, timeout=7200)
        if r.returncode != 0:
            return {"impl": "reference", "unavailable": f"{binary.name} dtcurve exited {r.returncode}"}
        rows = [ln.split() for ln in r.stdout.splitlines() if ln and not ln.startswith("#")]
        w2.append([float(x[1]) for x in rows])
    secs = time.perf_counter() - t0
    N = float(1 << (2 * lx))
    return {"metric": METRIC, "impl": "reference", "device": "gpu", "value": round(N * ts[-1] * len(w2) / (secs * 1e9), 3),
            "unit": UNIT, "n_gpus": 1, "config": {"workload": f"reference SchedulerDT ({(args.dt_inner or 'dbsh').upper()}) "
                                                              f"{1 << lx}^2, p=0.95 q=0.05, {len(w2)} seeds x {ts[-1]} MCS"},
            "curve": curve_stats(w2, ts), "timing": "host wall clock around the whole curve"}


def run_measure(args, world, rank, local):
    """Row f1 (measurement scheduling): a 16384^2 SCABit run at (1/2,1/2) to --mcs-per-step x
    10 MCS measured on the reference's default exponential schedule (SamplingParam::makeExp(0,
    0.1), kpz/sampling.h:84-100) three ways: kpzb_measure_run (MCS chunks and height reductions
    enqueued back to back, one record copy at the end); the frontend loop of
    kpz/kpzScaling.cpp:194-215 with the analysis on the device (kpzb_mcs + kpzb_roughness per
    sample); and the same loop with the reference's lattice pop per sample (64 MiB D2H, the
    host analysis itself not counted).  value = attempted updates/ns of the first."""
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    import cudakpz_b200 as kpzb
    lx = args.lx or LX
    end = args.mcs_per_step * 10
    smp = kpzb.make_sampling("exp", density=0.1)
    times = kpzb.sample_times(0, end, smp)
    N = float(1 << (2 * lx))

    def fresh():
        s = kpzb.Scheduler(lx, lx, scheduler="scaBit", device=local)
        s.setPQ(0.5, 0.5)
        s.supplySeed(SEED, rank)
        s.fusion()  # resolve the pass plan (tuner) outside the timed region
        return s

    out = {}
    for mode in ("measure_run", "device_roughness_loop", "pop_loop"):
        best = None
        for rep in range(max(1, args.warmup // 3) + 1):  # first repetition warms up
            s = fresh()
            # pinned, as the reference registers its host lattice (kpz/schedulerBase.cu:76-80)
            host = torch.empty(s.size_words(), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
            torch.cuda.synchronize()
            barrier(world)
            t0 = time.perf_counter()
            if mode == "measure_run":
                rows = s.measureRun(end, smp)
            else:
                t = 0
                for T in times:
                    s.mcsPQSyncRng(int(T) - t)
                    t = int(T)
                    if mode == "device_roughness_loop":
                        s.roughness()
                    else:
                        s.popSystem(host)
            torch.cuda.synchronize()
            dt = max_over_ranks(time.perf_counter() - t0, world)
            s.close()
            if rep > 0 or max(1, args.warmup // 3) == 0:
                best = dt if best is None else min(best, dt)
        out[mode] = N * end * world / (best * 1e9)
        if mode == "measure_run":
            best_run = best
    return _line(out["measure_run"], best_run * 1e3, args, world,
                 {"workload": f"SCABit {1 << lx}^2 (0.5,0.5) to t={end}, exp sampling density 0.1 "
                              f"({len(times)} measurements)", "parallelism": f"replicas x{world}"},
                 device_roughness_loop=round(out["device_roughness_loop"], 1),
                 pop_loop=round(out["pop_loop"], 1), measurements=int(len(times)),
                 timing="host wall clock around each whole run (includes every measurement)")


def run_gram(args, world, rank, local):
    """Config C5: exact height autocorrelator, 64 snapshots of a 16384^2 SCA run at p=1 q=0
    (snapshots after MCS 1..64), full 64x64 Gram over 2^28 sites on tcgen05 INT8 vs int64."""
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    import cudakpz_b200 as kpzb
    lx = args.lx or 14
    N = 1 << (2 * lx)
    s = kpzb.Scheduler(lx, lx, device=local)
    s.setPQ(1.0, 0.0)
    s.supplySeed(42)
    g = kpzb.Gram(lx, lx, 64, device=local)
    for _ in range(64):
        s.mcsPQSyncRng(1)
        g.add_device(s.devicePtr())
    for _ in range(args.warmup):
        g.compute(0)
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        G0, S0 = g.compute(0)
    dt0 = (time.perf_counter() - t0) / args.steps
    clk = clocks.stop()
    t0 = time.perf_counter()
    G1, S1 = g.compute(1)
    dt1 = time.perf_counter() - t0
    exact = bool(np.array_equal(G0, G1) and np.array_equal(S0, S1))
    tops = 2.0 * 64 * 64 * N / dt0 / 1e12
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    bf16 = peaks.get("bf16_tflops", 1590.0)
    int8_peak = 2.0 * bf16  # dense int8 tcgen05 issues twice the bf16 rate; bf16 measured
    hbm_bytes = 64 * N / 8.0  # the snapshots' X-slope bits, read once
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    g.close()
    s.close()
    return _line(tops, dt0 * 1e3, args, world,
                 {"workload": "64x64 exact height Gram, 16384^2 lattice, slope snapshots, limbs built in shared "
                              "memory, 3 int8 limbs, tcgen05 kind::i8",
                  "snapshots": 64, "sites": N},
                 unit="TOPS (2*64*64*N height-product ops / s)", dtype="int8->int32->int64",
                 int64_cuda_core_s=round(dt1, 4),
                 speedup_vs_int64=round(dt1 / dt0, 2), exact_match_int64=exact,
                 roofline={"bound": "tensor", "kernel": "gram_tc_kernel", "achieved": round(tops, 1),
                           "peak": round(int8_peak, 1),
                           "unit": "TOPS (the Gram's 2*64*64*N algorithmic ops against the int8 tcgen05 peak)",
                           "frac": round(tops / int8_peak, 4), "traffic": None,
                           "peak_source": "2 x measured bf16 (MEASURED_PEAKS.json bf16_tflops); of measured",
                           "hbm": {"achieved": round(hbm_bytes / dt0 / 1e9, 1), "peak": hbm_peak, "unit": "GB/s",
                                   "frac": round(hbm_bytes / dt0 / 1e9 / hbm_peak, 4),
                                   "note": "slope snapshots, N/8 bytes each"}},
                 storage_bytes=int(64 * N / 8 + 64 * (1 << lx) * 8),
                 clocks=clk, timing="host wall clock around synchronous compute calls",
                 cpu_baseline=gram_cpu_sample(os.cpu_count() or 1, N) if (rank == 0 and world == 1 and not args.no_cpu)
                 else None)


def run_configs(args, local):
    """The other configurations and the reference's own CUDA schedulers, measured after the
    headline in the same run (rank 0, one GPU): C3 (DT and the reference's default DBSH scheme
    on 65536^2, the reference's builds of the same schemes on 16384^2), C4 (512 batched
    replicas against the per-lattice loops), C5 (the exact 64x64 Gram against int64), and the
    reference's SchedulerSCABit<SLCG64> on the headline lattices.  A part that fails reports
    its error instead of a number."""
    import copy

    def sub(**kw):
        a = copy.copy(args)
        a.no_cpu, a.no_e2e = True, True
        for k, v in kw.items():
            setattr(a, k, v)
        return a

    def guard(fn):
        try:
            return fn()
        except Exception as e:  # reported in the line, never fatal to the headline
            return {"error": f"{type(e).__name__}: {e}"[:300]}

    t0 = time.perf_counter()
    out = {}
    out["reference_gpu"] = guard(lambda: {
        k: v for k, v in run_reference_gpu(sub(impl="reference", reference_gpu=True, workload="scabit", lx=14,
                                               steps=1, warmup=2, mcs_per_step=20), 1, 0, local).items()
        if k in ("value", "unit", "per_lattice", "timing", "clocks", "config", "unavailable")})

    def c3():
        res = {"ours_65536": {}, "reference_gpu_16384": {}, "ours_16384": {}}
        for inner in ("dt", "dbsh"):
            for lx, key in ((16, "ours_65536"), (14, "ours_16384")):
                ln = run_dt(sub(workload="dt", dt_inner=inner, lx=lx, steps=4, warmup=3, mcs_per_step=100), 1, 0,
                            local)
                res[key][inner] = {"upd_per_ns": ln["value"], "int_alu_frac": ln["roofline"]["frac"]}
            r = run_reference_gpu(sub(impl="reference", reference_gpu=True, workload="dt", dt_inner=inner, lx=14,
                                      steps=4, warmup=3, mcs_per_step=100), 1, 0, local)
            res["reference_gpu_16384"][inner] = r.get("value", r.get("unavailable"))
        for inner in ("dt", "dbsh"):
            ref = res["reference_gpu_16384"][inner]
            if isinstance(ref, (int, float)) and ref > 0:
                res[f"ratio_{inner}_16384"] = round(res["ours_16384"][inner]["upd_per_ns"] / ref, 2)
        res["workload"] = "DT random-sequential, p=0.95 q=0.05, flat start; dbsh = the reference's default scheme"
        return res
    out["C3"] = guard(c3)

    def c4():
        ln = run_batch(sub(workload="batch", steps=2, warmup=1), 1, 0, local)
        return {k: ln[k] for k in ("value", "unit", "plan", "breakdown", "plain_loop_value", "speedup_vs_plain_loop",
                                   "tuned_loop_value", "speedup_vs_tuned_loop",
                                   "replicas_bit_identical_to_single_runs", "config") if k in ln}
    out["C4"] = guard(c4)

    def c5():
        ln = run_gram(sub(workload="gram", steps=3, warmup=1), 1, 0, local)
        return {k: ln[k] for k in ("value", "unit", "speedup_vs_int64", "exact_match_int64", "int64_cuda_core_s", "storage_bytes",
                                   "ms_per_step", "roofline", "config") if k in ln}
    out["C5"] = guard(c5)
    out["seconds"] = round(time.perf_counter() - t0, 1)
    return out


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args))
    world, rank, local = dist_setup(args)
    if args.dry_run:
        line = run_dry(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "c3curve" and args.impl == "reference":
        line = run_reference_c3curve(args, rank, local)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if args.workload != "scabit" and args.impl == "ours":
        fn = {"dt": run_dt, "db4": run_dt, "batch": run_batch, "gram": run_gram,
              "measure": run_measure, "c3curve": run_c3curve}[args.workload]
        line = fn(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference" and args.reference_gpu:
        line = run_reference_gpu(args, world, rank, local)
        if line is not None:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        line = run_reference(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    value, ms, wall, clk, roofline, e2e, launches, ks, per_lattice = run_ours(args, world, rank, local)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample(os.cpu_count() or 1)
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic",
                "config": {"workload": "SCABit 16384^2 periodic, flat start, (p,q)=(1,0) and (0.5,0.5), "
                                       "seed 42, counter-based random bits",
                           "lattice": "16384x16384", "mcs_per_step": args.mcs_per_step,
                           "lattices_per_gpu": len(PQS), "mcs_per_pass": ks,
                           "l2": "flushed between steps (256 MiB write, untimed)",
                           "lattice_streams": ("concurrent: each lattice on its own stream, the step timed "
                                               "from the flush to both lattices done; per_lattice from a "
                                               "sequential run of the same steps")
                           if args.lattice_streams > 1 else "sequential on one stream",
                           "parallelism": f"replicas x{world}"},
                "per_lattice": per_lattice, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "clocks": clk,
                "gpu_launches": launches, "wall_s": round(wall, 3)}
        if world == 1 and not args.no_configs:
            extra = run_configs(args, local)
            line["reference_gpu"] = extra.pop("reference_gpu")
            line["configs"] = extra
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
