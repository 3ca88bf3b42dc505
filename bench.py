#!/usr/bin/env python
"""Headline benchmark: Cahn-Hilliard time steps per second of the FAS
V(2,2) multigrid solve on one B200 (or N independent replicas on N GPUs).

Workload: 3D 128^3 uniform grid on [0,1]^3, Neumann BCs, eps = 0.02,
dt = 1e-4, phi0 = 0.1 + 0.05 U(-1,1) (seeded SplitMix64), V(2,2) cycles to
residual 1e-8, plain FP64.  One "step" = one implicit time step
(CopyQToQold + MultigridIterations), inputs resident in HBM.

Output: one JSON line on rank 0 (see the keys below).  `--impl reference`
times the CPU restatement of the reference Fortran path (the reference itself
cannot be compiled: no Fortran compiler in the image) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CH time-steps/s (3D 128^3, FP64, V(2,2) to residual 1e-8)"
UNIT = "time-steps/s"
WORKLOAD = ("3D uniform 128^3 Cahn-Hilliard on [0,1]^3, Neumann, eps=0.02, dt=1e-4, "
            "phi0=0.1+0.05U(-1,1) seed 3, FAS V(2,2) red-black to residual 1e-8, FP64")
L2_BYTES = 126 * 1024 * 1024


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 20 ms with
    timestamps while the benchmark runs; summary() keeps the samples inside a
    wall-clock window (the timed region)."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(1.0)  # let the sampler start producing before timing
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self, t0: float, t1: float):
        import datetime
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                mhz, mx = float(parts[2]), float(parts[3])
            except ValueError:
                continue
            if not (t0 <= ts <= t1):
                continue
            sm.append(mhz)
            smax = mx
            for n, v in zip(names, parts[6:10]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(nsteps: int = 2):
    """The CPU oracle (a restatement of the reference Fortran path) on a
    bounded sample: the first `nsteps` time steps of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from bsam_b200 import workloads as W
    pyoracle.build()
    prob = W.config3(nsteps=nsteps)
    q0 = prob.q0()
    t0 = time.perf_counter()
    r = pyoracle.run_uniform(prob, nsteps=nsteps, keep_steps=False, q0=q0)
    dt = time.perf_counter() - t0
    return {"value": nsteps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"first {nsteps} time steps of the 128^3 workload, single thread "
                      f"(C++ restatement of the reference; {int(r['nvcycles'].sum())} V-cycles)"}


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from bsam_b200 import workloads as W
    pyoracle.build()
    prob = W.config3(nsteps=args.warmup + args.steps)
    q = prob.q0()
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = pyoracle.run_uniform(prob, nsteps=1, keep_steps=True, q0=q)
        dt = time.perf_counter() - t0
        q = r["q"][0]
        if s >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": "one full time step per step, single thread (the reference "
                                   "path is serial); C++ restatement of the Fortran reference, "
                                   "which cannot be compiled here"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    import bsam_b200 as B
    from bsam_b200 import build as BLD
    from bsam_b200 import workloads as W

    BLD.build()
    torch.cuda.set_device(local)
    prob = W.config3(nsteps=args.warmup + args.steps)
    solver = B.Solver(prob, device=local)
    stream = torch.cuda.ExternalStream(solver.stream(), device=local)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    for _ in range(args.warmup):
        solver.step()
    torch.cuda.synchronize()

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.fill_(1.0)

    # ---- device-resident timed region ----
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    nvc = []
    launches0 = solver.stats()["launches"]
    clk = ClockSampler(local)
    clk.start()
    barrier(world)
    torch.cuda.synchronize()
    t_wall0 = time.perf_counter()
    t_ep0 = time.time()
    for s in range(args.steps):
        flush_l2()
        evs[s][0].record(stream)
        nv, res, conv = solver.step()
        evs[s][1].record(stream)
        nvc.append(nv)
    torch.cuda.synchronize()
    t_ep1 = time.time()
    barrier(world)
    t_wall = time.perf_counter() - t_wall0
    # Keep the GPU busy with further steps (untimed) until the sampler has seen
    # at least half a second of load; used only if the timed region is too
    # short to hold a 20 ms sample.
    while time.time() - t_ep0 < 0.5:
        solver.step()
    torch.cuda.synchronize()
    t_ep2 = time.time()
    clk.stop()
    clocks = clk.summary(t_ep0, t_ep1)
    clocks["window"] = "timed region"
    if clocks["samples"] == 0:
        clocks = clk.summary(t_ep0, t_ep2)
        clocks["window"] = "timed region + continued steps of the same workload"
    step_ms = [a.elapsed_time(b) for a, b in evs]
    dev_s = sum(step_ms) / 1e3
    dev_s_max = allmax(world, dev_s)
    launches = solver.stats()["launches"] - launches0
    value = world * args.steps / dev_s_max

    # ---- smoother stage timing (roofline): CUDA events around every
    # finest-level smoothing stage, on a separate pass of the same steps ----
    solver.profile(True)
    for s in range(min(args.steps, 3)):
        flush_l2()
        solver.step()
    torch.cuda.synchronize()
    st = solver.stats()
    solver.profile(False)

    # ---- end-to-end through the C ABI with pinned host buffers ----
    qhost = torch.empty(int(np.prod(solver.qshape)), dtype=torch.float64, pin_memory=True)
    qh = qhost.numpy().reshape(solver.qshape, order="F")
    solver.get_q_into(qh)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    for s in range(args.steps):
        flush_l2()
        e2e_ev[s][0].record(stream)
        solver.put_q_async_safe(qh)
        solver.step()
        solver.get_q_into(qh)
        e2e_ev[s][1].record(stream)
    torch.cuda.synchronize()
    e2e_s = allmax(world, sum(a.elapsed_time(b) for a, b in e2e_ev) / 1e3)
    qbytes = int(qh.nbytes)

    peak, peak_kind = peaks()
    achieved = (st["smooth_bytes"] / (st["smooth_ms"] / 1e3) / 1e9) if st["smooth_ms"] > 0 else None
    per_stage_ms = st["smooth_ms"] / max(st["smooth_stages"], 1)
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get("relax_stage_bytes_128cubed_fp64")
        except Exception:
            traffic = None

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dev_s_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64", "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MB write) before every timed step",
                   "vcycles_per_step": statistics.mean(nvc),
                   "vcycles_per_s": world * sum(nvc) / dev_s_max,
                   "wall_s_timed_region": t_wall},
        "roofline": {"bound": "hbm", "kernel": "finest-level smoothing stage (nu=2 red-black "
                     "sweeps = 4 k_relax launches)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_stage": st["smooth_bytes"] / max(st["smooth_stages"], 1),
                     "stage_ms": per_stage_ms},
        "e2e": {"value": world * args.steps / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": qbytes, "d2h_bytes_per_step": qbytes},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    solver.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup(args) if args.impl == "ours" else (
        int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
        int(os.environ.get("LOCAL_RANK", "0")))
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_ours(args, world, rank, local)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
