#!/usr/bin/env python
"""Headline benchmark: Cahn-Hilliard time steps per second on one B200 (or
N GPUs, each with its own batch).

Workload (one bench "step"): 512 independent 2D Cahn-Hilliard problems with
sides uniform over {64, 96, 128, 192, 256}, eps ~ U(0.005, 0.02),
phi0 = m + 0.05 U(-1,1), m ~ U(-0.3, 0.3) (seeded SplitMix64), dt = 1e-4,
10 implicit time steps each, FAS V(2,2) to residual 1e-8, solved together in
the batched mixed-precision form (FP32 correction-form V-cycle inside an FP64
defect loop).  The metric counts problem time steps: 5120 per bench step.

Also reported beside the headline: the same problems in the FP64 batched form
and solved one at a time by the plain FP64 form; the 3D 128^3 single-problem
workload in both forms; one point of the served form (Poisson requests);
the smoother roofline; the CPU restatement of the reference (the reference
Fortran cannot be compiled here: no Fortran compiler in the image).

Output: one JSON line on rank 0.  `--impl reference` times the CPU
restatement of the reference path with all host cores on the same workload.
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

METRIC = "CH time-steps/s (512 batched 2D problems, mixed precision, V(2,2) to residual 1e-8)"
UNIT = "time-steps/s"
WORKLOAD = ("512 independent 2D Cahn-Hilliard problems on [0,1]^2, sides U{64,96,128,192,256}, "
            "Neumann, eps~U(0.005,0.02), phi0=m+0.05U(-1,1), m~U(-0.3,0.3), dt=1e-4, "
            "10 time steps each, FAS V(2,2) red-black to residual 1e-8, batched, mixed "
            "precision (FP32 correction-form V-cycle in an FP64 defect loop)")
NPROB, NSTEPS = 512, 10


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


def dist_setup():
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
    """Max over ranks (the timing rule for multi-GPU numbers)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_problems(rank: int):
    """Rank r's batch: the 512-problem workload drawn from seed 4 + 1000 r
    (weak scaling: every GPU solves its own 512 problems, no exchange)."""
    from bsam_b200 import workloads as W
    return W.config4(nprob=NPROB, nsteps=NSTEPS, seed=4 + 1000 * rank)


# ---- CPU restatement of the reference (the oracle) ---------------------------

_ORACLE_TIMING = None


def _oracle_timing_lib():
    """Loads the host-tuned timing build of the oracle in this process."""
    global _ORACLE_TIMING
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    if _ORACLE_TIMING is None:
        _ORACLE_TIMING = pyoracle.build_timing()
        pyoracle.use_library(_ORACLE_TIMING)
    return pyoracle


def _worker_init(path):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    pyoracle.use_library(path)


_WORKLOAD_CACHE = {}


def _workload(seed):
    from bsam_b200 import workloads as W
    if seed not in _WORKLOAD_CACHE:
        _WORKLOAD_CACHE[seed] = W.config4(nprob=NPROB, nsteps=NSTEPS, seed=seed)
    return _WORKLOAD_CACHE[seed]


def _oracle_solve(args):
    """One problem of the workload, its whole solve (every time step), through
    the CPU oracle: returns (problem index, time steps, V-cycles, seconds)."""
    idx, seed = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    prob = _workload(seed)[idx]
    t0 = time.perf_counter()
    r = pyoracle.run_uniform(prob, nsteps=prob.nsteps, keep_steps=False)
    return idx, prob.nsteps, int(r["nvcycles"].sum()), time.perf_counter() - t0


def cpu_baseline(per_side: int = 48):
    """The reference path on one core: the oracle's timing build, whole
    10-step solves of a sample stratified over the five sides (the first
    `per_side` problems of each side in workload order).  The workload's time
    is estimated side by side: its problem count per side x the sample's mean
    time per problem of that side.  Runs in one spawned process, so that this
    process keeps the parity build for the accuracy check."""
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    path = pyoracle.build_timing()
    with mp.get_context("spawn").Pool(1, initializer=_worker_init, initargs=(path,)) as pool:
        return pool.apply(_cpu_baseline_body, (per_side,))


def _cpu_baseline_body(per_side):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    probs = _workload(4)
    sides = sorted({p.mx[0] for p in probs})
    per_side_time, nv_sample, st_sample, t_sample = {}, 0, 0, 0.0
    for side in sides:
        idxs = [i for i, p in enumerate(probs) if p.mx[0] == side][:per_side]
        ts = []
        for i in idxs:
            _, st, nv, t = _oracle_solve((i, 4))
            ts.append(t)
            nv_sample += nv
            st_sample += st
        per_side_time[side] = statistics.mean(ts)
        t_sample += sum(ts)
    est = sum(per_side_time[p.mx[0]] for p in probs)
    steps = sum(p.nsteps for p in probs)
    out = {"value": steps / est, "unit": UNIT, "cores": 1, "kind": "port",
           "sample": f"whole {NSTEPS}-step solves of {per_side} problems per side (sides "
                     f"{sides}), one thread, {t_sample:.1f} s; workload time estimated from "
                     "the mean per side x the workload's problems per side.  C++ restatement "
                     "of the reference Fortran path, timing build (g++ -O3 -march=native, "
                     "contracted multiply-adds), built on this host",
           "vcycles_per_s": nv_sample / t_sample,
           "sample_time_steps": st_sample}
    # The AMR configuration with sustained refinement: the oracle (timing
    # build) through the same regrid driver, two steps after one warm-up
    # step, one thread.
    from bsam_b200 import amr as AMR
    hier, prm = AMR.config2(sustained=True)
    b = pyoracle.OracleBackend(2, hier.dt, hier.eps, hier.qerrortol)
    try:
        run = AMR.RegridRun(b, hier, prm)
        run.step()
        t0 = time.perf_counter()
        for _ in range(2):
            run.step()
        out["cfg2_amr_sustained_steps_per_s"] = 2 / (time.perf_counter() - t0)
    finally:
        b.close()
    return out


def run_reference(args, world, rank):
    """The reference arm: every bench step solves the whole 512-problem
    workload (every problem's 10 time steps) with the oracle's timing build,
    one problem at a time per worker process, on every host core."""
    if rank != 0:
        return 0
    import multiprocessing as mp
    _oracle_timing_lib()
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    probs = _workload(4)
    # Largest problems first, so that the pool's last jobs are short.
    order = sorted(range(NPROB), key=lambda i: -probs[i].mx[0] * probs[i].mx[1])
    times, steps_done, nv_done = [], 0, 0
    with ctx.Pool(cores, initializer=_worker_init, initargs=(_ORACLE_TIMING,)) as pool:
        for s in range(args.warmup + args.steps):
            jobs = [(i, 4) for i in order]
            t0 = time.perf_counter()
            res = pool.map(_oracle_solve, jobs, chunksize=1)
            dt = time.perf_counter() - t0
            if s >= args.warmup:
                times.append(dt)
                steps_done += sum(r[1] for r in res)
                nv_done += sum(r[2] for r in res)
    total = sum(times)
    value = steps_done / total
    sample = (f"every bench step: all {NPROB} problems of the workload, whole {NSTEPS}-step "
              f"solves, {cores} worker processes (C++ restatement of the reference Fortran "
              "path, which cannot be compiled here; timing build g++ -O3 -march=native "
              "with contracted multiply-adds, built on this host)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "vcycles_per_s": nv_done / total,
                   "step_ms": [round(1e3 * t, 1) for t in times]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---- our arm -----------------------------------------------------------------

def _interior_err(got, ref, prob):
    """Largest |got - ref| over the interior cells of both components, and
    the same relative to the largest |ref| per component."""
    import numpy as np
    inner = tuple(slice(1, m + 1) for m in prob.mx[:prob.ndims])
    ab, rel = 0.0, 0.0
    for v in range(2):
        d = float(np.max(np.abs(got[inner + (v,)] - ref[inner + (v,)])))
        ab = max(ab, d)
        rel = max(rel, d / max(float(np.max(np.abs(ref[inner + (v,)]))), 1e-300))
    return ab, rel


def accuracy_vs_oracle(batch, problems, per_side=2):
    """Checker, outside every timed region: the final state of a sample of
    the workload stratified over the sides (the first `per_side` problems of
    each side), solved by the batch, against the FP64 oracle (parity build)
    solving the same problems."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    sample = []
    for side in sorted({p.mx[0] for p in problems}):
        sample += [p for p in problems if p.mx[0] == side][:per_side]
    slots = [batch.submit_seeded(p) for p in sample]
    batch.run()
    got = [batch.collect(s, want_q=True) for s in slots]
    worst_abs, worst_rel, per = 0.0, 0.0, []
    for p, g in zip(sample, got):
        ref = pyoracle.run_uniform(p, nsteps=p.nsteps, keep_steps=False, final_q=True)
        ab, rel = _interior_err(g["q"], ref["q_final"], p)
        worst_abs, worst_rel = max(worst_abs, ab), max(worst_rel, rel)
        per.append({"side": p.mx[0], "max_abs": ab, "max_rel": rel,
                    "vcycles": int(g["nvcycles"].sum()),
                    "vcycles_fp64_oracle": int(ref["nvcycles"].sum()),
                    "max_residual": float(g["residual"].max())})
    return {"max_err_vs_fp64": worst_rel, "max_abs_err_vs_fp64": worst_abs,
            "sample": f"{len(sample)} problems ({per_side} per side), final state of all "
                      f"{NSTEPS} steps, interior cells, both components; relative to max |ref|",
            "per_problem": per}

def solve_batch(BB, problems, precision, device, want_q=False, q0s=None):
    """Submits every problem (device-side initial state unless q0s is given),
    runs the batch to completion and collects; returns (results, stats)."""
    with BB.Batch(2, precision=precision, max_slots=len(problems), device=device) as b:
        slots = []
        for i, p in enumerate(problems):
            s = b.submit(p, q0s[i]) if q0s is not None else b.submit_seeded(p)
            slots.append(s)
        b.run()
        st = b.stats()
        res = [b.collect(s, want_q=want_q) for s in slots]
    return res, st


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    import bsam_b200 as B
    from bsam_b200 import batch as BB
    from bsam_b200 import build as BLD
    from bsam_b200 import serve as SV
    from bsam_b200 import workloads as W

    BLD.build()
    torch.cuda.set_device(local)
    problems = shard_problems(rank)
    steps_per_bench_step = sum(p.nsteps for p in problems)

    # The batch's execution choices from the project autotuner, searched on
    # a stratified sample of this workload on this GPU (results are the same
    # under every choice; only the time differs).
    from bsam_b200 import autotune as AT
    tune = AT.tuned_choice(problems, BB.PREC_MIXED, device=local, per_side=16, retune=True)
    batch = BB.Batch(2, precision=BB.PREC_MIXED, max_slots=NPROB, device=local)
    batch.set_tuning(**tune["choice"])
    stream = torch.cuda.ExternalStream(batch.stream(), device=local)

    def one_step(timed_events=None):
        slots = batch.submit_many(problems)
        batch.sync()
        if timed_events is not None:
            timed_events[0].record(stream)
        batch.run()
        if timed_events is not None:
            timed_events[1].record(stream)
        nv = 0
        conv = True
        for r in batch.collect_many(slots, want_q=False):
            nv += int(r["nvcycles"].sum())
            conv = conv and int(r["converged"].min()) == 1
        return nv, conv

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()

    # ---- device-timed region: inputs resident (drawn on the device at
    # submission, before the timed interval); every step solves all problems.
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    ticks0 = batch.stats()["ticks"]
    clk = ClockSampler(local)
    clk.start()
    barrier(world)
    torch.cuda.synchronize()
    t_ep0 = time.time()
    nvc, conv_all = [], True
    for s in range(args.steps):
        nv, conv = one_step(evs[s])
        nvc.append(nv)
        conv_all = conv_all and conv
    torch.cuda.synchronize()
    t_ep1 = time.time()
    barrier(world)
    clk.stop()
    clocks = clk.summary(t_ep0, t_ep1)
    clocks["window"] = "timed region (submission + solve + collect loop)"
    step_ms = [a.elapsed_time(b) for a, b in evs]
    dev_s = sum(step_ms) / 1e3
    dev_s_max = allmax(world, dev_s)
    stats = batch.stats()
    ticks = stats["ticks"] - ticks0
    kpt = stats["kernels_per_tick"]
    value = world * args.steps * steps_per_bench_step / dev_s_max

    # ---- smoother roofline: finest-depth stages timed with events in the
    # first two ticks (every problem running) -----------------------------------
    slots = batch.submit_many(problems)
    batch.profile(True)
    batch.advance(2)
    batch.sync()
    pst = batch.stats()
    batch.profile(False)
    batch.run()
    batch.collect_many(slots, want_q=False)
    peak, peak_kind = peaks()
    stage_ms = pst["smooth_ms"] / max(pst["smooth_stages"], 1)
    stage_bytes = pst["smooth_bytes"] / max(pst["smooth_stages"], 1)
    achieved = stage_bytes / (stage_ms / 1e3) / 1e9 if stage_ms > 0 else None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            t = json.load(open(tfile))
            traffic = t["kb_smooth2_f32_bytes_per_cell"] * t_cells(problems)
        except Exception:
            traffic = None

    # Accuracy of the measured form against the FP64 oracle (rank 0 only).
    acc = accuracy_vs_oracle(batch, problems) if rank == 0 and not args.quick else None
    batch.close()

    # ---- end to end through the public API, host buffers both ways: every
    # step submits each problem's q0 from host memory (one contiguous copy
    # per problem into the engine's transfer buffer), solves, and reads every
    # final q back into host memory --------------------------------------------
    # Inputs and results in page-locked host memory (the caller's buffers).
    pinned = []

    def pinned_array(shape):
        t = torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True)
        pinned.append(t)
        return np.ndarray(shape, dtype=np.float64, buffer=t.numpy(), order="F")

    q0s = []
    for p in problems:
        q = p.q0()
        h = pinned_array(q.shape)
        h[...] = q
        q0s.append(h)
    outs = [pinned_array(q.shape) for q in q0s]
    h2d = sum(int(q.nbytes) for q in q0s)
    # A stream of bench steps through one engine with room for two of them:
    # step s+1 is submitted (host planning and its input copies queued) and
    # advanced while step s solves, then step s is collected while step s+1
    # solves.  Every step's inputs are copied in and its results copied out
    # inside the timed region.
    eb = BB.Batch(2, precision=BB.PREC_MIXED, max_slots=2 * NPROB, device=local)
    eb.set_tuning(**tune["choice"])

    def e2e_stream(nsteps):
        cur = eb.submit_many(problems, q0s)
        eb.advance(1 << 20)
        d2h = 0
        for s in range(nsteps):
            nxt = None
            if s + 1 < nsteps:
                nxt = eb.submit_many(problems, q0s)
                eb.advance(1 << 20)
            # Waits for step s only; step s+1 solves meanwhile.
            res = eb.collect_many(cur, outs=outs)
            d2h = sum(int(r["q"].nbytes) for r in res)
            if not all(int(r["converged"].min()) == 1 for r in res):
                raise RuntimeError("an end-to-end solve did not converge")
            cur = nxt
        return d2h

    e2e_stream(args.warmup)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    d2h = e2e_stream(args.steps)
    torch.cuda.synchronize()
    e2e_s = allmax(world, time.perf_counter() - t0)
    # The same calls one step at a time (submit, run, collect), for reference.
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(args.steps):
        slots = eb.submit_many(problems, q0s)
        eb.run()
        eb.collect_many(slots, outs=outs)
    e2e_seq_s = allmax(world, time.perf_counter() - t0)
    eb.close()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dev_s_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "problems_per_gpu": NPROB,
                   "time_steps_per_bench_step": steps_per_bench_step,
                   "precision": "mixed (FP32 working levels, FP64 defect/update/bottom)",
                   "parallelism": f"independent batches x{world}",
                   "l2": "inputs larger than L2 (about 1.4 GB resident per batch)",
                   "vcycles_per_bench_step": statistics.mean(nvc),
                   "vcycles_per_s": world * sum(nvc) / dev_s_max,
                   "ticks_per_bench_step": ticks / args.steps,
                   "all_converged": conv_all,
                   "step_ms": [round(x, 3) for x in step_ms],
                   "tuning": {"choice": tune["choice"], "gain_vs_default": tune["gain"],
                              "search_s": tune.get("tuning_s"),
                              "sample": tune.get("sample")}},
        "roofline": {"bound": "hbm", "kernel": "kb_smooth2<float> (fused finest-depth "
                     "smoothing stages: nu=2 red-black sweeps of every problem, one launch "
                     "each; the pre-smoothing launch also restricts into the parent, the "
                     "post-smoothing launch applies the coarse-grid correction and the FP64 "
                     "update q64 += e)",
                     "bytes_rule": "per finest cell, each field the stage must move once: "
                                   "pre 3s+2s+5sp/4 (f1, f2, base read; state written; "
                                   "parent q, qs, base written), post 5s+sp+32 (state, f1, "
                                   "f2, base, parent q and qs read; FP64 master read and "
                                   "written), s=4, sp=4 or 8",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": stage_bytes, "launch_ms": stage_ms},
        "e2e": {"value": world * args.steps * steps_per_bench_step / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "a stream of bench steps through one engine: bsam_batch_submit_many "
                        "of step s+1 (host q0 in page-locked memory) and bsam_batch_advance "
                        "queued while step s solves, then bsam_batch_collect_many of step s "
                        "(host q into page-locked memory) while step s+1 solves; host wall "
                        "clock over all steps, max over ranks",
                "one_step_at_a_time": world * args.steps * steps_per_bench_step / e2e_seq_s},
        # Timed region: every tick's kernels plus one budget kernel per run.
        "gpu_launches": int(ticks * kpt + args.steps),
        "clocks": clocks,
    }
    if acc is not None:
        line["max_err_vs_fp64"] = acc["max_err_vs_fp64"]
        line["accuracy"] = acc

    if world == 1 and rank == 0 and not args.quick:
        extra = {}
        # FP64 batched form of the same problems (device-timed like the
        # headline, with its own autotuned choices; mean of three runs).
        tune64 = AT.tuned_choice(problems, BB.PREC_FP64, device=local, per_side=16, retune=True)
        with BB.Batch(2, precision=BB.PREC_FP64, max_slots=NPROB, device=local) as b64:
            b64.set_tuning(**tune64["choice"])
            st64 = torch.cuda.ExternalStream(b64.stream(), device=local)
            ms64 = []
            for rep in range(3):
                slots = b64.submit_many(problems)
                b64.sync()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st64)
                b64.run()
                e1.record(st64)
                torch.cuda.synchronize()
                b64.collect_many(slots, want_q=False)
                ms64.append(e0.elapsed_time(e1))
            extra["fp64_batched_steps_per_s"] = steps_per_bench_step / (statistics.mean(ms64) / 1e3)
            extra["fp64_batched_tuning"] = tune64["choice"]
            extra["mixed_over_fp64_batched"] = value / extra["fp64_batched_steps_per_s"]
        # Plain FP64 form, one problem at a time (single-problem library), on a
        # sample of the problems (every 16th).
        tt, st_ = 0.0, 0
        for p in problems[::16]:
            with B.Solver(p, precision=B.PREC_FP64) as sv:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                sv.run(p.nsteps, keep_steps=False)
                tt += time.perf_counter() - t0
                st_ += p.nsteps
        extra["fp64_one_at_a_time_steps_per_s"] = st_ / tt
        extra["speedup_vs_fp64_one_at_a_time"] = value / extra["fp64_one_at_a_time_steps_per_s"]
        # 3D 128^3 single problem, both forms (config 3): 5 time steps through
        # the C++ host driver, host wall clock.
        for name, prec in (("fp64", B.PREC_FP64), ("mixed", B.PREC_MIXED)):
            prob = W.config3(nsteps=6)
            with B.Solver(prob, precision=prec) as sv:
                sv.run(1, keep_steps=False)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r3 = sv.run(5, keep_steps=False)
                dt3 = time.perf_counter() - t0
                extra[f"cfg3_128cubed_{name}_steps_per_s"] = 5 / dt3
                extra[f"cfg3_128cubed_{name}_vcycles_per_s"] = float(r3["nvcycles"].sum()) / dt3
        # Error of both forms against the FP64 oracle after each of the first
        # three time steps (checker, outside the timed runs).
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        prob = W.config3(nsteps=3)
        ref3 = pyoracle.run_uniform(prob, nsteps=3)
        for name, prec in (("fp64", B.PREC_FP64), ("mixed", B.PREC_MIXED)):
            with B.Solver(prob, precision=prec) as sv:
                g3 = sv.run(3)
            extra[f"cfg3_128cubed_{name}_err_vs_fp64_per_step"] = [
                _interior_err(g3["q"][k], ref3["q"][k], prob)[1] for k in range(3)]
            extra[f"cfg3_128cubed_{name}_vcycles_per_step"] = [int(x) for x in g3["nvcycles"]]
        extra["cfg3_128cubed_fp64_oracle_vcycles_per_step"] = [int(x) for x in ref3["nvcycles"]]
        # Config 1 (128^2, 20 steps, FP64 to 1e-9; L2-resident, latency-bound):
        # time steps and V-cycles per second of the single-problem library,
        # and its final state against the oracle.
        prob = W.config1()
        with B.Solver(prob, precision=B.PREC_FP64) as sv:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r1 = sv.run(prob.nsteps)
            dt1 = time.perf_counter() - t0
        ref1 = pyoracle.run_uniform(prob, keep_steps=False, final_q=True)
        extra["cfg1_128sq_fp64"] = {
            "steps_per_s": prob.nsteps / dt1, "vcycles_per_s": float(r1["nvcycles"].sum()) / dt1,
            "vcycles_equal_oracle": bool(np.array_equal(r1["nvcycles"], ref1["nvcycles"])),
            "max_rel_err_vs_oracle": _interior_err(r1["q"][-1], ref1["q_final"], prob)[1],
            "timing": "host wall clock over the 20 steps through the C++ host driver"}
        # 2D AMR (config 2): 256^2 root + two refined levels, regridded every
        # step in the native driver (bsam_amr_step), FP64; host wall clock.
        from bsam_b200 import amr as AMR
        for tag, sustained, nst in (("as_configured", False, 49), ("sustained", True, 20)):
            hier, prm = AMR.config2(sustained=sustained)
            with AMR.AmrRun(hier, prm, device=local) as r:
                r.step()
                torch.cuda.synchronize()
                p0 = r.profile()
                t0 = time.perf_counter()
                nv, pats, refined = [], [], []
                for _ in range(nst):
                    nv.append(r.step()[0])
                    t = r.table_array()
                    fine = t["level"] >= 1
                    pats.append(int(fine.sum()))
                    refined.append(int((t["mx"][:, 0] * t["mx"][:, 1])[fine].sum()))
                dt_ = time.perf_counter() - t0
                p1 = r.profile()
            extra[f"cfg2_amr_{tag}"] = {
                "ms_per_step_by_phase": {k: 1e3 * (p1[k] - p0[k]) / nst for k in r.PHASES},
                "steps_per_s": nst / dt_, "steps": nst, "vcycles_mean": statistics.mean(nv),
                "refined_patches_mean": statistics.mean(pats),
                "refined_cells_mean": statistics.mean(refined),
                "steps_with_refinement": sum(1 for x in pats if x > 0),
                "tag_threshold": "|grad phi| > %.2f/eps" % (0.25 if sustained else 0.5)}
        # The same AMR workload batched: 32 problems (seeds 2..33, sustained
        # refinement) whose V-cycles run in one FP64 batch's shared launches,
        # each regridded by its own native driver between its steps
        # (bsam_batch_submit_amr); host wall clock over 5 steps of all of
        # them, after one warm-up step each (graph capture, first regrid);
        # two timed runs, both reported (the regrids make it host-bound, so
        # load on the box's shared host cores shows in it), the faster one
        # as the rate.
        from bsam_b200 import batch as BB
        nb, nst = 32, 5
        runs = [AMR.AmrRun(*AMR.config2(sustained=True, seed=2 + i), device=local)
                for i in range(nb)]
        try:
            with BB.Batch(2, precision=BB.PREC_FP64, max_slots=nb, pool_bytes=1 << 20,
                          device=local) as ab:
                rates = []
                for steps, timed in ((1, False), (nst, True), (nst, True)):
                    slots = [ab.submit_amr(r, steps) for r in runs]
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    ab.run()
                    dt_ = time.perf_counter() - t0
                    res = [ab.collect_amr(s) for s in slots]
                    if timed:
                        rates.append(nb * steps / dt_)
                st = ab.stats()
            extra["cfg2_amr_batched"] = {
                "problems": nb, "steps_each": nst, "steps_per_s": max(rates),
                "steps_per_s_runs": rates,
                "over_one_at_a_time": max(rates) / extra["cfg2_amr_sustained"]["steps_per_s"],
                "vcycles_mean": float(np.mean([x["nvcycles"].mean() for x in res])),
                "all_converged": bool(all(int(x["converged"].min()) == 1 for x in res)),
                "refined_patches_mean": float(np.mean([int((r.table_array()["level"] >= 1).sum())
                                                       for r in runs])),
                "kernels_per_tick": int(st["kernels_per_tick"]),
                "timing": "host wall clock of bsam_batch_run over all problems' steps, "
                          "regrids included"}
        finally:
            for r in runs:
                r.close()
        # Served form: the Poisson request stream at every configured rate
        # (120 requests each); the capacity is the solves/s the server
        # sustains once the arrival rate exceeds it.
        sweep = {}
        with SV.Server(pool_bytes=32 << 30, max_slots=256, ticks=4, amr_workers=8) as srv:
            # Warm-up stream (graph captures, list and staging growth, the AMR
            # workers' first handles), not reported.
            srv.serve(W.config5(40, 200.0, seed=99))
            for rate in (50, 100, 200, 500, 1000, 2000):
                reqs = srv.serve(W.config5(120, float(rate)))
                sweep[str(rate)] = SV.summarize(reqs)
        extra["served_rate_sweep"] = sweep
        extra["served_capacity_solves_per_s"] = max(v["solves_per_s"] for v in sweep.values())
        line["forms"] = extra
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_case(args):
    """Small fixed cases for ncu captures (no timing is reported):
    smooth2-small  128 problems of 256^2, mixed, one eager tick;
    ticks          the full 512-problem workload, mixed, three eager ticks;
    amr2           the 2D AMR workload with sustained refinement (256^2 root,
                   two refined levels, regridded every step), FP64, three
                   steps in the native driver;
    cfg3           the 3D 128^3 configuration: one time step in FP64, then
                   one in the mixed form, V-cycle loops issued from the host
                   (every kernel its own launch);
    amr2-batch     32 problems of that workload in one FP64 batch
                   (bsam_batch_submit_amr): one warm-up step, then two steps
                   with eager ticks (each launch issued from the host),
                   printing the host time spent regridding between steps
                   and waiting for the device."""
    from bsam_b200 import batch as BB
    from bsam_b200 import build as BLD
    from bsam_b200 import workloads as W
    BLD.build()
    if args.case == "amr2":
        from bsam_b200 import amr as AMR
        import ctypes
        from bsam_b200 import Tuning, lib
        hier, prm = AMR.config2(sustained=True)
        with AMR.AmrRun(hier, prm) as r:
            # The V-cycle loop as host-issued launches (the same kernels as
            # its graph), so that a profiler lists them one by one.
            t = Tuning(fuse_min_n=64, graph=-1)
            assert lib().bsam_gpu_set_tuning(r.b.h, ctypes.byref(t)) == 0
            nv = [r.step()[0] for _ in range(3)]
            print(json.dumps({"case": args.case, "vcycles": nv, "patches": len(r.descs)}),
                  flush=True)
        return 0
    if args.case == "cfg3":
        import bsam_b200 as B
        out = {"case": args.case}
        for name, prec in (("fp64", B.PREC_FP64), ("mixed", B.PREC_MIXED)):
            with B.Solver(W.config3(nsteps=1), precision=prec, graph=-1) as sv:
                out[name] = [int(x) for x in sv.run(1, keep_steps=False)["nvcycles"]]
        print(json.dumps(out), flush=True)
        return 0
    if args.case == "amr2-batch":
        import time
        from bsam_b200 import amr as AMR
        runs = [AMR.AmrRun(*AMR.config2(sustained=True, seed=2 + i)) for i in range(32)]
        try:
            with BB.Batch(2, precision=BB.PREC_FP64, max_slots=32, pool_bytes=1 << 20) as ab:
                slots = [ab.submit_amr(r, 1) for r in runs]
                ab.run()
                for s in slots:
                    ab.collect_amr(s)
                ab.set_tuning(eager=1)
                slots = [ab.submit_amr(r, 2) for r in runs]
                t_adv = t_wait = 0.0
                ticks = 0
                while True:
                    t0 = time.perf_counter()
                    ab.advance(1)
                    t1 = time.perf_counter()
                    ab.sync()
                    t_wait += time.perf_counter() - t1
                    t_adv += t1 - t0
                    ticks += 1
                    if len(ab.poll()) == len(slots):
                        break
                res = [ab.collect_amr(s) for s in slots]
                print(json.dumps({"case": args.case, "ticks": ticks,
                                  "host_advance_s": t_adv, "device_wait_s": t_wait,
                                  "kernels_per_tick": ab.stats()["kernels_per_tick"],
                                  "vcycles": [int(x["nvcycles"].sum()) for x in res[:4]]}),
                      flush=True)
        finally:
            for r in runs:
                r.close()
        return 0
    if args.case == "smooth2-small":
        probs = [W.seeded(2, 256, 0.01, 10, seed=500 + p, cbar=0.5, amp=0.025) for p in range(128)]
        nticks = 1
    else:
        probs = W.config4(nprob=NPROB, nsteps=NSTEPS)
        nticks = 3
    with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=len(probs)) as b:
        b.set_tuning(eager=1, fused_occ=args.fused_occ)
        for p in probs:
            assert b.submit_seeded(p) is not None
        b.sync()
        b.advance(nticks)
        b.sync()
        print(json.dumps({"case": args.case, "ticks": b.stats()["ticks"]}), flush=True)
    return 0


def t_cells(problems) -> int:
    """Cells of the finest fused depth over the batch (problems above the
    bottom kernel's size)."""
    return sum(p.mx[0] * p.mx[1] for p in problems if p.mx[0] * p.mx[1] > 4096)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="skip the side-by-side forms")
    ap.add_argument("--case", choices=["smooth2-small", "ticks", "amr2", "amr2-batch", "cfg3"],
                    default=None,
                    help="run a fixed small case for a profiler capture and exit")
    ap.add_argument("--fused-occ", type=int, default=0, choices=[0, 2, 3, 4],
                    help="case mode: the fused 2D stage's build (bsam_batch_tuning.fused_occ)")
    args = ap.parse_args()
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        return run_reference(args, world, rank)
    world, rank, local = dist_setup()
    try:
        return run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
