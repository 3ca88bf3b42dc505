"""Served form: continuous batching of Cahn-Hilliard solve requests on one GPU.

Requests arrive over time (a Poisson stream in the benchmark).  The server
keeps one batch engine per dimensionality (include/bsam_batch.h), each on its
own CUDA stream, so 2D and 3D work overlaps on the device.  A request is
admitted as soon as its engine has a free slot and room for the request's
device footprint in its memory pool; otherwise it waits in FIFO order.
Admitted problems stay resident on the device for all their time steps and
are advanced together, a few V-cycle ticks per engine launch; every loop the
server collects what has finished and admits what now fits, so requests that
arrive while others are on the GPU join the running batch.

2D requests with refined levels (regridded every step) run in a third batch
engine (FP64, bsam_batch_submit_amr): worker threads build each request's
native AMR driver (its hierarchy and engine, amr.request_run), the server
admits the ready drivers into that batch, which runs the V-cycles of all of
them in shared launches and regrids each one between its time steps.

A result depends only on its own request: the batch engine computes every
problem exactly as it would alone, and an AMR request is solved exactly as
amr.solve_request solves it alone (tests/test_gpu_serve.py checks both).
"""
from __future__ import annotations

import dataclasses
import queue
import threading
import time
from collections import deque

import numpy as np

from . import amr as AMR
from . import batch as BB


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float           # seconds after the stream starts
    prob: object             # workloads.Problem (seeded form)
    admitted: float | None = None
    finished: float | None = None
    result: dict | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Server:
    """Continuous-batching server over one batch engine per dimensionality.

    pool_bytes: device memory for resident problem state, split between the
    2D and 3D engines by `share_2d`.  ticks: V-cycle ticks per engine launch
    (the admission / completion granularity).
    """

    def __init__(self, pool_bytes: int, precision: int = BB.PREC_MIXED, max_slots: int = 256,
                 share_2d: float = 0.5, ticks: int = 4, qerrortol: float = 1e-8,
                 maxvcycles: int = 20, device: int = 0, keep_q: bool = False,
                 amr_workers: int = 2, amr_slots: int = 64):
        p2 = int(pool_bytes * share_2d)
        self.engines = {
            2: BB.Batch(2, precision=precision, max_slots=max_slots, pool_bytes=p2,
                        qerrortol=qerrortol, maxvcycles=maxvcycles, device=device),
            3: BB.Batch(3, precision=precision, max_slots=max_slots,
                        pool_bytes=pool_bytes - p2, qerrortol=qerrortol,
                        maxvcycles=maxvcycles, device=device),
        }
        # Refined requests: their fields live in their own engines, so this
        # batch needs slots, not pool memory.
        self.amr_engine = BB.Batch(2, precision=BB.PREC_FP64, max_slots=amr_slots,
                                   pool_bytes=1 << 20, qerrortol=qerrortol,
                                   maxvcycles=maxvcycles, device=device)
        self.ticks = ticks
        self.keep_q = keep_q
        self.device = device
        self.amr_workers = amr_workers

    def close(self):
        for e in self.engines.values():
            e.close()
        self.amr_engine.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def fits_alone(self, prob) -> bool:
        if getattr(prob, "maxlevel", 0) >= 1:
            return True  # solved on its own handle, outside the pools
        e = self.engines[prob.ndims]
        return e.footprint(prob) <= e.stats()["pool_bytes"]

    def serve(self, stream, time_scale: float = 1.0) -> list:
        """Runs the (arrival_s, Problem) stream in real time; returns the
        Requests with arrival, admission and completion times."""
        reqs = [Request(i, a * time_scale, p) for i, (a, p) in enumerate(stream)]
        for r in reqs:
            if not self.fits_alone(r.prob):
                raise ValueError(f"request {r.rid} does not fit in its engine's pool")
        pending = deque()
        inflight = {}
        nxt = 0
        t0 = time.perf_counter()
        now = 0.0
        running = {2: 0, 3: 0}
        # AMR requests: FIFO to the worker threads, which build their drivers
        # (host fields, engine, hierarchy) and hand them back ready.
        amr_q: queue.Queue = queue.Queue()
        amr_ready: deque = deque()
        amr_inflight = {}
        amr_left = [sum(1 for r in reqs if getattr(r.prob, "maxlevel", 0) >= 1)]
        errors = []
        lock = threading.Lock()
        ae = self.amr_engine

        def worker():
            while True:
                r = amr_q.get()
                if r is None:
                    return
                try:
                    run = AMR.request_run(r.prob, self.device)
                    with lock:
                        amr_ready.append((r, run))
                except Exception as exc:  # reported by serve() after the stream
                    errors.append(exc)

        # Finished drivers are released on a thread of their own: freeing an
        # engine's device memory waits for the whole device, which the
        # server loop must not do while the batches have work queued.
        close_q: queue.Queue = queue.Queue()

        def closer():
            while True:
                run = close_q.get()
                if run is None:
                    return
                run.close()

        threads = [threading.Thread(target=worker, daemon=True)
                   for _ in range(self.amr_workers if amr_left[0] else 0)]
        if amr_left[0]:
            threads.append(threading.Thread(target=closer, daemon=True))
        for th in threads:
            th.start()
        while nxt < len(reqs) or pending or inflight or amr_left[0] > 0:
            if errors:
                break
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                if getattr(reqs[nxt].prob, "maxlevel", 0) >= 1:
                    amr_q.put(reqs[nxt])
                else:
                    pending.append(reqs[nxt])
                nxt += 1
            # Admission: FIFO per engine (a full engine does not block the
            # other), all of an engine's waiting requests offered in one
            # batched call; admission stops at the first that does not fit.
            if pending:
                keep = deque()
                for nd, e in self.engines.items():
                    mine = [r for r in pending if r.prob.ndims == nd]
                    if not mine:
                        continue
                    slots = e.submit_many([r.prob for r in mine])
                    for r, s in zip(mine, slots):
                        if s is None:
                            continue
                        r.admitted = now
                        inflight[(nd, s)] = r
                        running[nd] += 1
                keep.extend(r for r in pending if r.admitted is None)
                pending = keep
            # Refined requests whose drivers are ready join their batch.
            while True:
                with lock:
                    item = amr_ready.popleft() if amr_ready else None
                if item is None:
                    break
                r, run = item
                s = ae.submit_amr(run, int(r.prob.nsteps))
                if s is None:
                    with lock:
                        amr_ready.appendleft(item)
                    break
                r.admitted = time.perf_counter() - t0
                amr_inflight[s] = (r, run)
            # Keep every engine with running problems busy (advancing the
            # refined requests' batch also regrids those between two steps).
            for nd, e in self.engines.items():
                if running[nd] and not e.busy():
                    e.advance(self.ticks)
            if amr_inflight and not ae.busy():
                ae.advance(self.ticks)
            # Completions.
            done_any = False
            for nd, e in self.engines.items():
                if not running[nd]:
                    continue
                done = e.poll()
                if not done:
                    continue
                results = e.collect_many(done, want_q=self.keep_q, want_mass=True)
                t_done = time.perf_counter() - t0
                for s, res in zip(done, results):
                    r = inflight.pop((nd, s))
                    r.finished = t_done
                    r.result = res
                    running[nd] -= 1
                done_any = True
            if amr_inflight:
                for s in ae.poll():
                    r, run = amr_inflight.pop(s)
                    res = ae.collect_amr(s)
                    r.finished = time.perf_counter() - t0
                    if self.keep_q:
                        res["q"] = run.state()
                        res["descs"] = list(run.descs)
                    res["patches_final"] = run.npatch
                    close_q.put(run)
                    r.result = res
                    amr_left[0] -= 1
                    done_any = True
            if not done_any and not pending and not inflight and nxt < len(reqs):
                wait = reqs[nxt].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.01))
            elif not done_any:
                time.sleep(50e-6)
        for _ in range(self.amr_workers):
            amr_q.put(None)
        close_q.put(None)
        for th in threads:
            th.join()
        if errors:
            raise errors[0]
        return reqs


def _split_latency(reqs: list) -> dict:
    """p50 / p99 latency of the requests with refined levels and of the rest."""
    out = {}
    for name, sel in (("amr", lambda r: getattr(r.prob, "maxlevel", 0) >= 1),
                      ("uniform", lambda r: getattr(r.prob, "maxlevel", 0) < 1)):
        lat = np.array([r.latency for r in reqs if sel(r)])
        if lat.size:
            out[f"{name}_p50_ms"] = float(np.percentile(lat, 50) * 1e3)
            out[f"{name}_p99_ms"] = float(np.percentile(lat, 99) * 1e3)
    return out


def summarize(reqs: list) -> dict:
    """p50 / p99 latency, solves/s and time-steps/s over the whole stream."""
    lat = np.array([r.latency for r in reqs])
    makespan = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
    steps = sum(int(r.prob.nsteps) for r in reqs)
    vcycles = sum(int(r.result["nvcycles"].sum()) for r in reqs)
    conv = all(int(r.result["converged"].min()) == 1 for r in reqs)
    return {
        "requests": len(reqs),
        "p50_ms": float(np.percentile(lat, 50) * 1e3),
        "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "mean_ms": float(lat.mean() * 1e3),
        "solves_per_s": len(reqs) / makespan,
        "steps_per_s": steps / makespan,
        "vcycles": vcycles,
        "makespan_s": makespan,
        "all_converged": conv,
        "amr_requests": sum(1 for r in reqs if getattr(r.prob, "maxlevel", 0) >= 1),
        **_split_latency(reqs),
    }
