"""Batched and continuously batched Cahn-Hilliard solves (include/bsam_batch.h).

A Batch keeps many independent problems resident on one GPU and advances
them together, one V-cycle of every running problem per device "tick"; each
problem converges, steps and finishes on its own schedule.  Problems may be
submitted while others run (continuous batching); a submission is admitted
when a slot and the problem's device footprint fit in the batch's pool.

There is no CPU path: every call goes to libbsam_gpu.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

PREC_FP64, PREC_MIXED = 0, 1
SLOT_IDLE, SLOT_RUNNING, SLOT_DONE, SLOT_FAILED = 0, 1, 2, 3
MAX_STEPS = 256
ERR_NOMEM = -3
ERR_DIVERGED = -7


class BatchParams(ctypes.Structure):
    _fields_ = [("ndims", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("nsmoothingpasses", ctypes.c_int32), ("maxvcycles", ctypes.c_int32),
                ("max_slots", ctypes.c_int32), ("bottom_cells", ctypes.c_int32),
                ("pool_bytes", ctypes.c_int64), ("qerrortol", ctypes.c_double)]

# Default bottom kernel size of a batch (bsam_batch.cu DEFAULT_BOTTOM_CELLS);
# a single-problem Solver with bottom_cells=BOTTOM_CELLS computes the same bits.
BOTTOM_CELLS = 1024


def _host_grid_type():
    from . import HostGrid
    return HostGrid


class BatchProblem(ctypes.Structure):
    pass


class StepResult(ctypes.Structure):
    _fields_ = [("nvcycles", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("residual", ctypes.c_double)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("grid_ctas", ctypes.c_int32), ("eager", ctypes.c_int32),
                ("per_pass", ctypes.c_int32), ("fused_ctas", ctypes.c_int32),
                ("fused_occ", ctypes.c_int32), ("tile_chunk", ctypes.c_int32),
                ("fused_chunk", ctypes.c_int32), ("regrid_threads", ctypes.c_int32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("ticks", ctypes.c_int64), ("launches", ctypes.c_int64),
                ("kernels_per_tick", ctypes.c_int64), ("captures", ctypes.c_int64),
                ("pool_used", ctypes.c_int64), ("pool_bytes", ctypes.c_int64),
                ("resident", ctypes.c_int32), ("running", ctypes.c_int32),
                ("smooth_stages", ctypes.c_int64), ("smooth_ms", ctypes.c_double),
                ("smooth_bytes", ctypes.c_double), ("regrids", ctypes.c_int64),
                ("regrid_s", ctypes.c_double)]


def bind(L):
    """Declares the batch entry points' signatures on the loaded library."""
    HostGrid = _host_grid_type()
    if "_fields_" not in BatchProblem.__dict__:
        BatchProblem._fields_ = [("grid", HostGrid), ("nsteps", ctypes.c_int32),
                                 ("pad_", ctypes.c_int32), ("dt", ctypes.c_double),
                                 ("eps", ctypes.c_double), ("alpha", ctypes.c_double)]
    vp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    L.bsam_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(BatchParams)]
    L.bsam_batch_destroy.argtypes = [vp]
    L.bsam_batch_set_tuning.argtypes = [vp, ctypes.POINTER(BatchTuning)]
    L.bsam_batch_footprint.argtypes = [vp, ctypes.POINTER(BatchProblem),
                                       ctypes.POINTER(ctypes.c_int64)]
    L.bsam_batch_submit.argtypes = [vp, ctypes.POINTER(BatchProblem), dp, ip]
    L.bsam_batch_advance.argtypes = [vp, ctypes.c_int]
    L.bsam_batch_sync.argtypes = [vp]
    L.bsam_batch_run.argtypes = [vp]
    L.bsam_batch_poll.argtypes = [vp, ip, ctypes.c_int]
    L.bsam_batch_slot_phase.argtypes = [vp, ctypes.c_int, ip, ip]
    L.bsam_batch_collect.argtypes = [vp, ctypes.c_int, dp, ctypes.POINTER(StepResult), dp]
    L.bsam_batch_profile.argtypes = [vp, ctypes.c_int]
    L.bsam_batch_submit_seeded.argtypes = [vp, ctypes.POINTER(BatchProblem), ctypes.c_uint64,
                                           ctypes.c_double, ctypes.c_double, ip]
    dpp = ctypes.POINTER(dp)
    L.bsam_batch_submit_many.argtypes = [vp, ctypes.c_int, ctypes.POINTER(BatchProblem), dpp, ip]
    L.bsam_batch_submit_seeded_many.argtypes = [vp, ctypes.c_int, ctypes.POINTER(BatchProblem),
                                                ctypes.POINTER(ctypes.c_uint64), dp, dp, ip]
    L.bsam_batch_collect_many.argtypes = [vp, ctypes.c_int, ip, dpp,
                                          ctypes.POINTER(ctypes.POINTER(StepResult)), dp]
    L.bsam_batch_busy.argtypes = [vp]
    L.bsam_batch_submit_amr.argtypes = [vp, vp, ctypes.c_int, ip]
    L.bsam_batch_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.bsam_batch_get_stats.argtypes = [vp, ctypes.POINTER(BatchStats)]
    L.bsam_batch_last_error.argtypes = [vp]
    L.bsam_batch_last_error.restype = ctypes.c_char_p


def _lib():
    from . import lib
    return lib()


def _check(rc, h, what):
    if rc != 0:
        from . import BsamError
        L = _lib()
        msg = L.bsam_gpu_strerror(rc).decode()
        if h is not None and h.value:
            detail = L.bsam_batch_last_error(h)
            if detail:
                msg += ": " + detail.decode()
        raise BsamError(f"{what} failed ({rc}): {msg}")


def problem_struct(prob) -> BatchProblem:
    """The C descriptor of a workloads.Problem."""
    from . import host_grid
    _lib()  # binds BatchProblem's layout
    return BatchProblem(grid=host_grid(prob), nsteps=prob.nsteps, pad_=0, dt=prob.dt,
                        eps=prob.eps, alpha=prob.alpha)


def problem_array(probs):
    """The C descriptors of many problems in one array, filled column by
    column through a numpy view (the same values as problem_struct)."""
    _lib()
    n = len(probs)
    arr = (BatchProblem * n)()
    v = np.ctypeslib.as_array(arr)
    g = v["grid"]
    g["ndims"] = [p.ndims for p in probs]
    g["mx"] = [tuple(p.mx[k] if k < p.ndims else 1 for k in range(3)) for p in probs]
    g["mthbc"] = [tuple(p.mthbc[:6]) for p in probs]
    g["minlevel"] = [p.minlevel for p in probs]
    g["xupper"] = [tuple(p.xupper[:3]) for p in probs]
    v["nsteps"] = [p.nsteps for p in probs]
    v["dt"] = [p.dt for p in probs]
    v["eps"] = [p.eps for p in probs]
    v["alpha"] = [p.alpha for p in probs]
    return arr


class Batch:
    """Many problems of one dimensionality resident on one GPU.

    submit() admits a problem (returns its slot, or None when the pool or the
    slots are full); advance()/run() issue V-cycle ticks; poll() lists the
    finished slots; collect() reads one back and frees its slot.
    """

    def __init__(self, ndims: int, precision: int = PREC_MIXED, max_slots: int = 64,
                 pool_bytes: int = 0, qerrortol: float = 1e-8, maxvcycles: int = 20,
                 nsmoothingpasses: int = 2, device: int = 0, grid_ctas: int = 0,
                 bottom_cells: int = 0):
        L = _lib()
        bp = BatchParams(ndims=ndims, precision=precision, nsmoothingpasses=nsmoothingpasses,
                         maxvcycles=maxvcycles, max_slots=max_slots, bottom_cells=bottom_cells,
                         pool_bytes=pool_bytes, qerrortol=qerrortol)
        h = ctypes.c_void_p()
        _check(L.bsam_batch_create(ctypes.byref(h), device, ctypes.byref(bp)), None,
               "bsam_batch_create")
        self.h = h
        self.ndims = ndims
        self.max_slots = max_slots
        self.probs = {}
        self._q0_keep = {}
        if grid_ctas:
            self.set_tuning(grid_ctas=grid_ctas)

    def set_tuning(self, grid_ctas: int = 0, eager: int = 0, per_pass: int = 0,
                   fused_ctas: int = 0, fused_occ: int = 0, tile_chunk: int = 0,
                   fused_chunk: int = 0, regrid_threads: int = 0):
        t = BatchTuning(grid_ctas=grid_ctas, eager=eager, per_pass=per_pass,
                        fused_ctas=fused_ctas, fused_occ=fused_occ, tile_chunk=tile_chunk,
                        fused_chunk=fused_chunk, regrid_threads=regrid_threads)
        _check(_lib().bsam_batch_set_tuning(self.h, ctypes.byref(t)), self.h, "set_tuning")

    def profile(self, enable: bool = True):
        _check(_lib().bsam_batch_profile(self.h, int(enable)), self.h, "profile")

    def footprint(self, prob) -> int:
        n = ctypes.c_int64(0)
        ps = problem_struct(prob)
        _check(_lib().bsam_batch_footprint(self.h, ctypes.byref(ps), ctypes.byref(n)), self.h,
               "footprint")
        return n.value

    def submit(self, prob, q0=None):
        """Admits prob with initial state q0 (default prob.q0()); returns the
        slot, or None when it does not fit now."""
        q0 = prob.q0() if q0 is None else q0
        q0 = np.asfortranarray(q0, dtype=np.float64)
        ps = problem_struct(prob)
        slot = ctypes.c_int(-1)
        rc = _lib().bsam_batch_submit(self.h, ctypes.byref(ps),
                                      q0.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      ctypes.byref(slot))
        if rc == ERR_NOMEM:
            return None
        _check(rc, self.h, "submit")
        self.probs[slot.value] = prob
        return slot.value

    def submit_seeded(self, prob):
        """Admits prob with its initial state drawn on the device from
        (prob.seed, prob.cbar, prob.amp) -- the same bits as prob.q0()."""
        ps = problem_struct(prob)
        slot = ctypes.c_int(-1)
        rc = _lib().bsam_batch_submit_seeded(self.h, ctypes.byref(ps), prob.seed, prob.cbar,
                                             prob.amp, ctypes.byref(slot))
        if rc == ERR_NOMEM:
            return None
        _check(rc, self.h, "submit_seeded")
        self.probs[slot.value] = prob
        return slot.value

    def submit_many(self, probs, q0s=None) -> list:
        """Admits probs in order with batched device work (page-locked q0s
        are read asynchronously: keep them unchanged until the next run /
        sync / collect).  q0s: per problem its q0 (Fortran order), or None
        for the seeded form.  Returns the slots; None for every problem from
        the first one that did not fit."""
        n = len(probs)
        if n == 0:
            return []
        arr = problem_array(probs)
        slots = (ctypes.c_int * n)()
        L = _lib()
        if q0s is None:
            seeds = (ctypes.c_uint64 * n)(*[p.seed for p in probs])
            cbar = (ctypes.c_double * n)(*[p.cbar for p in probs])
            amp = (ctypes.c_double * n)(*[p.amp for p in probs])
            rc = L.bsam_batch_submit_seeded_many(self.h, n, arr, seeds, cbar, amp, slots)
        else:
            keep = [np.asfortranarray(q, dtype=np.float64) for q in q0s]
            ptrs = (ctypes.POINTER(ctypes.c_double) * n)(
                *[q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for q in keep])
            rc = L.bsam_batch_submit_many(self.h, n, arr, ptrs, slots)
        if rc < 0:
            _check(rc, self.h, "submit_many")
        out = []
        for k in range(n):
            if k < rc:
                self.probs[slots[k]] = probs[k]
                if q0s is not None:
                    # the queued copy may still be reading it: kept until collected
                    self._q0_keep[slots[k]] = keep[k]
                out.append(slots[k])
            else:
                out.append(None)
        return out

    def collect_many(self, slots, want_q: bool = True, outs=None, want_mass: bool = False):
        """collect() of many slots with one wait; returns their results in
        order.  The slots must be finished or finish with the work already
        queued; without want_mass only they are waited for, so ticks advanced
        since keep running while their results are copied out.  outs: per
        slot a Fortran-ordered float64 array of q's shape to copy into
        (page-locked ones are reached at full speed)."""
        n = len(slots)
        if n == 0:
            return []
        probs = [self.probs[s] for s in slots]
        shapes = [tuple(m + 2 for m in p.mx[:p.ndims]) + (2,) for p in probs]
        if outs is not None:
            for o, shp in zip(outs, shapes):
                if o.shape != shp or o.dtype != np.float64 or not o.flags["F_CONTIGUOUS"]:
                    raise ValueError("out must be a Fortran-ordered float64 array of q's shape")
            qs = list(outs)
        else:
            qs = [np.empty(shp, order="F") for shp in shapes] if want_q else [None] * n
        # Every slot's step log in one buffer, read back through numpy views.
        first = np.zeros(n + 1, dtype=np.int64)
        first[1:] = np.cumsum([p.nsteps for p in probs])
        logbuf = (StepResult * max(int(first[-1]), 1))()
        base = ctypes.addressof(logbuf)
        sz = ctypes.sizeof(StepResult)
        pq = (ctypes.POINTER(ctypes.c_double) * n)(
            *[q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if q is not None else None
              for q in qs])
        ps = (ctypes.POINTER(StepResult) * n)(
            *[ctypes.cast(base + int(o) * sz, ctypes.POINTER(StepResult)) for o in first[:-1]])
        masses = (ctypes.c_double * n)() if want_mass else None
        rc = _lib().bsam_batch_collect_many(self.h, n, (ctypes.c_int * n)(*slots), pq, ps,
                                            masses)
        if rc == 0 or rc == ERR_DIVERGED:
            for s in slots:
                self.probs.pop(s, None)
                self._q0_keep.pop(s, None)
        _check(rc, self.h, "collect_many")
        log = np.ctypeslib.as_array(logbuf)
        nv = log["nvcycles"].astype(np.int32)
        cv = log["converged"].astype(np.int32)
        rs = log["residual"].astype(np.float64)
        out = []
        for k in range(n):
            a, e = int(first[k]), int(first[k + 1])
            out.append({"q": qs[k], "nvcycles": nv[a:e], "converged": cv[a:e],
                        "residual": rs[a:e], "mass": masses[k] if want_mass else None})
        return out

    def busy(self) -> bool:
        rc = _lib().bsam_batch_busy(self.h)
        if rc < 0:
            _check(rc, self.h, "busy")
        return rc == 1

    def advance(self, max_ticks: int = 1):
        _check(_lib().bsam_batch_advance(self.h, max_ticks), self.h, "advance")

    def sync(self):
        _check(_lib().bsam_batch_sync(self.h), self.h, "sync")

    def submit_amr(self, run, nsteps: int):
        """Hands the next nsteps time steps of a refined hierarchy to the batch:
        run is an amr.AmrRun (its native driver regrids the problem before
        every step, the batch runs the steps' V-cycles with its other
        problems).  Returns the slot, or None when no slot is free.  Leave
        run alone until collect_amr(slot)."""
        slot = ctypes.c_int(-1)
        rc = _lib().bsam_batch_submit_amr(self.h, run.a, int(nsteps), ctypes.byref(slot))
        if rc == ERR_NOMEM:
            return None
        _check(rc, self.h, "submit_amr")
        self.probs[slot.value] = ("amr", run, int(nsteps))
        return slot.value

    def is_amr(self, slot: int) -> bool:
        p = self.probs.get(slot)
        return isinstance(p, tuple) and p[0] == "amr"

    def collect_amr(self, slot: int, want_mass: bool = False) -> dict:
        """Per-step results of a finished refined hierarchy (its fields stay in
        its AmrRun, whose patch table is brought up to date) and releases the
        slot."""
        _, run, nsteps = self.probs[slot]
        steps = (StepResult * nsteps)()
        mass = ctypes.c_double(0.0)
        rc = _lib().bsam_batch_collect(self.h, slot, None, steps,
                                       ctypes.byref(mass) if want_mass else None)
        if rc == 0 or rc == ERR_DIVERGED:
            self.probs.pop(slot, None)
        _check(rc, self.h, "collect")
        run.refresh()
        return {"nvcycles": np.array([s.nvcycles for s in steps], dtype=np.int32),
                "converged": np.array([s.converged for s in steps], dtype=np.int32),
                "residual": np.array([s.residual for s in steps]),
                "mass": mass.value if want_mass else None}

    def run(self):
        _check(_lib().bsam_batch_run(self.h), self.h, "run")

    def poll(self) -> list:
        buf = (ctypes.c_int * self.max_slots)()
        n = _lib().bsam_batch_poll(self.h, buf, self.max_slots)
        if n < 0:
            _check(n, self.h, "poll")
        return [buf[i] for i in range(min(n, self.max_slots))]

    def phase(self, slot: int):
        ph, st = ctypes.c_int(0), ctypes.c_int(0)
        _check(_lib().bsam_batch_slot_phase(self.h, slot, ctypes.byref(ph), ctypes.byref(st)),
               self.h, "slot_phase")
        return ph.value, st.value

    def collect(self, slot: int, want_q: bool = True, out=None, want_mass: bool = True):
        """Final root q (with ghosts), per-step results and FP64 mass of slot.
        out: a Fortran-ordered float64 array of q's shape to copy into (for
        instance one in page-locked memory, which the copy reaches at full
        speed); by default a new array.  want_mass=False skips the mass
        reduction (one kernel and one wait fewer; "mass" is then None).  A
        refined hierarchy's slot (submit_amr) is collected by collect_amr."""
        if self.is_amr(slot):
            return self.collect_amr(slot, want_mass=want_mass)
        prob = self.probs[slot]
        shape = tuple(m + 2 for m in prob.mx[:prob.ndims]) + (2,)
        if out is not None:
            if (out.shape != shape or out.dtype != np.float64 or
                    not out.flags["F_CONTIGUOUS"]):
                raise ValueError("out must be a Fortran-ordered float64 array of q's shape")
            q = out if want_q else None
        else:
            q = np.empty(shape, order="F") if want_q else None
        steps = (StepResult * prob.nsteps)()
        mass = ctypes.c_double(0.0)
        rc = _lib().bsam_batch_collect(
            self.h, slot, q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if want_q else None,
            steps, ctypes.byref(mass) if want_mass else None)
        # The native call releases the slot when it succeeds and when it
        # reports a diverged solve; any other failure leaves it resident.
        if rc == 0 or rc == ERR_DIVERGED:
            self.probs.pop(slot, None)
            self._q0_keep.pop(slot, None)
        _check(rc, self.h, "collect")
        return {"q": q,
                "nvcycles": np.array([s.nvcycles for s in steps], dtype=np.int32),
                "converged": np.array([s.converged for s in steps], dtype=np.int32),
                "residual": np.array([s.residual for s in steps]),
                "mass": mass.value if want_mass else None}

    def stream(self) -> int:
        p = ctypes.c_void_p()
        _check(_lib().bsam_batch_get_stream(self.h, ctypes.byref(p)), self.h, "get_stream")
        return p.value or 0

    def stats(self) -> dict:
        st = BatchStats()
        _check(_lib().bsam_batch_get_stats(self.h, ctypes.byref(st)), self.h, "get_stats")
        return {k: getattr(st, k) for k, _ in BatchStats._fields_}

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            _lib().bsam_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def solve_all(problems, precision: int = PREC_MIXED, max_slots: int | None = None,
              pool_bytes: int = 0, device: int = 0, grid_ctas: int = 0, eager: int = 0,
              per_pass: int = 0, fused_ctas: int = 0, fused_occ: int = 0, tile_chunk: int = 0,
              fused_chunk: int = 0):
    """Solves every problem (one dimensionality) in one batch; admits more as
    slots free up.  Returns the collect() results in input order."""
    if not problems:
        return []
    nd = problems[0].ndims
    ms = max_slots or len(problems)
    tol = problems[0].qerrortol
    with Batch(nd, precision=precision, max_slots=ms, pool_bytes=pool_bytes, qerrortol=tol,
               maxvcycles=problems[0].maxvcycles, device=device) as b:
        knobs = dict(grid_ctas=grid_ctas, eager=eager, per_pass=per_pass, fused_ctas=fused_ctas,
                     fused_occ=fused_occ, tile_chunk=tile_chunk, fused_chunk=fused_chunk)
        if any(knobs.values()):
            b.set_tuning(**knobs)
        out = [None] * len(problems)
        pending = list(range(len(problems)))
        slot_of = {}
        while pending or slot_of:
            while pending:
                s = b.submit(problems[pending[0]])
                if s is None:
                    break
                slot_of[s] = pending.pop(0)
            if not slot_of:
                raise RuntimeError("a problem does not fit in an empty batch")
            if pending:
                b.advance(4)  # then admit into the slots that freed up
            else:
                b.advance(1 << 20)
            b.sync()
            for s in b.poll():
                out[slot_of.pop(s)] = b.collect(s)
        return out
