"""Fixed block-structured AMR hierarchies for the V-cycle (2D and 3D).

The reference builds its hierarchy by tagging and Berger-Rigoutsos
clustering every time step (lib/bsamroutines.f90:939-1241, 1352-1579); the
multigrid solve itself (MultigridIterations) only reads the resulting patch
records.  This module builds such records for a hierarchy given box by box:
the root grid with its below-root levels (as RootInit / InitSeed do), and
refined patches on levels 1, 2, ... with their parent, their index box in
the parent (mbounds), their global index box (mglobal) and their face codes
(999 = internal face, else the root's physical code) -- the fields of
nodeinfo (lib/nodeinfodef.f90:124-219) that bsam_gpu_set_hierarchy takes.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

from . import workloads as W

INTERNAL = 999


@dataclasses.dataclass
class Hierarchy:
    ndims: int
    descs: list            # patch records, ApplyOnLevel order within a level
    q0s: list              # q (with ring) of every patch on a level >= 0, descs order
    dt: float
    eps: float
    qerrortol: float
    alpha: float = 1.0
    maxvcycles: int = 20
    nsmoothingpasses: int = 2

    @property
    def finestlevel(self) -> int:
        return max(d["level"] for d in self.descs)

    def state_patches(self) -> list:
        """Indices of the patches on levels >= 0 (the order of q0s)."""
        return [i for i, d in enumerate(self.descs) if d["level"] >= 0]


class HierSolver:
    """A fixed hierarchy resident on a GPU, driven through the C ABI
    (bsam_gpu_set_hierarchy with every level, put_field of every state patch,
    then the C++ host driver's time loop)."""

    def __init__(self, hier: Hierarchy, device: int = 0, bottom_cells: int = 0):
        import ctypes
        from . import FIELD_Q, PREC_FP64, PatchDesc, RunParams, Tuning, _check, _dp, lib
        L = lib()
        self.hier = hier
        rp = RunParams(ndims=hier.ndims, nrvars=2, mbc=1, maux=0,
                       nsmoothingpasses=hier.nsmoothingpasses, maxvcycles=hier.maxvcycles,
                       errortype=1, precision=PREC_FP64, dt=hier.dt, qerrortol=hier.qerrortol,
                       alpha=hier.alpha, eps=hier.eps)
        h = ctypes.c_void_p()
        _check(L.bsam_gpu_create(ctypes.byref(h), device, ctypes.byref(rp)), what="create")
        self.h = h
        try:
            t = Tuning(bottom_cells=bottom_cells)
            _check(L.bsam_gpu_set_tuning(h, ctypes.byref(t)), h, "set_tuning")
            n = len(hier.descs)
            arr = (PatchDesc * n)()
            for i, d in enumerate(hier.descs):
                o = arr[i]
                o.level, o.parent, o.dx = d["level"], d["parent"], d["dx"]
                for k in range(3):
                    o.mx[k] = d["mx"][k]
                    o.xlower[k] = d["xlower"][k]
                    for s in range(2):
                        o.mbounds[k][s] = d["mbounds"][k][s]
                        o.mglobal[k][s] = d["mglobal"][k][s]
                for f in range(6):
                    o.mthbc[f] = d["mthbc"][f]
            _check(L.bsam_gpu_set_hierarchy(h, n, arr, hier.finestlevel), h, "set_hierarchy")
            self.states = hier.state_patches()
            for p, q in zip(self.states, hier.q0s):
                q = np.asfortranarray(q, dtype=np.float64)
                _check(L.bsam_gpu_put_field(h, p, FIELD_Q, _dp(q)), h, "put_field")
            _check(L.bsam_gpu_set_ghost(h), h, "set_ghost")
            _check(L.bsam_gpu_copy_q_to_qold(h), h, "copy_q_to_qold")
        except Exception:
            self.close()
            raise

    def run(self, nsteps: int) -> dict:
        """TakeTimeSteps on the fixed hierarchy; final q of every state patch."""
        import ctypes
        from . import FIELD_Q, _check, _dp, lib
        L = lib()
        nvc = np.zeros(nsteps, dtype=np.int32)
        res = np.zeros(nsteps)
        conv = np.zeros(nsteps, dtype=np.int32)
        ipp = ctypes.POINTER(ctypes.c_int)
        _check(L.bsam_host_take_time_steps(self.h, nsteps, 0, None, 0, nvc.ctypes.data_as(ipp),
                                           _dp(res), conv.ctypes.data_as(ipp), None),
               self.h, "take_time_steps")
        qs = []
        for p, q0 in zip(self.states, self.hier.q0s):
            out = np.zeros(q0.shape, order="F")
            _check(L.bsam_gpu_get_field(self.h, p, FIELD_Q, _dp(out)), self.h, "get_field")
            qs.append(out)
        return {"q": qs, "nvcycles": nvc, "residual": res, "converged": conv}

    def errflags(self, patch: int, tol: float) -> np.ndarray:
        """SetErrFlagsUser of a state patch (descs index): 0/1 bytes (1:mx)^d."""
        import ctypes
        from . import _check, lib
        d = self.hier.descs[patch]
        shape = tuple(d["mx"][:self.hier.ndims])
        out = np.zeros(shape, dtype=np.uint8, order="F")
        _check(lib().bsam_gpu_errflags(self.h, patch, tol,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))),
               self.h, "errflags")
        return out

    def tag_level(self, level: int, tol: float, ibuffer: int) -> list:
        """Tagging, buffering and summed-area tables of a level on the device
        (bsam_gpu_tag_level): one int32 table (1:mx)^d per patch of the level,
        in table order."""
        import ctypes
        from . import _check, lib
        nd = self.hier.ndims
        pats = [d for d in self.hier.descs if d["level"] == level]
        sizes = [int(np.prod(d["mx"][:nd])) for d in pats]
        buf = np.zeros(sum(sizes), dtype=np.int32)
        _check(lib().bsam_gpu_tag_level(self.h, level, tol, ibuffer,
                                        buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
               self.h, "tag_level")
        out, off = [], 0
        for d, n in zip(pats, sizes):
            out.append(buf[off:off + n].reshape(tuple(d["mx"][:nd]), order="F"))
            off += n
        return out

    def init_patch(self, patch: int):
        """InitFields of a refined patch from its parent (mass-corrected
        prolongation; qold = q)."""
        from . import _check, lib
        _check(lib().bsam_gpu_init_patch(self.h, patch), self.h, "init_patch")

    def get_q(self, patch: int) -> np.ndarray:
        from . import FIELD_Q, _check, _dp, lib
        d = self.hier.descs[patch]
        shape = tuple(m + 2 for m in d["mx"][:self.hier.ndims]) + (2,)
        out = np.zeros(shape, order="F")
        _check(lib().bsam_gpu_get_field(self.h, patch, FIELD_Q, _dp(out)), self.h, "get_field")
        return out

    def get_qold(self, patch: int) -> np.ndarray:
        from . import FIELD_QOLD, _check, _dp, lib
        d = self.hier.descs[patch]
        shape = tuple(m + 2 for m in d["mx"][:self.hier.ndims]) + (2,)
        out = np.zeros(shape, order="F")
        _check(lib().bsam_gpu_get_field(self.h, patch, FIELD_QOLD, _dp(out)), self.h,
               "get_field")
        return out

    def close(self):
        from . import lib
        if getattr(self, "h", None) is not None and self.h.value:
            lib().bsam_gpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def new_subgrids(flags: np.ndarray, desfill: float, mgp: int, maxboxes: int = 4096) -> np.ndarray:
    """Berger-Rigoutsos boxes (NewSubGrids) of a patch's 0/1 flags (1:mx)^d:
    array (nbox, 3, 2) of lo/hi per dimension, in the reference's order.
    Runs in the native library (bsam_host_new_subgrids)."""
    import ctypes
    from . import BsamError, lib
    fl = np.asfortranarray(flags, dtype=np.uint8)
    nd = fl.ndim
    mx = np.array(list(fl.shape) + [1] * (3 - nd), dtype=np.int32)
    boxes = np.zeros(6 * maxboxes, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    n = lib().bsam_host_new_subgrids(nd, mx.ctypes.data_as(ip),
                                     fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                     float(desfill), int(mgp), boxes.ctypes.data_as(ip), maxboxes)
    if n < 0:
        raise BsamError(f"bsam_host_new_subgrids failed ({n})")
    return boxes[:6 * n].reshape(n, 3, 2)


def summed_area(flags: np.ndarray) -> np.ndarray:
    """Inclusive summed-area table of 0/1 flags (1:mx)^d, int32, Fortran
    order (the layout bsam_gpu_tag_level returns per patch)."""
    s = np.asarray(flags, dtype=np.int64)
    for ax in range(s.ndim):
        s = np.cumsum(s, axis=ax)
    return np.asfortranarray(s, dtype=np.int32)


def new_subgrids_sat(sat: np.ndarray, desfill: float, mgp: int,
                     maxboxes: int = 4096) -> np.ndarray:
    """new_subgrids from a patch's summed-area table of its flags
    (bsam_host_new_subgrids_sat)."""
    import ctypes
    from . import BsamError, lib
    st = np.asfortranarray(sat, dtype=np.int32)
    nd = st.ndim
    mx = np.array(list(st.shape) + [1] * (3 - nd), dtype=np.int32)
    boxes = np.zeros(6 * maxboxes, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    n = lib().bsam_host_new_subgrids_sat(nd, mx.ctypes.data_as(ip),
                                         st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                         float(desfill), int(mgp), boxes.ctypes.data_as(ip),
                                         maxboxes)
    if n < 0:
        raise BsamError(f"bsam_host_new_subgrids_sat failed ({n})")
    return boxes[:6 * n].reshape(n, 3, 2)


def _desc(level, parent, mx, mbounds, mglobal, mthbc, dx, xlower):
    return {"level": level, "parent": parent, "mx": list(mx) + [1] * (3 - len(mx)),
            "mbounds": [list(b) for b in mbounds] + [[1, 1]] * (3 - len(mbounds)),
            "mglobal": [list(b) for b in mglobal] + [[1, 1]] * (3 - len(mglobal)),
            "mthbc": list(mthbc) + [1] * (6 - len(mthbc)), "dx": dx,
            "xlower": list(xlower) + [0.0] * (3 - len(xlower))}


def build(n_root: int, boxes: list, eps: float, dt: float = 5e-5, qerrortol: float = 1e-9,
          mthbc=1, minlevel: int = 1, seed: int = 2, field: str = "drop",
          maxvcycles: int = 20, ndims: int = 2) -> Hierarchy:
    """Hierarchy on [0,1]^d (d = ndims, 2 or 3): an n_root^d root, its
    below-root levels (automatic minlevel: halve while even, at most 10
    times), and refined patches `boxes` = [(level, lo, size), ...] with lo the
    1-based global index of the patch's first cell on its level (odd in every
    dimension) and even sizes.  Each patch's parent is the patch of the level
    below that contains its footprint (the first one listed).

    Initial composition (field "drop", as the AMR benchmark configuration):
    phi0 = tanh((0.25 - r)/(sqrt(2) eps)) + 1e-3 U(-1, 1) (seeded per
    patch), c0 = (1 + phi0)/2, mu0 from the operator (workloads.initial_q);
    any other field: phi0 = 0.1 sin(2 pi x) cos(2 pi y) [cos(2 pi z)] plus
    the same noise."""
    nd = ndims
    if nd not in (2, 3):
        raise ValueError("ndims must be 2 or 3")
    h0 = 1.0 / n_root
    descs = []
    # Root (patch 0) and the below-root chain (patch l = level -l).
    nlev = 0
    if minlevel == 1:
        m = n_root
        while m % 2 == 0 and nlev < 10:
            m //= 2
            nlev += 1
    else:
        nlev = -minlevel
    sizes = [n_root // (2 ** l) for l in range(nlev + 1)]
    # Face codes of the root and the levels below it: one code for every
    # face, or one per face (x-lo, x-hi, y-lo, y-hi[, z-lo, z-hi]).
    codes = [mthbc] * (2 * nd) if isinstance(mthbc, int) else list(mthbc)[:2 * nd]
    for l in range(nlev + 1):
        n = sizes[l]
        parent = l + 1 if l < nlev else -1
        mb = [(1, n // 2)] * nd if l < nlev else [(1, n)] * nd
        descs.append(_desc(-l, parent, (n,) * nd, mb, [(1, n)] * nd, list(codes),
                           h0 * (2 ** l), (0.0,) * nd))
    # Refined patches.
    for (level, lo, size) in boxes:
        if len(lo) != nd or len(size) != nd:
            raise ValueError("box dimensionality differs from ndims")
        if level < 1 or any(x % 2 == 0 for x in lo) or any(s % 2 for s in size):
            raise ValueError("patch origin must be odd and its size even")
        nglob = n_root * 2 ** level
        glo = list(lo)
        ghi = [lo[k] + size[k] - 1 for k in range(nd)]
        if any(glo[k] < 1 or ghi[k] > nglob for k in range(nd)):
            raise ValueError("patch outside the domain")
        foot_lo = [(glo[k] + 1) // 2 for k in range(nd)]
        foot_hi = [ghi[k] // 2 for k in range(nd)]
        parent = None
        for pi, d in enumerate(descs):
            if d["level"] != level - 1:
                continue
            if all(d["mglobal"][k][0] <= foot_lo[k] and foot_hi[k] <= d["mglobal"][k][1]
                   for k in range(nd)):
                parent = pi
                break
        if parent is None:
            raise ValueError("no parent patch contains the footprint")
        pg = descs[parent]["mglobal"]
        mb = [(foot_lo[k] - pg[k][0] + 1, foot_hi[k] - pg[k][0] + 1) for k in range(nd)]
        pc = []
        for k in range(nd):
            pc.append(codes[2 * k] if glo[k] == 1 else INTERNAL)
            pc.append(codes[2 * k + 1] if ghi[k] == nglob else INTERNAL)
        h = h0 / (2 ** level)
        descs.append(_desc(level, parent, size, mb, [(glo[k], ghi[k]) for k in range(nd)],
                           pc, h, tuple((glo[k] - 1) * h for k in range(nd))))
    # Initial states.
    q0s = []
    for i, d in enumerate(descs):
        if d["level"] < 0:
            continue
        mx = d["mx"][:nd]
        h = d["dx"]
        axes = [d["xlower"][k] + (np.arange(mx[k]) + 0.5) * h for k in range(nd)]
        X = np.meshgrid(*axes, indexing="ij")
        if field == "drop":
            r = np.sqrt(sum((X[k] - 0.5) ** 2 for k in range(nd)))
            phi = np.tanh((0.25 - r) / (math.sqrt(2.0) * eps))
        else:
            phi = 0.1 * np.sin(2 * math.pi * X[0]) * np.cos(2 * math.pi * X[1])
            if nd == 3:
                phi = phi * np.cos(2 * math.pi * X[2])
        ncell = int(np.prod(mx))
        noise = W.uniform(seed * 1000 + i, ncell, -1.0, 1.0).reshape(mx, order="F")
        c0 = 0.5 * (1.0 + (phi + 1e-3 * noise))
        q0s.append(W.initial_q(nd, tuple(d["mx"]), c0.ravel(order="F"), h, eps, 1.0))
    return Hierarchy(ndims=nd, descs=descs, q0s=q0s, dt=dt, eps=eps, qerrortol=qerrortol,
                     maxvcycles=maxvcycles)


def desc_array(descs):
    """The patch table as bsam_patch_desc records."""
    from . import PatchDesc
    arr = (PatchDesc * len(descs))()
    for i, d in enumerate(descs):
        o = arr[i]
        o.level, o.parent, o.dx = d["level"], d["parent"], d["dx"]
        for k in range(3):
            o.mx[k] = d["mx"][k]
            o.xlower[k] = d["xlower"][k]
            for s in range(2):
                o.mbounds[k][s] = d["mbounds"][k][s]
                o.mglobal[k][s] = d["mglobal"][k][s]
        for f in range(6):
            o.mthbc[f] = d["mthbc"][f]
    return arr


def desc_dict(o) -> dict:
    """A bsam_patch_desc record as the dict the builders use."""
    return {"level": o.level, "parent": o.parent, "mx": list(o.mx),
            "mbounds": [list(o.mbounds[k]) for k in range(3)],
            "mglobal": [list(o.mglobal[k]) for k in range(3)], "mthbc": list(o.mthbc),
            "dx": o.dx, "xlower": list(o.xlower)}


def format_frame(path: str, nd: int, time: float, descs: list, qs: dict):
    """WriteQ's frame file from host arrays (bsam_host_format_frame): qs maps
    the index of every patch on a level >= 0 to its q with ring."""
    import ctypes
    from . import BsamError, lib
    dp = ctypes.POINTER(ctypes.c_double)
    keep = {i: np.asfortranarray(q, dtype=np.float64) for i, q in qs.items()}
    ptrs = (dp * len(descs))()
    for i in range(len(descs)):
        ptrs[i] = keep[i].ctypes.data_as(dp) if i in keep else dp()
    finest = max(d["level"] for d in descs)
    rc = lib().bsam_host_format_frame(os.fsencode(path), nd, time, finest, len(descs),
                                      desc_array(descs), ptrs)
    if rc != 0:
        raise BsamError(f"bsam_host_format_frame failed ({rc})")


def frame_path(outdir: str, nframe: int) -> str:
    """The reference's frame name: <outdir>/mNNNNN.dat."""
    return os.path.join(outdir, "m%05d.dat" % nframe)


# ---- regridding every time step --------------------------------------------------

@dataclasses.dataclass
class RegridParams:
    """The &amrdata values a regrid reads, per level 0 .. maxlevel - 1
    (lib/nodeinfodef.f90:87-103): qtolerance (tag threshold on the undivided
    gradient), ibuffer (buffer cells), desiredfillratios, minimumgridpoints."""
    maxlevel: int
    qtolerance: list
    ibuffer: list
    desfill: list
    mgp: list


class GpuBackend:
    """The engine (C ABI, FP64 form) as the regrid driver's backend: one
    handle whose hierarchy is re-set at every regrid."""

    def __init__(self, ndims: int, dt: float, eps: float, qerrortol: float, alpha: float = 1.0,
                 maxvcycles: int = 20, nsmoothingpasses: int = 2, device: int = 0):
        import ctypes
        from . import PREC_FP64, RunParams, _check, lib
        self.nd = ndims
        rp = RunParams(ndims=ndims, nrvars=2, mbc=1, maux=0, nsmoothingpasses=nsmoothingpasses,
                       maxvcycles=maxvcycles, errortype=1, precision=PREC_FP64, dt=dt,
                       qerrortol=qerrortol, alpha=alpha, eps=eps)
        self.h = ctypes.c_void_p()
        _check(lib().bsam_gpu_create(ctypes.byref(self.h), device, ctypes.byref(rp)),
               what="create")
        self.descs = []

    def _call(self, what, rc):
        from . import _check
        _check(rc, self.h, what)

    def set_hierarchy(self, descs):
        from . import lib
        self.descs = list(descs)
        self._call("set_hierarchy", lib().bsam_gpu_set_hierarchy(
            self.h, len(descs), desc_array(descs), max(d["level"] for d in descs)))

    def stash(self):
        from . import lib
        self._call("stash", lib().bsam_gpu_stash(self.h))

    def regrid(self, descs, carry, transfers):
        """The new patch table filled on the device: carried patches keep
        their state, new ones take InitFields' prolongation, then the
        stashed old grids' overlaps (bsam_gpu_regrid)."""
        import ctypes
        from . import lib
        self.descs = list(descs)
        cv = np.array(carry, dtype=np.int32)
        tv = np.array([x for pair in transfers for x in pair] or [0], dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        self._call("regrid", lib().bsam_gpu_regrid(
            self.h, len(descs), desc_array(descs), max(d["level"] for d in descs),
            cv.ctypes.data_as(ip), len(transfers), tv.ctypes.data_as(ip)))

    def write_frame(self, path, time):
        """WriteQ from the device (bsam_host_write_frame)."""
        from . import lib
        self._call("write_frame", lib().bsam_host_write_frame(
            self.h, os.fsencode(path), self.nd, time, len(self.descs), desc_array(self.descs)))

    def _shape(self, p):
        d = self.descs[p]
        return tuple(m + 2 for m in d["mx"][:self.nd]) + (2,)

    def put_q(self, p, q):
        from . import FIELD_Q, _dp, lib
        q = np.asfortranarray(q, dtype=np.float64)
        self._call("put_field", lib().bsam_gpu_put_field(self.h, p, FIELD_Q, _dp(q)))

    def get_q(self, p):
        from . import FIELD_Q, _dp, lib
        out = np.zeros(self._shape(p), order="F")
        self._call("get_field", lib().bsam_gpu_get_field(self.h, p, FIELD_Q, _dp(out)))
        return out

    def set_ghost_level(self, level):
        from . import lib
        self._call("set_ghost_level", lib().bsam_gpu_set_ghost_level(self.h, level))

    def errflags(self, p, tol):
        import ctypes
        from . import lib
        d = self.descs[p]
        out = np.zeros(tuple(d["mx"][:self.nd]), dtype=np.uint8, order="F")
        self._call("errflags", lib().bsam_gpu_errflags(
            self.h, p, tol, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return out

    def init_patch(self, p):
        from . import lib
        self._call("init_patch", lib().bsam_gpu_init_patch(self.h, p))

    def restrict_level(self, level):
        from . import lib
        self._call("restrict_level", lib().bsam_gpu_restrict_level(self.h, level))

    def fill_down(self):
        from . import lib
        self._call("fill_down", lib().bsam_gpu_fill_down(self.h))

    def copy_q_to_qold(self):
        from . import lib
        self._call("copy_q_to_qold", lib().bsam_gpu_copy_q_to_qold(self.h))

    def multigrid(self):
        import ctypes
        from . import lib
        nv, conv = ctypes.c_int(0), ctypes.c_int(0)
        res = ctypes.c_double(0.0)
        self._call("multigrid_iterations", lib().bsam_gpu_multigrid_iterations(
            self.h, ctypes.byref(nv), ctypes.byref(res), ctypes.byref(conv)))
        return nv.value, res.value

    def after_step_stats(self):
        import ctypes
        from . import lib
        out = (ctypes.c_double * 2)()
        self._call("after_step_stats", lib().bsam_gpu_after_step_stats(self.h, out))
        return out[0], out[1]

    def buffer_flags(self, descs, flags, ibuffer):
        return buffer_flags(self.nd, descs, flags, ibuffer)

    def new_subgrids(self, flags, desfill, mgp):
        return new_subgrids(flags, desfill, mgp)

    def child_desc(self, parent, parent_index, box):
        return child_desc(self.nd, parent, parent_index, box)

    def close(self):
        from . import lib
        if self.h is not None and self.h.value:
            lib().bsam_gpu_destroy(self.h)
            self.h = None


def buffer_flags(nd: int, descs: list, flags: list, ibuffer: int) -> list:
    """BufferAndList + InflateEdgeTags over one level's patches (the native
    library's bsam_host_buffer_flags); flags: one (1:mx)^d uint8 array per
    desc, buffered copies returned."""
    import ctypes
    from . import BsamError, lib
    if ibuffer <= 0 or not descs:
        return [f.copy() for f in flags]
    mx = np.array([list(d["mx"]) for d in descs], dtype=np.int32).ravel()
    mg = np.array([[v for b in d["mglobal"] for v in b] for d in descs], dtype=np.int32).ravel()
    flat = np.concatenate([np.asfortranarray(f, dtype=np.uint8).ravel(order="F") for f in flags])
    ip = ctypes.POINTER(ctypes.c_int)
    rc = lib().bsam_host_buffer_flags(nd, len(descs), mx.ctypes.data_as(ip), mg.ctypes.data_as(ip),
                                      flat.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ibuffer)
    if rc != 0:
        raise BsamError(f"bsam_host_buffer_flags failed ({rc})")
    out, off = [], 0
    for f in flags:
        out.append(flat[off:off + f.size].reshape(f.shape, order="F").copy())
        off += f.size
    return out


def child_desc(nd: int, parent: dict, parent_index: int, box) -> dict:
    """MakeNewGrid's record of the child over `box` (the native library's
    bsam_host_child_desc)."""
    import ctypes
    from . import BsamError, PatchDesc, lib
    pd, cd = PatchDesc(), PatchDesc()
    pd.level, pd.parent, pd.dx = parent["level"], parent["parent"], parent["dx"]
    for k in range(3):
        pd.mx[k] = parent["mx"][k]
        pd.xlower[k] = parent["xlower"][k]
        for s in range(2):
            pd.mbounds[k][s] = parent["mbounds"][k][s]
            pd.mglobal[k][s] = parent["mglobal"][k][s]
    for f in range(6):
        pd.mthbc[f] = parent["mthbc"][f]
    b = np.array(box, dtype=np.int32).ravel()
    rc = lib().bsam_host_child_desc(nd, ctypes.byref(pd), parent_index,
                                    b.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    ctypes.byref(cd))
    if rc != 0:
        raise BsamError(f"bsam_host_child_desc failed ({rc})")
    return {"level": cd.level, "parent": cd.parent, "mx": list(cd.mx),
            "mbounds": [list(cd.mbounds[k]) for k in range(3)],
            "mglobal": [list(cd.mglobal[k]) for k in range(3)], "mthbc": list(cd.mthbc),
            "dx": cd.dx, "xlower": list(cd.xlower)}


class RegridRun:
    """TakeTimeSteps with regridding every step (lib/bsamroutines.f90:632-762):
    AMR(rootlevel) (939-961) -- for level = 0 .. maxlevel - 1: SetGhost(level),
    EstimateLevelErrors (963-1002: RestrictSolution of the level into its
    parents, then SetErrFlagsUser and the buffer), GridAdapt (1299-1350:
    NewSubGrids per patch in ApplyOnLevel order, MakeNewGrid + InitFields per
    box, TransferValues from the level's old grids, the old grids released) --
    then FillDown on the first step, CopyQToQold, MultigridIterations.

    New grids join their level youngest first (TreeOps prepends them,
    lib/treeops.f90:339-430), so a new level lists its grids in the reverse
    of the order they were made.  The hierarchy starts from `hier` as given
    (its grids are not re-made by QInit).  `backend` does the numerics:
    GpuBackend (the engine), or any object with the same methods."""

    def __init__(self, backend, hier: Hierarchy, params: RegridParams):
        self.b = backend
        self.nd = hier.ndims
        self.prm = params
        self.descs = [dict(d) for d in hier.descs]
        self.b.set_hierarchy(self.descs)
        for p, q in zip(hier.state_patches(), hier.q0s):
            self.b.put_q(p, q)
        # BSAMSolver: SetGhost on every level, CopyQToQold (bsamroutines.f90:144-147).
        for level in range(0, max(d["level"] for d in self.descs) + 1):
            self.b.set_ghost_level(level)
        self.b.copy_q_to_qold()
        self.firstamr = True

    def levels(self):
        return sorted({d["level"] for d in self.descs})

    def step(self):
        """One time step: AMR(rootlevel), FillDown on the first step,
        CopyQToQold, MultigridIterations.  Returns (V-cycles, residual)."""
        b, nd, prm = self.b, self.nd, self.prm
        start = self.descs
        descs = start
        # The old grids of the refined levels as TransferValues reads them:
        # their interiors do not change before GridAdapt reaches their level.
        b.stash()
        b.set_ghost_level(0)  # AMR(rootlevel)
        # EstimateLevelErrors(0)'s RestrictSolution of the root into the level
        # below and that level's SetGhost are left out: the V-cycle restricts
        # the root again before it reads that level's q, and qold below the
        # root is never read.
        for L in range(0, prm.maxlevel):
            if L >= 1:
                b.restrict_level(L)  # EstimateLevelErrors(L): RestrictSolution, SetGhost(L - 1)
            lvl = [i for i, d in enumerate(descs) if d["level"] == L]
            flags = b.buffer_flags([descs[i] for i in lvl],
                                   [b.errflags(i, prm.qtolerance[L]) for i in lvl],
                                   prm.ibuffer[L])
            made = []  # GridAdapt(L): RefineGrid over the level, creation order
            for i, fl in zip(lvl, flags):
                for box in b.new_subgrids(fl, prm.desfill[L], prm.mgp[L]):
                    made.append(b.child_desc(descs[i], i, box[:nd].ravel()))
            # Levels <= L keep their grids; level L + 1 becomes the new grids,
            # youngest first; deeper levels lose their grids.
            keep = [i for i, d in enumerate(descs) if d["level"] <= L]
            index = {o: n for n, o in enumerate(keep)}
            new_descs = []
            for i in keep:
                d = dict(descs[i])
                d["parent"] = index[d["parent"]] if d["parent"] >= 0 else -1
                new_descs.append(d)
            for c in reversed(made):
                c = dict(c)
                c["parent"] = index[c["parent"]]
                new_descs.append(c)
            carry = list(keep) + [-1] * len(made)
            # TransferValues: each new grid with each old grid of its level.
            transfers = []
            for c in range(len(keep), len(new_descs)):
                dc = new_descs[c]
                for o, do in enumerate(start):
                    if do["level"] != L + 1:
                        continue
                    if all(max(dc["mglobal"][k][0], do["mglobal"][k][0])
                           <= min(dc["mglobal"][k][1], do["mglobal"][k][1]) for k in range(nd)):
                        transfers.append((c, o))
            b.regrid(new_descs, carry, transfers)
            descs = new_descs
            if not made:
                # AMR(L + 1) on an empty level: EstimateLevelErrors(L + 1)
                # still sets the ghosts of level L.
                if L + 1 < prm.maxlevel:
                    b.set_ghost_level(L)
                break
            b.set_ghost_level(L + 1)  # AMR(L + 1)
        self.descs = descs
        if self.firstamr:
            b.fill_down()
            self.firstamr = False
        b.copy_q_to_qold()
        return b.multigrid()

    def stats(self):
        """AfterStepStatistics after the step: (composite mass, composite
        Energy2D; 0 in 3D)."""
        return self.b.after_step_stats()

    def state(self):
        """q of every patch on a level >= 0 (descs order)."""
        return [(i, self.b.get_q(i)) for i, d in enumerate(self.descs) if d["level"] >= 0]


class AmrRun:
    """Time steps with regridding every step in the native host library
    (bsam_amr_*): the same sequence as RegridRun, without Python in the loop.
    The hierarchy starts from `hier` as given, on device `device`."""

    def __init__(self, hier: Hierarchy, params: RegridParams, device: int = 0):
        import ctypes
        from . import AMR_MAXLEVEL, RegridParamsC, _check, lib
        if params.maxlevel > AMR_MAXLEVEL:
            raise ValueError("maxlevel above the native limit")
        self.nd = hier.ndims
        self.b = GpuBackend(hier.ndims, hier.dt, hier.eps, hier.qerrortol, hier.alpha,
                            hier.maxvcycles, hier.nsmoothingpasses, device)
        self.a = ctypes.c_void_p()
        try:
            self.b.set_hierarchy(hier.descs)
            for p, q in zip(hier.state_patches(), hier.q0s):
                self.b.put_q(p, q)
            rp = RegridParamsC()
            rp.maxlevel = params.maxlevel
            for L in range(params.maxlevel):
                rp.ibuffer[L] = params.ibuffer[L]
                rp.minimumgridpoints[L] = params.mgp[L]
                rp.qtolerance[L] = params.qtolerance[L]
                rp.desiredfillratios[L] = params.desfill[L]
            _check(lib().bsam_amr_create(ctypes.byref(self.a), self.b.h, self.nd, ctypes.byref(rp),
                                         len(hier.descs), desc_array(hier.descs)),
                   self.b.h, "amr_create")
        except Exception:
            self.close()
            raise
        self._descs = list(hier.descs)
        self._table = None
        self.npatch = len(hier.descs)

    @property
    def descs(self) -> list:
        """The current patch table as dicts (converted on first use after a
        step)."""
        if self._descs is None:
            self._descs = [desc_dict(self._table[i]) for i in range(self.npatch)]
            self.b.descs = list(self._descs)
        return self._descs

    def table_array(self) -> np.ndarray:
        """The current patch table as a numpy structured array (no copy of
        the records into Python objects): fields level, parent, mx, ..."""
        if self._table is None:
            return np.ctypeslib.as_array(desc_array(self._descs))
        return np.ctypeslib.as_array(self._table)

    def step(self):
        """One time step (bsam_amr_step): (V-cycles, residual)."""
        import ctypes
        from . import PatchDesc, _check, lib
        nv, conv = ctypes.c_int(0), ctypes.c_int(0)
        res = ctypes.c_double(0.0)
        _check(lib().bsam_amr_step(self.a, ctypes.byref(nv), ctypes.byref(res),
                                   ctypes.byref(conv)), self.b.h, "amr_step")
        self.converged = conv.value
        self.refresh()
        return nv.value, res.value

    def refresh(self):
        """Re-reads the driver's patch table (after steps run elsewhere, such
        as in a batch)."""
        from . import PatchDesc, lib
        n = lib().bsam_amr_table(self.a, None, 0)
        arr = (PatchDesc * n)()
        lib().bsam_amr_table(self.a, arr, n)
        self._table, self.npatch, self._descs = arr, n, None

    def stats(self):
        return self.b.after_step_stats()

    PHASES = ("stash", "ghost", "tag", "cluster", "regrid", "solve")

    def profile(self) -> dict:
        """Host seconds per phase of the steps so far (bsam_amr_profile)."""
        import ctypes
        from . import lib
        out = (ctypes.c_double * len(self.PHASES))()
        n = lib().bsam_amr_profile(self.a, out, len(self.PHASES))
        return {"steps": n, **{k: out[i] for i, k in enumerate(self.PHASES)}}

    def state(self):
        """q of every patch on a level >= 0 (table order)."""
        return [(i, self.b.get_q(i)) for i, d in enumerate(self.descs) if d["level"] >= 0]

    def write_frame(self, path, time):
        _ = self.descs  # the backend's table follows the last step
        self.b.write_frame(path, time)

    def close(self):
        from . import lib
        if getattr(self, "a", None) is not None and self.a.value:
            lib().bsam_amr_destroy(self.a)
            self.a = None
        if getattr(self, "b", None) is not None:
            self.b.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def config2(sustained: bool = False, seed: int = 2):
    """The 2D AMR workload: a 256^2 root on [0,1]^2 with two refined levels,
    eps = 0.005, dt = 5e-5, residual 1e-9, the circular drop
    phi0 = tanh((0.25 - r)/(sqrt(2) eps)) + 1e-3 U(-1, 1), regridded every
    step: ibuffer 1, desiredfillratios 0.9, minimumgridpoints 8, and the tag
    threshold |grad phi| > 0.5/eps on the undivided central gradient of c
    (qtolerance = 0.5 h / eps per level).

    With c = (1 + phi)/2 and the reference's potential (alpha = 1) the
    equilibrium interface is twice as wide as the initial one
    (max |grad phi| = 1/(2 sqrt(2) eps), about 0.35/eps), so the refined
    levels disappear once the initial profile has relaxed (two steps).
    sustained=True halves the threshold (0.25/eps), which keeps about 40
    level-1 and 100 level-2 grids on the interface every step."""
    hier = build(256, [], eps=0.005, dt=5e-5, qerrortol=1e-9, field="drop", seed=seed)
    k = 0.25 if sustained else 0.5
    tol = [k * (1.0 / 256) / 0.005, k * (1.0 / 512) / 0.005]
    return hier, RegridParams(maxlevel=2, qtolerance=tol, ibuffer=[1, 1], desfill=[0.9, 0.9],
                              mgp=[8, 8])


def request_params(n_root: int, eps: float, maxlevel: int) -> RegridParams:
    """Regridding of a served AMR request: the AMR workload's settings on an
    n_root^2 root (tag threshold |grad phi| > 0.5/eps, qtolerance = 0.5 h /
    eps per level; ibuffer 1, desiredfillratios 0.9, minimumgridpoints 8)."""
    tol = [0.5 * (1.0 / (n_root * 2 ** l)) / eps for l in range(maxlevel)]
    return RegridParams(maxlevel=maxlevel, qtolerance=tol, ibuffer=[1] * maxlevel,
                        desfill=[0.9] * maxlevel, mgp=[8] * maxlevel)


def request_run(prob, device: int = 0) -> "AmrRun":
    """The native driver of a served 2D request with refined levels
    (prob.maxlevel >= 1): the circular drop seeded by prob.seed on a
    prob.mx[0]^2 root with the request's regridding settings."""
    n = int(prob.mx[0])
    hier = build(n, [], eps=float(prob.eps), dt=float(prob.dt), qerrortol=float(prob.qerrortol),
                 field="drop", seed=int(prob.seed), maxvcycles=int(prob.maxvcycles))
    return AmrRun(hier, request_params(n, float(prob.eps), int(prob.maxlevel)), device)


def solve_request(prob, device: int = 0, keep_q: bool = False) -> dict:
    """One served 2D request with refined levels (prob.maxlevel >= 1): the
    circular drop seeded by prob.seed on a prob.mx[0]^2 root, prob.nsteps
    time steps regridded every step in the native driver (FP64).  Returns the
    per-step V-cycles, residuals and convergence flags, the largest patch
    count, and (keep_q) the final q of every patch on a level >= 0."""
    nsteps = int(prob.nsteps)
    nvc = np.zeros(nsteps, dtype=np.int32)
    res = np.zeros(nsteps)
    conv = np.zeros(nsteps, dtype=np.int32)
    most = 0
    with request_run(prob, device) as r:
        for k in range(nsteps):
            nvc[k], res[k] = r.step()
            conv[k] = r.converged
            most = max(most, r.npatch)
        out = {"nvcycles": nvc, "residual": res, "converged": conv, "patches_max": most}
        if keep_q:
            out["q"] = r.state()
            out["descs"] = list(r.descs)
    return out
