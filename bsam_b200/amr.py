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


def _desc(level, parent, mx, mbounds, mglobal, mthbc, dx, xlower):
    return {"level": level, "parent": parent, "mx": list(mx) + [1] * (3 - len(mx)),
            "mbounds": [list(b) for b in mbounds] + [[1, 1]] * (3 - len(mbounds)),
            "mglobal": [list(b) for b in mglobal] + [[1, 1]] * (3 - len(mglobal)),
            "mthbc": list(mthbc) + [1] * (6 - len(mthbc)), "dx": dx,
            "xlower": list(xlower) + [0.0] * (3 - len(xlower))}


def build(n_root: int, boxes: list, eps: float, dt: float = 5e-5, qerrortol: float = 1e-9,
          mthbc: int = 1, minlevel: int = 1, seed: int = 2, field: str = "drop",
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
    for l in range(nlev + 1):
        n = sizes[l]
        parent = l + 1 if l < nlev else -1
        mb = [(1, n // 2)] * nd if l < nlev else [(1, n)] * nd
        descs.append(_desc(-l, parent, (n,) * nd, mb, [(1, n)] * nd, [mthbc] * (2 * nd),
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
        codes = []
        for k in range(nd):
            codes.append(mthbc if glo[k] == 1 else INTERNAL)
            codes.append(mthbc if ghi[k] == nglob else INTERNAL)
        h = h0 / (2 ** level)
        descs.append(_desc(level, parent, size, mb, [(glo[k], ghi[k]) for k in range(nd)],
                           codes, h, tuple((glo[k] - 1) * h for k in range(nd))))
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
