"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module.  See bsam_oracle.h for what the oracle restates and how far its
parity is pinned.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libbsam_oracle.so")


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("ndims", ctypes.c_int32), ("mx", ctypes.c_int32 * 3), ("mthbc", ctypes.c_int32 * 6),
        ("minlevel", ctypes.c_int32), ("nsmoothingpasses", ctypes.c_int32),
        ("maxvcycles", ctypes.c_int32), ("errortype", ctypes.c_int32), ("pad_", ctypes.c_int32),
        ("xlower", ctypes.c_double * 3), ("xupper", ctypes.c_double * 3),
        ("dt", ctypes.c_double), ("qerrortol", ctypes.c_double),
        ("alpha", ctypes.c_double), ("eps", ctypes.c_double),
    ]


class OrcPatch(ctypes.Structure):
    _fields_ = [
        ("level", ctypes.c_int32), ("parent", ctypes.c_int32), ("mx", ctypes.c_int32 * 3),
        ("mbounds", (ctypes.c_int32 * 2) * 3), ("mglobal", (ctypes.c_int32 * 2) * 3),
        ("mthbc", ctypes.c_int32 * 6), ("dx", ctypes.c_double), ("xlower", ctypes.c_double * 3),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


# The timing build: the same source for speed on the machine that runs it
# (g++ -O3 -march=native, multiply-adds contracted), as a Fortran build of the
# reference with gfortran -O3 -march=native would be.  It is not the parity
# build (contraction changes the last bits), so nothing checks results with
# it.  It is compiled on the host that times it, into a file named after that
# host's CPU, so that a build made for another CPU is never loaded.
TIMING_FLAGS = ["-O3", "-march=native", "-ffp-contract=fast", "-std=c++17", "-fPIC", "-shared"]


def _cpu_key() -> str:
    import hashlib
    import platform
    desc = platform.machine()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    desc += line
                if line.startswith("flags"):
                    break
    except OSError:
        pass
    return hashlib.sha1(desc.encode()).hexdigest()[:12]


def build_timing() -> str:
    """Compile the timing build for this host (no-op when present); returns
    its path.  Load it with use_library(path) before the first lib() call."""
    out_dir = os.path.join(_HERE, "_timing")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, f"libbsam_oracle_native_{_cpu_key()}.so")
    src = os.path.join(_HERE, "bsam_oracle.cpp")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        tmp = out + f".{os.getpid()}.tmp"
        subprocess.run([os.environ.get("CXX", "g++"), *TIMING_FLAGS, "-o", tmp, src], check=True)
        os.replace(tmp, out)
    return out


_lib = None
_lib_path = None


def use_library(path: str) -> None:
    """Selects the shared library lib() loads (default: the parity build)."""
    global _lib_path
    if _lib is not None and path != _lib_path:
        raise RuntimeError("the oracle library is already loaded")
    _lib_path = path


def lib():
    global _lib
    if _lib is None:
        path = _lib_path or _LIB
        if path == _LIB and not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_run_uniform.argtypes = [ctypes.POINTER(OrcParams), dp, ctypes.c_int, dp, ip, dp, dp, dp]
        L.orc_run_uniform.restype = ctypes.c_int
        L.orc_minlevel.argtypes = [ctypes.POINTER(OrcParams)]
        L.orc_relax_grid.argtypes = [ctypes.c_int, ip, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp]
        L.orc_operator.argtypes = [ctypes.c_int, ip, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, dp, dp]
        L.orc_restriction.argtypes = [ctypes.c_int, ip, ctypes.c_int, dp, dp]
        L.orc_prolongation_p1.argtypes = [ctypes.c_int, ip, ctypes.c_int, dp, dp]
        L.orc_setbc.argtypes = [ctypes.c_int, ip, ctypes.c_int, ip, dp]
        L.orc_setbc.restype = ctypes.c_int
        L.orc_source.argtypes = [ctypes.c_int, ip, ctypes.c_double, dp, dp]
        L.orc_energy2d.argtypes = [ip, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]
        L.orc_energy2d.restype = ctypes.c_double
        L.orc_run_hier.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int,
                                   ctypes.POINTER(OrcPatch), dp, ctypes.c_int, dp, ip, dp]
        L.orc_run_hier.restype = ctypes.c_int
        L.orc_interpolate2d.argtypes = [ip, ctypes.c_int, ip, ip, ctypes.c_int, dp, ip, dp]
        L.orc_interpolate3d.argtypes = [ip, ctypes.c_int, ip, ip, ctypes.c_int, dp, ip, dp]
        L.orc_errflags.argtypes = [ctypes.c_int, ip, ctypes.c_double, dp, ip]
        L.orc_prolong_mc.argtypes = [ctypes.c_int, ip, ctypes.c_int, dp, dp]
        L.orc_new_subgrids.argtypes = [ctypes.c_int, ip, ip, ctypes.c_double, ctypes.c_int, ip,
                                       ctypes.c_int]
        L.orc_new_subgrids.restype = ctypes.c_int
        L.orc_hier_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int,
                                      ctypes.POINTER(OrcPatch)]
        L.orc_hier_create.restype = ctypes.c_void_p
        L.orc_hier_destroy.argtypes = [ctypes.c_void_p]
        L.orc_hier_q.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, ctypes.c_int]
        for name in ("orc_hier_set_ghost", "orc_hier_restrict_level"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int]
        for name in ("orc_hier_fill_down", "orc_hier_copy_q_to_qold"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.orc_hier_multigrid.argtypes = [ctypes.c_void_p, ip, dp]
        L.orc_hier_after_step.argtypes = [ctypes.c_void_p, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def params_of(prob) -> OrcParams:
    p = OrcParams()
    p.ndims = prob.ndims
    for n in range(3):
        p.mx[n] = prob.mx[n] if n < prob.ndims else 1
        p.xlower[n] = 0.0
        p.xupper[n] = prob.xupper[n]
    for f in range(6):
        p.mthbc[f] = prob.mthbc[f]
    p.minlevel = prob.minlevel
    p.nsmoothingpasses = prob.nsmoothingpasses
    p.maxvcycles = prob.maxvcycles
    p.errortype = 1
    p.dt = prob.dt
    p.qerrortol = prob.qerrortol
    p.alpha = prob.alpha
    p.eps = prob.eps
    return p


def _patch_table(descs):
    arr = (OrcPatch * len(descs))()
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


def run_hier(hier, nsteps):
    """Oracle time stepping on a fixed hierarchy (bsam_b200.amr.Hierarchy):
    returns the final q of every patch on a level >= 0, V-cycles and final
    residual per step."""
    L = lib()
    n = len(hier.descs)
    arr = _patch_table(hier.descs)
    p = OrcParams()
    p.ndims = hier.ndims
    p.nsmoothingpasses = hier.nsmoothingpasses
    p.maxvcycles = hier.maxvcycles
    p.errortype = 1
    p.dt, p.qerrortol, p.alpha, p.eps = hier.dt, hier.qerrortol, hier.alpha, hier.eps
    q0 = np.concatenate([np.asfortranarray(q).ravel(order="F") for q in hier.q0s])
    qout = np.zeros_like(q0)
    nvc = np.zeros(nsteps, dtype=np.int32)
    res = np.zeros(nsteps)
    rc = L.orc_run_hier(ctypes.byref(p), n, arr, _dp(q0), nsteps, _dp(qout), _ip(nvc), _dp(res))
    if rc != 0:
        raise RuntimeError(f"orc_run_hier failed: {rc}")
    out, off = [], 0
    for q in hier.q0s:
        out.append(qout[off:off + q.size].reshape(q.shape, order="F"))
        off += q.size
    return {"q": out, "nvcycles": nvc, "residual": res}


def interpolate2d(qf, qc, mbounds, mthbc, ipass):
    """Interpolate2D on copies of qf (0:mx+1)^2 x nv and qc (parent)."""
    qf = np.array(qf, dtype=np.float64, order="F", copy=True)
    qc = np.asfortranarray(qc, dtype=np.float64)
    mx = np.array([qf.shape[0] - 2, qf.shape[1] - 2], dtype=np.int32)
    pmx = np.array([qc.shape[0] - 2, qc.shape[1] - 2], dtype=np.int32)
    mb = np.array(mbounds, dtype=np.int32)
    bc = np.array(mthbc, dtype=np.int32)
    lib().orc_interpolate2d(_ip(mx), qf.shape[2], _ip(mb), _ip(bc), ipass, _dp(qf), _ip(pmx),
                            _dp(qc))
    return qf


def interpolate3d(qf, qc, mbounds, mthbc, ipass):
    """Interpolate3D on copies of qf (0:mx+1)^3 x nv and qc (parent)."""
    qf = np.array(qf, dtype=np.float64, order="F", copy=True)
    qc = np.asfortranarray(qc, dtype=np.float64)
    mx = np.array([qf.shape[d] - 2 for d in range(3)], dtype=np.int32)
    pmx = np.array([qc.shape[d] - 2 for d in range(3)], dtype=np.int32)
    mb = np.array(mbounds, dtype=np.int32)
    bc = np.array(mthbc, dtype=np.int32)
    lib().orc_interpolate3d(_ip(mx), qf.shape[3], _ip(mb), _ip(bc), ipass, _dp(qf), _ip(pmx),
                            _dp(qc))
    return qf


def errflags(c, tol):
    """SetErrFlagsUser of c with its ring (shape mx + 2 per dimension)."""
    c = np.asfortranarray(c, dtype=np.float64)
    nd = c.ndim
    mx = np.array([s - 2 for s in c.shape] + [1] * (3 - nd), dtype=np.int32)
    out = np.zeros(tuple(mx[:nd]), dtype=np.int32, order="F")
    lib().orc_errflags(nd, _ip(mx), tol, _dp(c), _ip(out))
    return out


def prolong_mc(nd, a):
    """Bi/TriLinProlongationP1MC of a (0:cmx+1)^d x nv."""
    a = np.asfortranarray(a, dtype=np.float64)
    cmx = np.array([a.shape[k] - 2 for k in range(nd)] + [1] * (3 - nd), dtype=np.int32)
    out = np.zeros(tuple(2 * cmx[k] + 2 for k in range(nd)) + (a.shape[nd],), order="F")
    lib().orc_prolong_mc(nd, _ip(cmx), a.shape[nd], _dp(a), _dp(out))
    return out


def new_subgrids(flags, desfill, mgp, maxboxes=4096):
    """NewSubGrids boxes of 0/1 flags (1:mx)^d: array (nbox, 3, 2)."""
    fl = np.asfortranarray(flags, dtype=np.int32)
    nd = fl.ndim
    mx = np.array(list(fl.shape) + [1] * (3 - nd), dtype=np.int32)
    boxes = np.zeros(maxboxes * 6, dtype=np.int32)
    n = lib().orc_new_subgrids(nd, _ip(mx), _ip(fl), desfill, mgp, _ip(boxes), maxboxes)
    if n < 0:
        raise RuntimeError("too many boxes")
    return boxes[:6 * n].reshape(n, 3, 2)


def run_uniform(prob, nsteps=None, keep_steps=True, q0=None, final_q=False):
    """Run the oracle time loop.  Returns a dict with q per step (Fortran
    layout with ring), V-cycle counts, final residuals, traces and mass;
    final_q (with keep_steps=False) adds the last step's q as "q_final"."""
    L = lib()
    nsteps = prob.nsteps if nsteps is None else nsteps
    p = params_of(prob)
    q0 = prob.q0() if q0 is None else q0
    q0 = np.asfortranarray(q0, dtype=np.float64)
    qsize = q0.size
    if final_q and not keep_steps:
        out = run_uniform(prob, nsteps=nsteps, keep_steps=True, q0=q0)
        out["q_final"] = out["q"][-1]
        out["q"] = None
        return out
    q_steps = np.zeros((nsteps,) + q0.shape, dtype=np.float64) if keep_steps else None
    buf = np.zeros(nsteps * qsize) if keep_steps else None
    nvc = np.zeros(nsteps, dtype=np.int32)
    rfin = np.zeros(nsteps)
    tr = np.zeros(nsteps * prob.maxvcycles)
    mass = np.zeros(nsteps)
    rc = L.orc_run_uniform(ctypes.byref(p), _dp(q0.ravel(order="F")), nsteps,
                           _dp(buf) if keep_steps else None, _ip(nvc), _dp(rfin), _dp(tr), _dp(mass))
    if rc != 0:
        raise RuntimeError(f"orc_run_uniform failed: {rc}")
    if keep_steps:
        for s in range(nsteps):
            q_steps[s] = buf[s * qsize:(s + 1) * qsize].reshape(q0.shape, order="F")
    return {"q": q_steps, "nvcycles": nvc, "residual": rfin,
            "trace": tr.reshape(nsteps, prob.maxvcycles), "mass": mass}


def relax_grid(ndims, mx, h, dt, alpha, eps, ipass, q, f):
    q = np.array(q, dtype=np.float64, order="F", copy=True)
    f = np.asfortranarray(f, dtype=np.float64)
    mxa = np.array(list(mx) + [1] * (3 - len(mx)), dtype=np.int32)
    lib().orc_relax_grid(ndims, _ip(mxa), h, dt, alpha, eps, ipass,
                         q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _dp(f))
    return q


def operator(ndims, mx, h, dt, alpha, eps, q):
    q = np.asfortranarray(q, dtype=np.float64)
    mxa = np.array(list(mx) + [1] * (3 - len(mx)), dtype=np.int32)
    res = np.zeros(tuple(mx[:ndims]) + (2,), order="F")
    lib().orc_operator(ndims, _ip(mxa), h, dt, alpha, eps, _dp(q), _dp(res))
    return res


def restriction(ndims, a):
    a = np.asfortranarray(a, dtype=np.float64)
    mx = a.shape[:ndims]
    nv = a.shape[ndims]
    mxa = np.array(list(mx) + [1] * (3 - ndims), dtype=np.int32)
    out = np.zeros(tuple(m // 2 for m in mx) + (nv,), order="F")
    lib().orc_restriction(ndims, _ip(mxa), nv, _dp(a), _dp(out))
    return out


def prolongation_p1(ndims, a):
    a = np.asfortranarray(a, dtype=np.float64)
    cmx = [s - 2 for s in a.shape[:ndims]]
    nv = a.shape[ndims]
    ca = np.array(cmx + [1] * (3 - ndims), dtype=np.int32)
    out = np.zeros(tuple(2 * c + 2 for c in cmx) + (nv,), order="F")
    lib().orc_prolongation_p1(ndims, _ip(ca), nv, _dp(a), _dp(out))
    return out


def setbc(ndims, q, mthbc):
    q = np.array(q, dtype=np.float64, order="F", copy=True)
    mx = [s - 2 for s in q.shape[:ndims]]
    nv = q.shape[ndims]
    mxa = np.array(mx + [1] * (3 - ndims), dtype=np.int32)
    bc = np.array(list(mthbc) + [1] * (6 - len(mthbc)), dtype=np.int32)
    rc = lib().orc_setbc(ndims, _ip(mxa), nv, _ip(bc), _dp(q))
    if rc:
        raise ValueError("unsupported boundary code")
    return q


def source(ndims, alpha, qold):
    qold = np.asfortranarray(qold, dtype=np.float64)
    mx = [s - 2 for s in qold.shape[:ndims]]
    mxa = np.array(mx + [1] * (3 - ndims), dtype=np.int32)
    f = np.zeros(tuple(mx) + (2,), order="F")
    lib().orc_source(ndims, _ip(mxa), alpha, _dp(qold), _dp(f))
    return f


def energy2d(h, alpha, eps, c):
    c = np.asfortranarray(c, dtype=np.float64)
    mxa = np.array([c.shape[0] - 2, c.shape[1] - 2, 1], dtype=np.int32)
    return lib().orc_energy2d(_ip(mxa), h, alpha, eps, _dp(c))


# ---- regridding: the oracle side of a regrid run ------------------------------------

def buffer_flags(nd, descs, flags, ibuffer):
    """BufferAndList (lib/bsamroutines.f90:1159-1206) of every patch of a
    level in ApplyOnLevel order, then InflateEdgeTags (1208-1241) with
    BufferTaggedCells (1243-1284): a flagged cell whose buffer box lies inside
    its patch flags that box there; one whose box crosses the patch's edge is
    listed by global index, and each listed cell (last listed first) flags
    its box, clipped, on every patch of the level.  Non-periodic boundaries
    only.  flags: (1:mx)^d 0/1 arrays; returns buffered copies."""
    out = [np.array(f, dtype=np.int32, copy=True) for f in flags]
    if ibuffer <= 0:
        return out
    listed = []
    for d, f in zip(descs, out):
        tmp = f.copy()
        mx = d["mx"][:nd]
        for flat in range(tmp.size):
            idx = np.unravel_index(flat, tmp.shape, order="F")
            if tmp[idx] != 1:
                continue
            lo = [idx[k] + 1 - ibuffer for k in range(nd)]
            hi = [idx[k] + 1 + ibuffer for k in range(nd)]
            if any(lo[k] < 1 or hi[k] > mx[k] for k in range(nd)):
                listed.append([idx[k] + 1 + d["mglobal"][k][0] - 1 for k in range(nd)])
            else:
                f[tuple(slice(lo[k] - 1, hi[k]) for k in range(nd))] = 1
    for cell in reversed(listed):
        for d, f in zip(descs, out):
            lo = [max(cell[k] - ibuffer, d["mglobal"][k][0]) for k in range(nd)]
            hi = [min(cell[k] + ibuffer, d["mglobal"][k][1]) for k in range(nd)]
            if any(hi[k] < lo[k] for k in range(nd)):
                continue
            f[tuple(slice(lo[k] - d["mglobal"][k][0], hi[k] - d["mglobal"][k][0] + 1)
                    for k in range(nd))] = 1
    return out


def child_desc(nd, parent, parent_index, box):
    """MakeNewGrid's geometry (lib/bsamroutines.f90:1582-1684) of the child of
    `parent` over index box `box` = [lo1, hi1, lo2, hi2(, lo3, hi3)]."""
    internal = 999
    b = [(int(box[2 * k]), int(box[2 * k + 1])) for k in range(nd)]
    mx = [2 * (b[k][1] - b[k][0] + 1) for k in range(nd)] + [1] * (3 - nd)
    mg = []
    for k in range(nd):
        glo = parent["mglobal"][k][0] + b[k][0] - 1
        ghi = glo + b[k][1] - b[k][0]
        mg.append([(glo - 1) * 2 + 1, ghi * 2])
    codes = [internal] * 6
    for k in range(nd):
        if parent["mthbc"][2 * k] < internal and b[k][0] == 1:
            codes[2 * k] = parent["mthbc"][2 * k]
        if parent["mthbc"][2 * k + 1] < internal and b[k][1] == parent["mx"][k]:
            codes[2 * k + 1] = parent["mthbc"][2 * k + 1]
    return {"level": parent["level"] + 1, "parent": parent_index, "mx": mx,
            "mbounds": [list(x) for x in b] + [[1, 1]] * (3 - nd),
            "mglobal": mg + [[1, 1]] * (3 - nd), "mthbc": codes,
            "dx": parent["dx"] / 2.0,
            "xlower": [float(b[k][0] - 1) * parent["dx"] + parent["xlower"][k] for k in range(nd)]
            + [0.0] * (3 - nd)}


class OracleBackend:
    """The regrid driver's numerics on the oracle: a held hierarchy
    (orc_hier_*), SetErrFlagsUser, the mass-corrected prolongation of
    InitFields, Berger-Rigoutsos, the buffer and MakeNewGrid's geometry
    above."""

    def __init__(self, ndims, dt, eps, qerrortol, alpha=1.0, maxvcycles=20, nsmoothingpasses=2):
        self.nd = ndims
        p = OrcParams()
        p.ndims = ndims
        p.nsmoothingpasses = nsmoothingpasses
        p.maxvcycles = maxvcycles
        p.errortype = 1
        p.dt, p.qerrortol, p.alpha, p.eps = dt, qerrortol, alpha, eps
        self.p = p
        self.h = None
        self.descs = []

    def set_hierarchy(self, descs):
        self.close()
        self.descs = list(descs)
        h = lib().orc_hier_create(ctypes.byref(self.p), len(descs), _patch_table(descs))
        if not h:
            raise RuntimeError("orc_hier_create failed")
        self.h = ctypes.c_void_p(h)

    def _shape(self, i):
        return tuple(m + 2 for m in self.descs[i]["mx"][:self.nd]) + (2,)

    def put_q(self, i, q):
        q = np.asfortranarray(q, dtype=np.float64).copy(order="F")
        if lib().orc_hier_q(self.h, i, _dp(q), 1) != 0:
            raise RuntimeError("orc_hier_q")

    def get_q(self, i):
        out = np.zeros(self._shape(i), order="F")
        if lib().orc_hier_q(self.h, i, _dp(out), 0) != 0:
            raise RuntimeError("orc_hier_q")
        return out

    def _rc(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed: {rc}")

    def set_ghost_level(self, level):
        self._rc(lib().orc_hier_set_ghost(self.h, level), "set_ghost")

    def restrict_level(self, level):
        self._rc(lib().orc_hier_restrict_level(self.h, level), "restrict_level")

    def fill_down(self):
        self._rc(lib().orc_hier_fill_down(self.h), "fill_down")

    def copy_q_to_qold(self):
        self._rc(lib().orc_hier_copy_q_to_qold(self.h), "copy_q_to_qold")

    def multigrid(self):
        nv = np.zeros(1, dtype=np.int32)
        res = np.zeros(1)
        self._rc(lib().orc_hier_multigrid(self.h, _ip(nv), _dp(res)), "multigrid")
        return int(nv[0]), float(res[0])

    def stash(self):
        """q of every refined patch, kept aside for the transfers."""
        self._stash = [(d, self.get_q(i) if d["level"] >= 1 else None)
                       for i, d in enumerate(self.descs)]

    def regrid(self, descs, carry, transfers):
        """The new table: carried patches keep q (held in the host), new
        grids take InitFields' prolongation in table order, then the
        stashed old grids' interiors over the overlaps (TransferOverlap,
        lib/bsamroutines.f90:1832-1867)."""
        kept = {i: self.get_q(o) for i, o in enumerate(carry) if o >= 0}
        self.set_hierarchy(descs)
        for i, q in kept.items():
            self.put_q(i, q)
        for i, o in enumerate(carry):
            if o < 0:
                self.init_patch(i)
        nd = self.nd
        for c, o in transfers:
            dc = descs[c]
            do, qo = self._stash[o]
            lo = [max(dc["mglobal"][k][0], do["mglobal"][k][0]) for k in range(nd)]
            hi = [min(dc["mglobal"][k][1], do["mglobal"][k][1]) for k in range(nd)]
            if any(hi[k] < lo[k] for k in range(nd)):
                continue
            qc = self.get_q(c)
            ts = tuple(slice(lo[k] - dc["mglobal"][k][0] + 1, hi[k] - dc["mglobal"][k][0] + 2)
                       for k in range(nd))
            ss = tuple(slice(lo[k] - do["mglobal"][k][0] + 1, hi[k] - do["mglobal"][k][0] + 2)
                       for k in range(nd))
            qc[ts] = qo[ss]
            self.put_q(c, qc)

    def after_step_stats(self):
        out = np.zeros(2)
        self._rc(lib().orc_hier_after_step(self.h, _dp(out)), "after_step")
        return float(out[0]), float(out[1])

    def errflags(self, i, tol):
        q = self.get_q(i)
        return errflags(q[..., 0], tol).astype(np.uint8)

    def init_patch(self, i):
        d = self.descs[i]
        par = self.get_q(d["parent"])
        sl = tuple(slice(d["mbounds"][k][0] - 1, d["mbounds"][k][1] + 2) for k in range(self.nd))
        self.put_q(i, prolong_mc(self.nd, par[sl + (slice(None),)]))

    def buffer_flags(self, descs, flags, ibuffer):
        return [f.astype(np.uint8) for f in buffer_flags(self.nd, descs, flags, ibuffer)]

    def new_subgrids(self, flags, desfill, mgp):
        return new_subgrids(flags, desfill, mgp)

    def child_desc(self, parent, parent_index, box):
        return child_desc(self.nd, parent, parent_index, box)

    def close(self):
        if self.h is not None:
            lib().orc_hier_destroy(self.h)
            self.h = None


# ---- frame output ---------------------------------------------------------------

def _f(x, w, d):
    """Fortran Fw.d output."""
    return "%*.*f" % (w, d, x)


def _es(x, w, d):
    """Fortran ESw.d output: d.ddd...E+nn, a three-digit exponent without
    the E."""
    if x == 0.0:
        m, e = ("-" if np.signbit(x) else "") + "0." + "0" * d, 0
    else:
        t = "%.*e" % (d, x)
        mant, ex = t.split("e")
        m, e = mant, int(ex)
    es = ("E%+03d" % e) if abs(e) < 100 else ("%+04d" % e)
    s = m + es
    return " " * max(0, w - len(s)) + s


def format_frame(nd, time, descs, qs):
    """WriteQ (lib/bsaminputoutput.f90:51-76) with OutputQ (78-131) and
    WriteQ2D/3D (133-172): the text of a frame file.  descs: the patch table;
    qs: patch index -> q with ring (levels >= 0).  xupper as MakeNewGrid sets
    it (mbounds(:,2) * parent dx + parent xlower), xlower + mx dx on the
    root."""
    finest = max(d["level"] for d in descs)
    out = [_f(time, 25, 12), "%3d" % finest]
    for level in range(0, finest + 1):
        for i, d in enumerate(descs):
            if d["level"] != level:
                continue
            out.append("  ")
            out.append("%3d %3d %3d %3d" % (level, nd, 2, 2))
            if level == 0:
                xu = [d["xlower"][k] + d["mx"][k] * d["dx"] for k in range(nd)]
            else:
                p = descs[d["parent"]]
                xu = [float(d["mbounds"][k][1]) * p["dx"] + p["xlower"][k] for k in range(nd)]
            out.append(" ".join(_f(d["dx"], 25, 12) for _ in range(nd)))
            out.append(" ".join(_f(d["xlower"][k], 25, 12) for k in range(nd)))
            out.append(" ".join(_f(xu[k], 25, 12) for k in range(nd)))
            out.append(" ".join("%8d" % d["mx"][k] for k in range(nd)))
            out.append(" ".join("%8d" % d["mglobal"][k][s] for k in range(nd) for s in range(2)))
            q = np.asarray(qs[i])
            flat = q.reshape(-1, 2, order="F")
            for c in range(flat.shape[0]):
                if nd == 2:
                    out.append("  ".join(_es(v, 20, 12) for v in flat[c]))
                else:
                    out.append("  ".join(_f(v, 25, 12) for v in flat[c]))
    return "\n".join(out) + "\n"
