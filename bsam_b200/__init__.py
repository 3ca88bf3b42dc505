"""bsam_b200 -- B200-native FAS multigrid V-cycle for BSAM's Cahn-Hilliard module.

The compute path is the native library libbsam_gpu.so (CUDA sm_100a kernels
behind the C ABI declared in include/bsam_gpu.h, plus the C++ host driver of
include/bsam_host.h).  This module binds that ABI with ctypes.  There is no
CPU fallback: if the library is missing or no CUDA device is usable, every
entry point raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import workloads  # noqa: F401  (re-exported)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbsam_gpu.so")

FIELD_Q, FIELD_QOLD, FIELD_F = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1


class BsamError(RuntimeError):
    pass


class RunParams(ctypes.Structure):
    _fields_ = [
        ("ndims", ctypes.c_int32), ("nrvars", ctypes.c_int32), ("mbc", ctypes.c_int32),
        ("maux", ctypes.c_int32), ("nsmoothingpasses", ctypes.c_int32),
        ("maxvcycles", ctypes.c_int32), ("errortype", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("dt", ctypes.c_double), ("qerrortol", ctypes.c_double),
        ("alpha", ctypes.c_double), ("eps", ctypes.c_double),
    ]


class PatchDesc(ctypes.Structure):
    _fields_ = [
        ("level", ctypes.c_int32), ("parent", ctypes.c_int32), ("mx", ctypes.c_int32 * 3),
        ("mbounds", (ctypes.c_int32 * 2) * 3), ("mglobal", (ctypes.c_int32 * 2) * 3),
        ("mthbc", ctypes.c_int32 * 6), ("dx", ctypes.c_double), ("xlower", ctypes.c_double * 3),
    ]


class HostGrid(ctypes.Structure):
    _fields_ = [
        ("ndims", ctypes.c_int32), ("mx", ctypes.c_int32 * 3), ("mthbc", ctypes.c_int32 * 6),
        ("minlevel", ctypes.c_int32), ("pad_", ctypes.c_int32),
        ("xlower", ctypes.c_double * 3), ("xupper", ctypes.c_double * 3),
    ]


_lib = None

# Every symbol the C ABI headers declare (include/bsam_gpu.h, bsam_host.h).
ABI_SYMBOLS = (
    "bsam_gpu_create", "bsam_gpu_set_hierarchy", "bsam_gpu_put_field", "bsam_gpu_get_field",
    "bsam_gpu_set_ghost", "bsam_gpu_copy_q_to_qold", "bsam_gpu_multigrid_iterations",
    "bsam_gpu_residual_trace", "bsam_gpu_mass", "bsam_gpu_energy", "bsam_gpu_destroy",
    "bsam_gpu_strerror",
    "bsam_gpu_last_error", "bsam_gpu_get_stream", "bsam_gpu_profile", "bsam_gpu_get_stats",
    "bsam_host_levels", "bsam_host_build_uniform", "bsam_host_take_time_steps",
    "bsam_gpu_resid_norm_noalloc", "bsam_gpu_set_tuning", "bsam_gpu_fill_down",
    "bsam_gpu_errflags", "bsam_gpu_init_patch", "bsam_host_new_subgrids",
    "bsam_gpu_restrict_level", "bsam_host_buffer_flags", "bsam_host_child_desc",
    "bsam_host_format_frame", "bsam_host_write_frame",
    "bsam_gpu_set_ghost_level", "bsam_gpu_after_step_stats", "bsam_gpu_stash", "bsam_gpu_regrid",
    "bsam_gpu_errflags_level", "bsam_gpu_tag_level", "bsam_host_new_subgrids_sat",
    "bsam_amr_create", "bsam_amr_step", "bsam_amr_regrid", "bsam_amr_table",
    "bsam_amr_destroy", "bsam_amr_profile",
    "bsam_batch_create", "bsam_batch_destroy", "bsam_batch_set_tuning", "bsam_batch_footprint",
    "bsam_batch_submit", "bsam_batch_advance", "bsam_batch_sync", "bsam_batch_run",
    "bsam_batch_poll", "bsam_batch_slot_phase", "bsam_batch_collect", "bsam_batch_get_stream", "bsam_batch_profile", "bsam_batch_submit_seeded", "bsam_batch_busy",
    "bsam_batch_get_stats", "bsam_batch_last_error", "bsam_batch_submit_many",
    "bsam_batch_submit_seeded_many", "bsam_batch_collect_many", "bsam_batch_submit_amr",
)


class Tuning(ctypes.Structure):
    _fields_ = [("fuse_smoother", ctypes.c_int32), ("fuse_min_n", ctypes.c_int32),
                ("chunk", ctypes.c_int32), ("bottom_cells", ctypes.c_int32),
                ("graph", ctypes.c_int32), ("reserved", ctypes.c_int32 * 3)]


AMR_MAXLEVEL = 8


class RegridParamsC(ctypes.Structure):
    """bsam_regrid_params (include/bsam_host.h)."""
    _fields_ = [("maxlevel", ctypes.c_int32), ("ibuffer", ctypes.c_int32 * AMR_MAXLEVEL),
                ("minimumgridpoints", ctypes.c_int32 * AMR_MAXLEVEL), ("pad_", ctypes.c_int32),
                ("qtolerance", ctypes.c_double * AMR_MAXLEVEL),
                ("desiredfillratios", ctypes.c_double * AMR_MAXLEVEL)]


class Stats(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64), ("smooth_stages", ctypes.c_int64),
                ("smooth_cells", ctypes.c_int64), ("smooth_ms", ctypes.c_double),
                ("smooth_bytes", ctypes.c_double)]


def lib():
    """Load libbsam_gpu.so (raises BsamError when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise BsamError(f"native library missing: {LIB_PATH} (run __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    L.bsam_gpu_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(RunParams)]
    L.bsam_gpu_set_hierarchy.argtypes = [vp, ctypes.c_int, ctypes.POINTER(PatchDesc), ctypes.c_int]
    L.bsam_gpu_put_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
    L.bsam_gpu_get_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
    L.bsam_gpu_set_ghost.argtypes = [vp]
    L.bsam_gpu_copy_q_to_qold.argtypes = [vp]
    L.bsam_gpu_multigrid_iterations.argtypes = [vp, ip, dp, ip]
    L.bsam_gpu_residual_trace.argtypes = [vp, dp, ctypes.c_int]
    L.bsam_gpu_mass.argtypes = [vp, dp]
    L.bsam_gpu_energy.argtypes = [vp, dp]
    L.bsam_gpu_errflags.argtypes = [vp, ctypes.c_int, ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_uint8)]
    L.bsam_gpu_init_patch.argtypes = [vp, ctypes.c_int]
    L.bsam_gpu_restrict_level.argtypes = [vp, ctypes.c_int]
    L.bsam_gpu_set_ghost_level.argtypes = [vp, ctypes.c_int]
    L.bsam_gpu_after_step_stats.argtypes = [vp, dp]
    L.bsam_gpu_stash.argtypes = [vp]
    L.bsam_gpu_errflags_level.argtypes = [vp, ctypes.c_int, ctypes.c_double,
                                          ctypes.POINTER(ctypes.c_uint8)]
    L.bsam_amr_create.argtypes = [ctypes.POINTER(vp), vp, ctypes.c_int,
                                  ctypes.POINTER(RegridParamsC), ctypes.c_int,
                                  ctypes.POINTER(PatchDesc)]
    L.bsam_amr_step.argtypes = [vp, ip, dp, ip]
    L.bsam_amr_regrid.argtypes = [vp]
    L.bsam_amr_table.argtypes = [vp, ctypes.POINTER(PatchDesc), ctypes.c_int]
    L.bsam_amr_destroy.argtypes = [vp]
    L.bsam_amr_destroy.restype = None
    L.bsam_amr_profile.argtypes = [vp, dp, ctypes.c_int]
    L.bsam_gpu_regrid.argtypes = [vp, ctypes.c_int, ctypes.POINTER(PatchDesc), ctypes.c_int, ip,
                                  ctypes.c_int, ip]
    L.bsam_host_buffer_flags.argtypes = [ctypes.c_int, ctypes.c_int, ip, ip,
                                         ctypes.POINTER(ctypes.c_uint8), ctypes.c_int]
    L.bsam_host_child_desc.argtypes = [ctypes.c_int, ctypes.POINTER(PatchDesc), ctypes.c_int,
                                       ip, ctypes.POINTER(PatchDesc)]
    L.bsam_host_format_frame.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, ctypes.POINTER(PatchDesc),
                                         ctypes.POINTER(dp)]
    L.bsam_host_write_frame.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int, ctypes.POINTER(PatchDesc)]
    L.bsam_host_new_subgrids.argtypes = [ctypes.c_int, ip, ctypes.POINTER(ctypes.c_uint8),
                                         ctypes.c_double, ctypes.c_int, ip, ctypes.c_int]
    L.bsam_host_new_subgrids_sat.argtypes = [ctypes.c_int, ip, ctypes.POINTER(ctypes.c_int32),
                                             ctypes.c_double, ctypes.c_int, ip, ctypes.c_int]
    L.bsam_gpu_tag_level.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_int32)]
    L.bsam_gpu_destroy.argtypes = [vp]
    L.bsam_gpu_strerror.argtypes = [ctypes.c_int]
    L.bsam_gpu_strerror.restype = ctypes.c_char_p
    L.bsam_gpu_last_error.argtypes = [vp]
    L.bsam_gpu_last_error.restype = ctypes.c_char_p
    L.bsam_gpu_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.bsam_gpu_profile.argtypes = [vp, ctypes.c_int]
    L.bsam_gpu_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.bsam_gpu_resid_norm_noalloc.argtypes = [
        ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.c_double,
        ctypes.c_double, ctypes.c_double, ctypes.c_double, vp, vp, vp, vp]
    L.bsam_gpu_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.bsam_gpu_fill_down.argtypes = [vp]
    L.bsam_host_levels.argtypes = [ctypes.POINTER(HostGrid)]
    L.bsam_host_build_uniform.argtypes = [ctypes.POINTER(HostGrid), ctypes.POINTER(PatchDesc),
                                          ctypes.c_int, ip]
    L.bsam_host_take_time_steps.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int64,
                                            ip, dp, ip, dp]
    from . import batch as _batch
    _batch.bind(L)
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc, h=None, what=""):
    if rc != 0:
        L = lib()
        msg = L.bsam_gpu_strerror(rc).decode()
        if h is not None:
            detail = L.bsam_gpu_last_error(h)
            if detail:
                msg += ": " + detail.decode()
        raise BsamError(f"{what} failed ({rc}): {msg}")


def host_grid(prob) -> HostGrid:
    g = HostGrid()
    g.ndims = prob.ndims
    for n in range(3):
        g.mx[n] = prob.mx[n] if n < prob.ndims else 1
        g.xlower[n] = 0.0
        g.xupper[n] = prob.xupper[n]
    for f in range(6):
        g.mthbc[f] = prob.mthbc[f]
    g.minlevel = prob.minlevel
    return g


def build_uniform(prob):
    """Patch descriptors of the root grid and its below-root levels."""
    L = lib()
    g = host_grid(prob)
    n = L.bsam_host_levels(ctypes.byref(g))
    if n <= 0:
        raise BsamError("invalid grid")
    arr = (PatchDesc * n)()
    npatch = ctypes.c_int(0)
    _check(L.bsam_host_build_uniform(ctypes.byref(g), arr, n, ctypes.byref(npatch)),
           what="bsam_host_build_uniform")
    return arr, npatch.value


class Solver:
    """One Cahn-Hilliard solve resident on a GPU, driven through the C ABI.

    Mirrors the reference's driver: construction = RootInit/InitSeed +
    QInit + SetGhost + CopyQToQold (lib/bsamroutines.f90:115-147); step() =
    one TakeTimeSteps iteration (CopyQToQold + MultigridIterations).
    """

    def __init__(self, prob, device: int = 0, precision: int = PREC_FP64, q0=None,
                 fuse: int = 0, fuse_min_n: int = 64, chunk: int = 0, bottom_cells: int = 0,
                 graph: int = 0):
        L = lib()
        self.prob = prob
        rp = RunParams(ndims=prob.ndims, nrvars=2, mbc=1, maux=0,
                       nsmoothingpasses=prob.nsmoothingpasses, maxvcycles=prob.maxvcycles,
                       errortype=1, precision=precision, dt=prob.dt, qerrortol=prob.qerrortol,
                       alpha=prob.alpha, eps=prob.eps)
        h = ctypes.c_void_p()
        _check(L.bsam_gpu_create(ctypes.byref(h), device, ctypes.byref(rp)), what="bsam_gpu_create")
        self.h = h
        try:
            t = Tuning(fuse_smoother=fuse, fuse_min_n=fuse_min_n, chunk=chunk,
                       bottom_cells=bottom_cells, graph=graph)
            _check(L.bsam_gpu_set_tuning(h, ctypes.byref(t)), h, "bsam_gpu_set_tuning")
            self.patches, self.npatch = build_uniform(prob)
            _check(L.bsam_gpu_set_hierarchy(h, self.npatch, self.patches, 0), h,
                   "bsam_gpu_set_hierarchy")
            q0 = prob.q0() if q0 is None else q0
            self.qshape = q0.shape
            self.put_q(q0)
            _check(L.bsam_gpu_set_ghost(h), h, "bsam_gpu_set_ghost")
            _check(L.bsam_gpu_copy_q_to_qold(h), h, "bsam_gpu_copy_q_to_qold")
        except Exception:
            self.close()
            raise

    def put_q(self, q):
        q = np.asfortranarray(q, dtype=np.float64)
        _check(lib().bsam_gpu_put_field(self.h, 0, FIELD_Q, _dp(q)), self.h, "put_field")

    def get_q(self, patch: int = 0):
        d = self.patches[patch]
        shape = tuple(d.mx[n] + 2 for n in range(self.prob.ndims)) + (2,)
        out = np.zeros(shape, order="F")
        _check(lib().bsam_gpu_get_field(self.h, patch, FIELD_Q, _dp(out)), self.h, "get_field")
        return out

    def get_f(self, patch: int = 0):
        d = self.patches[patch]
        shape = tuple(d.mx[n] for n in range(self.prob.ndims)) + (2,)
        out = np.zeros(shape, order="F")
        _check(lib().bsam_gpu_get_field(self.h, patch, FIELD_F, _dp(out)), self.h, "get_field")
        return out

    def step(self):
        """One time step: SetGhost(root) + CopyQToQold + MultigridIterations."""
        L = lib()
        _check(L.bsam_gpu_set_ghost(self.h), self.h, "set_ghost")
        _check(L.bsam_gpu_copy_q_to_qold(self.h), self.h, "copy_q_to_qold")
        nv, conv = ctypes.c_int(0), ctypes.c_int(0)
        res = ctypes.c_double(0.0)
        _check(L.bsam_gpu_multigrid_iterations(self.h, ctypes.byref(nv), ctypes.byref(res),
                                               ctypes.byref(conv)), self.h, "multigrid_iterations")
        return nv.value, res.value, bool(conv.value)

    def trace(self):
        buf = np.zeros(self.prob.maxvcycles)
        n = lib().bsam_gpu_residual_trace(self.h, _dp(buf), buf.size)
        return buf[:max(0, min(n, buf.size))]

    def mass(self) -> float:
        m = ctypes.c_double(0.0)
        _check(lib().bsam_gpu_mass(self.h, ctypes.byref(m)), self.h, "mass")
        return m.value

    def energy(self) -> float:
        """Energy2D of the root state (2D, no refined levels)."""
        e = ctypes.c_double(0.0)
        _check(lib().bsam_gpu_energy(self.h, ctypes.byref(e)), self.h, "energy")
        return e.value

    def run(self, nsteps: int, keep_steps: bool = True):
        """TakeTimeSteps through the C++ host driver."""
        L = lib()
        qsize = int(np.prod(self.qshape))
        buf = np.zeros(nsteps * qsize) if keep_steps else None
        nvc = np.zeros(nsteps, dtype=np.int32)
        res = np.zeros(nsteps)
        conv = np.zeros(nsteps, dtype=np.int32)
        mass = np.zeros(nsteps)
        ipp = ctypes.POINTER(ctypes.c_int)
        _check(L.bsam_host_take_time_steps(
            self.h, nsteps, 0, _dp(buf) if keep_steps else None, qsize,
            nvc.ctypes.data_as(ipp), _dp(res), conv.ctypes.data_as(ipp), _dp(mass)),
            self.h, "bsam_host_take_time_steps")
        q = None
        if keep_steps:
            q = np.stack([buf[s * qsize:(s + 1) * qsize].reshape(self.qshape, order="F")
                          for s in range(nsteps)])
        return {"q": q, "nvcycles": nvc, "residual": res, "converged": conv, "mass": mass}

    def stream(self) -> int:
        """cudaStream_t of the handle (as an integer)."""
        p = ctypes.c_void_p()
        _check(lib().bsam_gpu_get_stream(self.h, ctypes.byref(p)), self.h, "get_stream")
        return p.value or 0

    def profile(self, enable: bool = True):
        _check(lib().bsam_gpu_profile(self.h, int(enable)), self.h, "profile")

    def stats(self) -> dict:
        st = Stats()
        _check(lib().bsam_gpu_get_stats(self.h, ctypes.byref(st)), self.h, "get_stats")
        return {k: getattr(st, k) for k, _ in Stats._fields_}

    def put_q_async_safe(self, q):
        """put_field from a (pinned) host array: H2D copy of q with ring."""
        _check(lib().bsam_gpu_put_field(self.h, 0, FIELD_Q, _dp(q)), self.h, "put_field")

    def get_q_into(self, out):
        _check(lib().bsam_gpu_get_field(self.h, 0, FIELD_Q, _dp(out)), self.h, "get_field")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().bsam_gpu_destroy(self.h)
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
