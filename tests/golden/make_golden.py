#!/usr/bin/env python
"""Generate golden fixtures by executing the reference's own Fortran source.

Reads the reference tree (default /root/reference; it must be present, so
this runs in the build container only) and, with the Fortran-subset
interpreter in fsubset.py, runs the reference's leaf routines of the hot path
on seeded inputs:

  RelaxGrid2D/3D, Operator2D/3D (+ ULapMob, ULap, UDiv, Dfc), Source2D/3D
      problems/simple_cahn-hilliard/problem.f90
  Restriction2D/3D, BiLinProlongationP1, TriLinProlongationP1
      lib/gridutilities.f90
  SetBC2D/3D (+ the problem's UserBC2D/3D), Interpolate2D, Interpolate3D
      lib/boundary.f90

the regridding leaves

  SetErrFlagsUser2D/3D (problem.f90), Bi/TriLinProlongationP1MC
  (gridutilities.f90), NewSubGrids with GetSignatures and GridFlagRatio
  (lib/bsamroutines.f90; MakeNewGrid stood in for, recording the boxes),
  BufferAndList, InflateEdgeTags and BufferTaggedCells (lib/bsamroutines.f90)

and their composition, the time loop's multigrid solve on fixed hierarchies
(uniform 2D and 3D, and 2D with refined levels):

  MultigridIterations, AFASVcycle, LevelRelax, FillDown(Level), ErrorAFAS,
  L2Error, SquareSum, GetSourceFunction, UpdateSourceFunction,
  UpdateAuxInVcycle, RelaxPatch, RestrictSolution, CoarseLoadingFunction,
  Residual, CorrectFine                       lib/afasroutines.f90
  SetGhost, InterpolateCoarseFine, TransferBC, GhostOverlap, SetBC,
  GetCoarseGhostPoints                        lib/boundary.f90
  CopyQToQold                                 lib/bsamroutines.f90

Each case's inputs and outputs go to tests/golden/ref_<case>.npz.  The tests
compare the CPU oracle's restatement of the same routines with these outputs
bit for bit (tests/test_golden_reference.py).

What is restated here rather than interpreted: TreeOps' level lists and
traversal (ApplyOnLevel order = the order of the patch records given),
AllocFields (q and qold zeroed, every other field NaN so that a read of an
undefined value shows in the output), and TakeTimeSteps' step sequence on an
unchanged hierarchy -- SetGhost(level, 0) from the root up (what
AMR(rootlevel) leaves), FillDown(solutionfield) on the first step,
CopyQToQold on every level, MultigridIterations (bsamroutines.f90:632-723).

Usage: python tests/golden/make_golden.py [reference_dir] [--only name,name,...]
(--only writes just the named fixtures; the seeded inputs do not depend on it.)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import fsubset as F  # noqa: E402
from bsam_b200 import amr, workloads as W  # noqa: E402  (pure-Python hierarchy builders)

ARGS = [a for a in sys.argv[1:] if not a.startswith("--only")]
if __name__ == "__main__" and not ARGS:
    sys.exit("usage: make_golden.py REFERENCE_DIR [--only=name,...]  "
             "(REFERENCE_DIR: the root of the BSAM source tree)")
REF = ARGS[0] if ARGS else None
ONLY = None
for a in sys.argv[1:]:
    if a.startswith("--only="):
        ONLY = set(a.split("=", 1)[1].split(","))
DT, EPS, ALPHA = 1.0e-4, 0.02, 1.0


def load() -> F.Interp:
    routines = {}
    consts = {}
    for rel in ("problems/simple_cahn-hilliard/problem.f90", "lib/gridutilities.f90",
                "lib/boundary.f90"):
        src = open(os.path.join(REF, rel)).read()
        routines.update(F.extract_routines(src))
        consts.update(F.parse_module_parameters(src))
    interp = F.Interp(routines, {"dt": DT, "eps": EPS, "eps2": EPS * EPS, "alpha": ALPHA})
    for name, expr in consts.items():
        interp.globals[name] = interp.ev(F.parse_expr(expr), {})
    return interp


def fa(a, lb):
    return F.FArray(np.array(a, dtype=np.float64, copy=True), lb)


# ---- the composition ---------------------------------------------------------------

COMPOSITION_FILES = ("problems/simple_cahn-hilliard/problem.f90", "lib/gridutilities.f90",
                     "lib/boundary.f90", "lib/afasroutines.f90")


class Tree:
    """TreeOps' level lists: on(level) in ApplyOnLevel order."""

    def __init__(self, recs):
        self.levels, self.errcode = {}, 0
        for r in recs:
            self.levels.setdefault(r.level, []).append(r)

    def on(self, level):
        return self.levels.get(level, [])


def records(hier):
    """nodeinfo records of a hierarchy's patches, fields as AllocFields
    leaves them (lib/bsamstorage.f90:46-123) except that the values it leaves
    undefined are NaN."""
    nd = hier.ndims
    recs = []
    for d in hier.descs:
        mx = list(d["mx"])
        r = F.Record(level=d["level"], nrvars=2, maux=0, mbc=1, tobedeleted=False, parent=None,
                     mx=F.FArray(np.array(mx, dtype=np.int64), (1,)),
                     mbounds=F.FArray(np.array(d["mbounds"], dtype=np.int64), (1, 1)),
                     mglobal=F.FArray(np.array(d["mglobal"], dtype=np.int64), (1, 1)),
                     mthbc=F.FArray(np.array(d["mthbc"], dtype=np.int64), (1,)),
                     dx=fa([d["dx"]] * 3, (1,)), xlower=fa(d["xlower"], (1,)))
        cmx = [1 if m % 2 else m // 2 for m in mx]
        ring = lambda m: tuple(m[n] + 2 if n < nd else 1 for n in range(3))
        inner = tuple(mx[n] if n < nd else 1 for n in range(3))
        lbr = (0, 0, 0 if nd == 3 else 1, 1)
        nan = lambda shp, lb: F.FArray(np.full(shp, np.nan, order="F"), lb)
        r.q = F.FArray(np.zeros(ring(mx) + (2,), order="F"), lbr)
        r.qold = F.FArray(np.zeros(ring(mx) + (2,), order="F"), lbr)
        r.qc = nan(ring(cmx) + (2,), lbr)
        r.aux = nan(ring([1, 1, 1]) + (1,), lbr)  # maux = 0: mmaux = 1, amx = 1
        for name in ("f", "rf", "ftmp"):
            setattr(r, name, nan(inner + (2,), (1, 1, 1, 1)))
        recs.append(r)
    for r, d in zip(recs, hier.descs):
        if d["parent"] >= 0:
            r.parent = recs[d["parent"]]
    return recs


def run_composition(hier, nsteps):
    """The reference's multigrid solve, interpreted, for nsteps time steps.
    Returns (final q of every patch on a level >= 0, V-cycles per step,
    residual trace per step as MultigridIterations prints it)."""
    routines, consts = {}, {}
    for rel in COMPOSITION_FILES:
        src = open(os.path.join(REF, rel)).read()
        got = F.extract_routines(src)
        clash = set(got) & set(routines)
        if clash:
            raise RuntimeError(f"routine names defined twice: {clash}")
        routines.update(got)
        consts.update(F.parse_module_parameters(src))
    bsam = F.extract_routines(open(os.path.join(REF, "lib/bsamroutines.f90")).read())
    routines["copyqtoqold"] = bsam["copyqtoqold"]
    recs = records(hier)
    for k, i in enumerate(hier.state_patches()):
        recs[i].q.data[...] = hier.q0s[k].reshape(recs[i].q.data.shape, order="F")
    levels = [d["level"] for d in hier.descs]
    minlevel, finest = min(levels), max(levels)
    g = {"dt": hier.dt, "eps": hier.eps, "eps2": hier.eps * hier.eps, "alpha": hier.alpha,
         "ndims": hier.ndims, "maxdims": 3, "maxnrvars": 25, "rootlevel": 0,
         "sourcefield": 1, "solutionfield": 2, "err_ok": 0, "finestlevel": finest,
         "minlevel": minlevel, "maxvcycles": hier.maxvcycles, "qerrortol": hier.qerrortol,
         "nsmoothingpasses": hier.nsmoothingpasses, "updateauxfreq": 1, "errortype": 1,
         "eqtag": 1, "lconverged": False,
         # PeriodicSetup (boundary.f90:893-963) for a root with periodic
         # faces; qpo = 0 (bsamroutines.f90:241).
         "periodicboundaryconditions": any(c == 2 for d in hier.descs for c in d["mthbc"]),
         "qpo": fa(np.zeros(25), (1,)),
         "integralresult": fa(np.zeros(2), (1,)), "componentintegral": fa(np.zeros(25), (1,))}
    I = F.Interp(routines, g, Tree(recs))
    for name, expr in consts.items():
        I.globals[name] = I.ev(F.parse_expr(expr), {})
    dummy = F.Record(iswitch=0)

    def ghosts():
        for level in range(0, finest + 1):
            I.run(routines["setghost"], [level, 0])

    def copy_q_to_qold():
        for level in range(minlevel, finest + 1):
            I.apply_on_level(level, routines["copyqtoqold"], dummy, pairs=False)

    ghosts()            # BSAMSolver: SetGhost, CopyQToQold (bsamroutines.f90:144-147)
    copy_q_to_qold()
    nvc, traces = [], []
    for step in range(nsteps):
        ghosts()
        if step == 0:
            I.run(routines["filldown"], [g["solutionfield"]])
        copy_q_to_qold()
        I.printed.clear()
        I.run(routines["multigriditerations"], [])
        if I.tree.errcode:
            raise RuntimeError(f"ApplyOnLevel error {I.tree.errcode}")
        trace = [float(p[1]) for p in I.printed]  # print *, 'it =', itmg, ' residual =', r
        nvc.append(len(trace))
        traces.append(trace + [-1.0] * (hier.maxvcycles - len(trace)))
    q = [recs[i].q.data.reshape(hier.q0s[k].shape, order="F").copy()
         for k, i in enumerate(hier.state_patches())]
    for a in q:
        if not np.all(np.isfinite(a)):
            raise RuntimeError("an undefined value reached q")
    return q, np.array(nvc, dtype=np.int32), np.array(traces)


def uniform_hierarchy(nd, n, mthbc, eps, qerrortol, maxvcycles, seed):
    """A uniform n^nd root on [0,1]^nd with its below-root levels (automatic
    minlevel), as RootInit / CreateBelowSeedLevels build it.  Initial
    composition: 2D, amr.build's sine wave with seeded 1e-3 noise; 3D, the
    seeded spinodal field c0 = 0.5 + 0.05 U(-1, 1)."""
    if nd == 2:
        return amr.build(n, [], eps=eps, qerrortol=qerrortol, mthbc=mthbc, seed=seed,
                         field="wave", maxvcycles=maxvcycles)
    descs, m, lev = [], n, 0
    codes = [mthbc] * 6 if isinstance(mthbc, int) else list(mthbc)
    while True:
        coarser = m % 2 == 0 and lev < 10
        descs.append({"level": -lev, "parent": lev + 1 if coarser else -1, "mx": [m] * 3,
                      "mbounds": [[1, m // 2 if coarser else m]] * 3, "mglobal": [[1, m]] * 3,
                      "mthbc": list(codes), "dx": (1.0 / n) * 2 ** lev, "xlower": [0.0] * 3})
        if not coarser:
            break
        m //= 2
        lev += 1
    h = 1.0 / n
    c0 = 0.5 + 0.05 * W.uniform(seed, n ** 3, -1.0, 1.0)
    q0 = W.initial_q(3, (n, n, n), c0, h, eps, 1.0)
    return amr.Hierarchy(ndims=3, descs=descs, q0s=[q0], dt=5e-5, eps=eps,
                         qerrortol=qerrortol, maxvcycles=maxvcycles)


def hier_arrays(hier):
    """A hierarchy as flat arrays for a fixture."""
    D = hier.descs
    return {"ndims": hier.ndims, "level": np.array([d["level"] for d in D]),
            "parent": np.array([d["parent"] for d in D]),
            "mx": np.array([d["mx"] for d in D]), "mbounds": np.array([d["mbounds"] for d in D]),
            "mglobal": np.array([d["mglobal"] for d in D]),
            "mthbc": np.array([d["mthbc"] for d in D]), "dxs": np.array([d["dx"] for d in D]),
            "xlower": np.array([d["xlower"] for d in D]),
            "q0": np.concatenate([q.ravel(order="F") for q in hier.q0s]),
            "hdt": hier.dt, "heps": hier.eps, "qerrortol": hier.qerrortol,
            "maxvcycles": hier.maxvcycles, "nsmoothingpasses": hier.nsmoothingpasses}


# ---- regridding leaves -----------------------------------------------------------

def regrid_interp(extra_globals):
    """An interpreter over problem.f90, gridutilities.f90 and the regrid
    routines of bsamroutines.f90 (NewSubGrids, GetSignatures,
    GridFlagRatio)."""
    routines = {}
    for rel in ("problems/simple_cahn-hilliard/problem.f90", "lib/gridutilities.f90"):
        routines.update(F.extract_routines(open(os.path.join(REF, rel)).read()))
    bsam = F.extract_routines(open(os.path.join(REF, "lib/bsamroutines.f90")).read())
    for name in ("newsubgrids", "getsignatures", "gridflagratio"):
        routines[name] = bsam[name]
    g = {"dt": DT, "eps": EPS, "eps2": EPS * EPS, "alpha": ALPHA, "maxdims": 3,
         "maxsubgrids": 1024}
    g.update(extra_globals)
    return F.Interp(routines, g)


def blob_flags(shape, rng, n_blobs):
    """0/1 flags: the union of a few random ellipsoids and a ring band."""
    grids = np.meshgrid(*[np.arange(s) + 0.5 for s in shape], indexing="ij")
    fl = np.zeros(shape, dtype=np.int64)
    for _ in range(n_blobs):
        c = [rng.uniform(0.2, 0.8) * s for s in shape]
        r = [rng.uniform(0.05, 0.25) * s for s in shape]
        fl |= (sum(((grids[k] - c[k]) / r[k]) ** 2 for k in range(len(shape))) < 1.0)
    rr = np.sqrt(sum((grids[k] - 0.55 * shape[k]) ** 2 for k in range(len(shape))))
    fl |= (np.abs(rr - 0.3 * min(shape)) < 1.5)
    return fl.astype(np.int64)


def regrid_cases(rng):
    out = {}
    maxdepth = 10
    # SetErrFlagsUser2D / 3D: |undivided central gradient of c| > qtolerance.
    for nd, mx in ((2, (24, 20)), (3, (10, 8, 12))):
        tol = 0.2
        I = regrid_interp({"qtolerance": fa(np.full(maxdepth + 1, tol), (0,))})
        qnew = 0.5 + 0.3 * rng.standard_normal(tuple(m + 2 for m in mx) + (2,))
        cmx = tuple(m // 2 for m in mx)
        qrte = np.zeros(cmx + (2,))
        flags = F.FArray(np.full(mx, 7, dtype=np.int64), (1,) * nd)
        I.run(I.routines[f"seterrflagsuser{nd}d"],
              [fa(qrte, (1,) * (nd + 1)), fa(qnew, (0,) * nd + (1,)), flags, ia(mx), ia(cmx), 2,
               1.0 / mx[0], fa(np.zeros(nd), (1,)), 1])
        out[f"errflags{nd}d"] = {"qnew": qnew, "tol": tol, "flags": flags.data}
    # Bi/TriLinProlongationP1MC: bilinear prolongation with the mass correction.
    for nd, cmx in ((2, (7, 5)), (3, (4, 3, 5))):
        I = regrid_interp({})
        a = rng.standard_normal(tuple(m + 2 for m in cmx) + (2,))
        name = "bilinprolongationp1mc" if nd == 2 else "trilinprolongationp1mc"
        p = I.run(I.routines[name], [fa(a, (0,) * nd + (1,))])
        out[f"prolong_mc{nd}d"] = {"a": a, "p": p}
    # NewSubGrids (Berger-Rigoutsos) with MakeNewGrid standing in: the boxes,
    # in the order the reference makes them.
    cases = [(2, (32, 32), 2, 0.9, 4), (2, (64, 48), 3, 0.7, 8), (2, (40, 40), 4, 0.9, 2),
             (3, (16, 16, 16), 2, 0.8, 4)]
    for n, (nd, mx, nblob, fill, mgp) in enumerate(cases):
        fl = blob_flags(mx, rng, nblob)
        mx3 = tuple(mx) + (1,) * (3 - nd)
        made = []
        I = regrid_interp({"ndims": nd,
                           "desiredfillratios": fa(np.full(maxdepth + 1, fill), (0,)),
                           "minimumgridpoints": F.FArray(np.full(maxdepth + 1, mgp,
                                                                 dtype=np.int64), (0,))})
        I.stubs["makenewgrid"] = lambda parent, mb: made.append(np.array(mb.data, copy=True))
        info = F.Record(mx=F.FArray(np.array(mx3, dtype=np.int64), (1,)), level=1, nsubgrids=0,
                        errorflags=F.FArray(fl.reshape(mx3, order="F").copy(order="F"),
                                            (1, 1, 1)))
        mb = F.FArray(np.array([[1, mx3[k]] for k in range(3)], dtype=np.int64), (1, 1))
        I.run(I.routines["newsubgrids"], [info, mb])
        boxes = np.array(made, dtype=np.int64).reshape(-1, 3, 2)
        out[f"subgrids_{n}"] = {"ndims": nd, "flags": fl, "fill": fill, "mgp": mgp,
                                "boxes": boxes, "nsubgrids": info.nsubgrids}
        print(f"subgrids_{n}", nd, mx, "boxes", len(made))
    # BufferAndList per patch of a level (ErrFlag, in ApplyOnLevel order),
    # then InflateEdgeTags over the level, with the tagged-cell list set up as
    # EstimateLevelErrors does (bsamroutines.f90:985-999).
    bcases = [(2, 1, [((1, 1), (16, 12)), ((17, 1), (10, 12)), ((5, 25), (20, 14))]),
              (2, 2, [((1, 1), (16, 12)), ((17, 1), (10, 12)), ((5, 25), (20, 14))]),
              (3, 1, [((1, 1, 1), (10, 8, 6)), ((11, 1, 1), (6, 8, 6)),
                      ((3, 13, 9), (8, 6, 10))])]
    for n, (nd, ib, boxes) in enumerate(bcases):
        recs, fl_in = [], []
        for lo, sz in boxes:
            mx3 = tuple(sz) + (1,) * (3 - nd)
            fl = (rng.random(mx3) < 0.03).astype(np.int64)
            fl_in.append(fl.copy())
            mg = [[lo[k], lo[k] + sz[k] - 1] for k in range(nd)] + [[1, 1]] * (3 - nd)
            recs.append(F.Record(level=1, tobedeleted=False,
                                 mx=F.FArray(np.array(mx3, dtype=np.int64), (1,)),
                                 mglobal=F.FArray(np.array(mg, dtype=np.int64), (1, 1)),
                                 errorflags=F.FArray(fl.copy(order="F"), (1, 1, 1))))
        # a flagged cell on the face patches 0 and 1 share
        recs[0].errorflags.data[(-1,) + (0,) * 2] = 1
        fl_in[0][(-1,) + (0,) * 2] = 1
        bsam = F.extract_routines(open(os.path.join(REF, "lib/bsamroutines.f90")).read())
        routines = {k: bsam[k] for k in ("bufferandlist", "inflateedgetags",
                                         "buffertaggedcells")}
        newcell = lambda: F.Record(id=0, coordinate=F.FArray(np.ones(3, dtype=np.int64), (1,)),
                                   prevcell=None)
        zeroth = newcell()  # allocate(zerothtaggedcell); nullify(...%prevcell)
        I = F.Interp(routines, {"ndims": nd, "maxdims": 3,
                                "ibuffer": F.FArray(np.full(maxdepth + 1, ib, dtype=np.int64),
                                                    (0,)),
                                "periodicboundaryconditions": False, "nperiodicoffsets": 0, "err_ok": 0,
                                "ntaggedcells": 0, "zerothtaggedcell": zeroth,
                                "lasttaggedcell": zeroth, "currenttaggedcell": None},
                     tree=Tree(recs))
        I.derived["currenttaggedcell"] = newcell
        for r in recs:
            I.run(I.routines["bufferandlist"], [r.errorflags, r.mglobal, r.mx, 1])
        if I.globals["ntaggedcells"] > 0:
            I.run(I.routines["inflateedgetags"], [1])
        res = {"ndims": nd, "ibuffer": ib, "npatch": len(recs),
               "ntagged_listed": I.globals["ntaggedcells"]}
        for k, r in enumerate(recs):
            res[f"mglobal_{k}"] = r.mglobal.data
            res[f"flags_in_{k}"] = fl_in[k]
            res[f"flags_out_{k}"] = r.errorflags.data
        out[f"buffer_{n}"] = res
        print(f"buffer_{n}", nd, "ibuffer", ib, "listed", I.globals["ntaggedcells"])
    return out


def composition_cases():
    out = {}
    cases = {
        # 16^2 root, levels 0..-4, Neumann faces.
        "mg_uniform2d": (uniform_hierarchy(2, 16, 1, 0.05, 1e-10, 8, 7), 2),
        # 8^3 root, levels 0..-3, user-coded faces.
        "mg_uniform3d": (uniform_hierarchy(3, 8, 10, 0.1, 1e-10, 6, 8), 2),
        # 16^2 root, levels 0..-4, periodic in x, Neumann in y (the shipped
        # example's x faces, griddata.dat:61-62).
        "mg_periodic2d": (uniform_hierarchy(2, 16, (2, 2, 1, 1), 0.05, 1e-10, 8, 7), 2),
        # 8^3 root, levels 0..-3, periodic in x and z, user-coded y faces.
        "mg_periodic3d": (uniform_hierarchy(3, 8, (2, 2, 12, 11, 2, 2), 0.1, 1e-10, 6, 8), 2),
        # 16^2 root, two siblings on level 1 (one on a physical corner), one
        # level-2 patch.
        "mg_amr2d": (amr.build(16, [(1, (1, 1), (12, 16)), (1, (13, 9), (14, 12)),
                                    (2, (5, 9), (12, 12))],
                               eps=0.05, qerrortol=1e-10, maxvcycles=8, seed=9), 2),
        # 8^3 root, two level-1 siblings sharing a y face (both on the z-low
        # physical face).
        "mg_amr3d": (amr.build(8, [(1, (5, 3, 1), (8, 8, 6)), (1, (5, 11, 1), (8, 4, 6))],
                               eps=0.1, qerrortol=1e-10, maxvcycles=6, seed=4, field="wave",
                               ndims=3), 2),
    }
    for name, (hier, nsteps) in cases.items():
        if ONLY is not None and name not in ONLY:
            continue
        q, nvc, tr = run_composition(hier, nsteps)
        d = hier_arrays(hier)
        d.update({"nsteps": nsteps, "q_out": np.concatenate([a.ravel(order="F") for a in q]),
                  "nvcycles": nvc, "trace": tr})
        out[name] = d
        print(name, "V-cycles per step", nvc.tolist())
    return out


def ia(v):
    return F.FArray(np.array(v, dtype=np.int64), (1,))


def main():
    I = load()
    rng = np.random.default_rng(20261203)
    out = {}

    # RelaxGrid2D / 3D: one colour pass in place.
    for nd, mx in ((2, (12, 10)), (3, (8, 6, 4))):
        h = 1.0 / mx[0]
        q = 0.5 + 0.1 * rng.standard_normal(tuple(m + 2 for m in mx) + (2,))
        f = 0.1 * rng.standard_normal(tuple(mx) + (2,))
        res = {"q_in": q, "f": f, "h": h, "mx": np.array(mx)}
        for ipass in (1, 2):
            qq = fa(q, (0,) * nd + (1,))
            zero = fa(np.zeros_like(q), (0,) * nd + (1,))
            name = "relaxgrid2d" if nd == 2 else "relaxgrid3d"
            I.run(I.routines[name], [qq, zero, zero, fa(f, (1,) * nd + (1,)), ia(mx), 2, 0, h,
                                     fa(np.zeros(nd), (1,)), ipass])
            res[f"q_out_{ipass}"] = qq.data
        out[f"relax{nd}d"] = res

    # Operator2D / 3D and Source2D / 3D.
    for nd, mx in ((2, (12, 10)), (3, (8, 6, 4))):
        h = 1.0 / mx[0]
        q = 0.5 + 0.1 * rng.standard_normal(tuple(m + 2 for m in mx) + (2,))
        qq = fa(q, (0,) * nd + (1,))
        zero = fa(np.zeros_like(q), (0,) * nd + (1,))
        op = I.run(I.routines[f"operator{nd}d"],
                   [qq, zero, zero, ia(mx), 2, 0, h, fa(np.zeros(nd), (1,))])
        src = I.run(I.routines[f"source{nd}d"],
                    [zero, qq, zero, 0, ia(mx), 2, 0, 1, h, fa(np.zeros(nd), (1,))])
        out[f"operator{nd}d"] = {"q": q, "h": h, "mx": np.array(mx), "res": op, "source": src}

    # Restriction and P1 prolongation.
    for nd, mx in ((2, (12, 10)), (3, (8, 6, 4))):
        a = rng.standard_normal(tuple(mx) + (2,))
        r = I.run(I.routines[f"restriction{nd}d"], [fa(a, (1,) * (nd + 1))])
        cmx = tuple(m // 2 for m in mx)
        c = rng.standard_normal(tuple(m + 2 for m in cmx) + (2,))
        pname = "bilinprolongationp1" if nd == 2 else "trilinprolongationp1"
        p = I.run(I.routines[pname], [fa(c, (0,) * nd + (1,))])
        out[f"transfer{nd}d"] = {"a": a, "restriction": r, "c": c, "prolongation": p}

    # SetBC2D / 3D with UserBC, several face-code mixes.
    codes2 = [(1, 1, 1, 1), (10, 20, 30, 40), (999, 1, 10, 999), (1, 999, 999, 15)]
    codes3 = [(1, 1, 1, 1, 1, 1), (10, 11, 12, 13, 14, 15), (999, 1, 10, 999, 1, 999)]
    for nd, mx, codes in ((2, (7, 5), codes2), (3, (5, 4, 3), codes3)):
        res = {"mx": np.array(mx)}
        q = rng.standard_normal(tuple(m + 2 for m in mx) + (2,))
        res["q_in"] = q
        for n, mth in enumerate(codes):
            qq = fa(q, (0,) * nd + (1,))
            if nd == 2:
                I.run(I.routines["setbc2d"], [qq, 0, ia(mx), 2, 1.0 / mx[0],
                                               fa(np.zeros(2), (1,)), 1, ia(mth)])
            else:
                I.run(I.routines["setbc3d"], [qq, 0, ia(mx), 2, 1, ia(mth)])
            res[f"mthbc_{n}"] = np.array(mth)
            res[f"q_out_{n}"] = qq.data
        out[f"setbc{nd}d"] = res

    # Interpolate2D: a 16 x 12 fine patch over parent cells 5..12 x 3..8 of a
    # 14 x 11 parent; every face-code mix and colour.
    pmx, mb = (14, 11), (5, 12, 3, 8)
    mx = (2 * (mb[1] - mb[0] + 1), 2 * (mb[3] - mb[2] + 1))
    qc = rng.standard_normal((pmx[0] + 2, pmx[1] + 2, 2))
    qf = rng.standard_normal((mx[0] + 2, mx[1] + 2, 2))
    res = {"qc": qc, "qf_in": qf, "mb": np.array(mb)}
    mixes = [(999, 999, 999, 999), (1, 999, 999, 10), (999, 2, 1, 999)]
    for n, mth in enumerate(mixes):
        res[f"mthbc_{n}"] = np.array(mth)
        for ipass in (0, 1, 2):
            qq = fa(qf, (0, 0, 1))
            I.run(I.routines["interpolate2d"],
                  [qq, fa(qc, (0, 0, 1)), ia(mx), 2,
                   F.FArray(np.array([[mb[0], mb[1]], [mb[2], mb[3]]], dtype=np.int64), (1, 1)),
                   ia(mth), ipass])
            res[f"qf_out_{n}_{ipass}"] = qq.data
    out["interpolate2d"] = res

    # Interpolate3D: an 8 x 6 x 10 fine patch over parent cells
    # 3..6 x 2..4 x 4..8 of a 9 x 7 x 10 parent; face-code mixes with internal
    # (999), periodic (2), physical (1, 10) faces and a z face coded 99 (the
    # edge check of boundary.f90:1354); every colour.
    pmx3, mb3 = (9, 7, 10), (3, 6, 2, 4, 4, 8)
    mx3 = tuple(2 * (mb3[2 * k + 1] - mb3[2 * k] + 1) for k in range(3))
    qc = rng.standard_normal(tuple(m + 2 for m in pmx3) + (2,))
    qf = rng.standard_normal(tuple(m + 2 for m in mx3) + (2,))
    res = {"qc": qc, "qf_in": qf, "mb": np.array(mb3)}
    mixes3 = [(999,) * 6, (1, 999, 10, 999, 999, 1), (999, 1, 999, 999, 99, 999),
              (2, 2, 999, 1, 99, 99)]
    for n, mth in enumerate(mixes3):
        res[f"mthbc_{n}"] = np.array(mth)
        for ipass in (0, 1, 2):
            qq = fa(qf, (0, 0, 0, 1))
            I.run(I.routines["interpolate3d"],
                  [qq, fa(qc, (0, 0, 0, 1)), ia(mx3), 2,
                   F.FArray(np.array([[mb3[0], mb3[1]], [mb3[2], mb3[3]], [mb3[4], mb3[5]]],
                                     dtype=np.int64), (1, 1)),
                   ia(mth), ipass])
            res[f"qf_out_{n}_{ipass}"] = qq.data
    out["interpolate3d"] = res

    # Energy2D of a 12 x 10 field with its ring (AfterStep2D at level 0).
    h = 1.0 / 12
    c = 0.5 + 0.3 * rng.standard_normal((14, 12))
    e = I.run(I.routines["energy2d"], [fa(c, (0, 0)), h])
    out["energy2d"] = {"c": c, "h": h, "energy": np.float64(e)}

    out.update(regrid_cases(rng))

    if ONLY is None or any(n.startswith("mg_") for n in ONLY):
        out.update(composition_cases())

    for name, d in out.items():
        if ONLY is not None and name not in ONLY:
            continue
        np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"),
                            **{k: np.asarray(v) for k, v in d.items()},
                            dt=DT, eps=EPS, alpha=ALPHA)
        print("wrote", f"ref_{name}.npz")


if __name__ == "__main__":
    main()
