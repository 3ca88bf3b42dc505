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
  SetBC2D/3D (+ the problem's UserBC2D/3D), Interpolate2D
      lib/boundary.f90

Each case's inputs and outputs go to tests/golden/ref_<routine>.npz.  The
tests compare the CPU oracle's restatement of the same routines with these
outputs bit for bit (tests/test_golden_reference.py).

Usage: python tests/golden/make_golden.py [reference_dir]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import fsubset as F  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
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

    for name, d in out.items():
        np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"),
                            **{k: np.asarray(v) for k, v in d.items()},
                            dt=DT, eps=EPS, alpha=ALPHA)
        print("wrote", f"ref_{name}.npz")


if __name__ == "__main__":
    main()
