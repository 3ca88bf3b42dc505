#!/usr/bin/env python
"""Generate the frame-output fixture (tests/golden/frame2d.dat + .npz).

The reference writes frames with Fortran formatted output (WriteQ,
lib/bsaminputoutput.f90:51-172), which cannot run here (no Fortran
compiler), and reads them back with its own Python reader
(lib_python/bsam_io.py:4-73, parse_adaptive_data_file).  This script formats
a small two-level 2D hierarchy with the oracle's restatement of WriteQ
(oracle/pyoracle.py: format_frame), then checks that the REFERENCE's reader,
imported from the reference tree, reads back the time, the finest level, the
patch count, each patch's level, h, x/y extents, sizes, global index boxes
and q (ring included) -- to the 13 significant digits es20.12 keeps.  Only
then are the text and its inputs written.  It needs the reference tree, so
it runs in the build container only.

Usage: python tests/golden/make_frame_golden.py [reference_dir]
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from bsam_b200 import amr  # noqa: E402  (pure-Python hierarchy builder)
from oracle import pyoracle  # noqa: E402

if __name__ == "__main__" and len(sys.argv) < 2:
    sys.exit("usage: make_frame_golden.py REFERENCE_DIR  (the root of the BSAM source tree)")
REF = sys.argv[1] if len(sys.argv) > 1 else None


def reference_reader():
    spec = importlib.util.spec_from_file_location(
        "bsam_io", os.path.join(REF, "lib_python", "bsam_io.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.xrange = range  # the reader is written for Python 2
    return mod


def main():
    hier = amr.build(8, [(1, (5, 3), (6, 8)), (1, (11, 11), (4, 4))], eps=0.05, dt=1e-4,
                     field="drop", seed=5)
    rng = np.random.default_rng(11)
    qs = {}
    for i, q in zip(hier.state_patches(), hier.q0s):
        q = np.array(q, order="F")
        # Values across many decades and both signs, ring included.
        q[..., 1] = rng.standard_normal(q.shape[:2]) * 10.0 ** rng.integers(-30, 30, q.shape[:2])
        qs[i] = q
    time = 0.0123
    text = pyoracle.format_frame(2, time, hier.descs, qs)
    path = os.path.join(HERE, "frame2d.dat")
    with open(path, "w") as f:
        f.write(text)
    got = reference_reader().parse_adaptive_data_file(path)
    assert got["time"] == time and got["maxlevel"] == 1
    order = [i for lv in (0, 1) for i, d in enumerate(hier.descs) if d["level"] == lv]
    assert got["npatches"] == len(order)
    flat = [p for lv in got["levels"] for p in lv]
    for p, i in zip(flat, order):
        d = hier.descs[i]
        assert p["level"] == d["level"] and p["nx"] == d["mx"][0] and p["ny"] == d["mx"][1]
        assert p["h"] == d["dx"]
        assert p["mgx"] == d["mglobal"][0] and p["mgy"] == d["mglobal"][1]
        assert abs(p["x"][0] - d["xlower"][0]) < 1e-12 and abs(p["y"][0] - d["xlower"][1]) < 1e-12
        want = np.transpose(qs[i], (2, 1, 0))  # reader: [var, j, i]
        assert np.allclose(p["data"], want, rtol=1e-12, atol=0)
    np.savez_compressed(os.path.join(HERE, "frame2d.npz"), time=time,
                        descs=np.array([repr(d) for d in hier.descs]),
                        **{f"q{i}": q for i, q in qs.items()})
    print("wrote frame2d.dat, frame2d.npz;", got["npatches"], "patches read back by the "
          "reference reader")


if __name__ == "__main__":
    main()
