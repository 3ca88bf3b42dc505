"""Frame output (WriteQ, lib/bsaminputoutput.f90:51-172), CPU side.

tests/golden/frame2d.dat is a two-level 2D frame whose every field the
reference's own reader (lib_python/bsam_io.py) read back to the inputs when
the fixture was made (tests/golden/make_frame_golden.py).  The native
library's writer (bsam_host_format_frame) must produce it byte for byte, as
must the oracle's restatement; in 3D the two are compared with each other.
"""
import ast
import os

import numpy as np

from bsam_b200 import amr

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fixture():
    z = np.load(os.path.join(GOLD, "frame2d.npz"))
    descs = [ast.literal_eval(s) for s in z["descs"]]
    qs = {int(k[1:]): z[k] for k in z.files if k.startswith("q")}
    with open(os.path.join(GOLD, "frame2d.dat")) as f:
        text = f.read()
    return float(z["time"]), descs, qs, text


def test_oracle_frame_matches_fixture(oracle):
    time, descs, qs, text = _fixture()
    assert oracle.format_frame(2, time, descs, qs) == text


def test_native_frame_matches_fixture(gpu_free_lib, tmp_path):
    time, descs, qs, text = _fixture()
    path = str(tmp_path / "m00007.dat")
    amr.format_frame(path, 2, time, descs, qs)
    with open(path) as f:
        assert f.read() == text


def test_native_frame_3d_matches_oracle(gpu_free_lib, oracle, tmp_path):
    hier = amr.build(4, [(1, (3, 1, 5), (4, 2, 4))], eps=0.05, ndims=3, field="drop", seed=9)
    qs = dict(zip(hier.state_patches(), hier.q0s))
    qs[hier.state_patches()[0]][1, 1, 1, 0] = -123.456789012345678
    path = str(tmp_path / "f.dat")
    amr.format_frame(path, 3, 2.5, hier.descs, qs)
    with open(path) as f:
        assert f.read() == oracle.format_frame(3, 2.5, hier.descs, qs)


def test_frame_path():
    assert amr.frame_path("out", 42) == os.path.join("out", "m00042.dat")
