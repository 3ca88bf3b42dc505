"""The oracle's leaf routines against the reference's own code (CPU only).

The fixtures in tests/golden/ref_*.npz were produced by executing the
reference's Fortran source text (problem.f90, gridutilities.f90,
boundary.f90) with the Fortran-subset interpreter in
tests/golden/fsubset.py (generator: tests/golden/make_golden.py).  The
oracle restates the same routines in C++; here it must reproduce every
fixture bit for bit.  The CUDA kernels are in turn bit-identical to the
oracle (tests/test_gpu_parity.py), so these fixtures pin the whole chain to
the reference's own arithmetic for: RelaxGrid2D/3D, Operator2D/3D,
Source2D/3D, Restriction2D/3D, Bi/TriLinProlongationP1, SetBC2D/3D with
UserBC2D/3D, Interpolate2D, Interpolate3D, Energy2D -- and for their composition, the
multigrid solve of the time loop (MultigridIterations with the V-cycle,
SetGhost, FillDown, ErrorAFAS; afasroutines.f90, boundary.f90) on uniform 2D
and 3D hierarchies, a 2D hierarchy with two refined levels and a 3D one with
two refined siblings.
"""
import ctypes
import os
import types

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fix(name):
    return np.load(os.path.join(GOLD, f"ref_{name}.npz"))


@pytest.mark.parametrize("nd", [2, 3])
def test_relax_grid_matches_reference(oracle, nd):
    d = fix(f"relax{nd}d")
    mx = tuple(int(m) for m in d["mx"])
    for ipass in (1, 2):
        assert not np.array_equal(d["q_in"], d[f"q_out_{ipass}"])  # the fixture moved
        got = oracle.relax_grid(nd, mx, float(d["h"]), float(d["dt"]), float(d["alpha"]),
                                float(d["eps"]), ipass, d["q_in"], d["f"])
        assert np.array_equal(got, d[f"q_out_{ipass}"]), ipass


@pytest.mark.parametrize("nd", [2, 3])
def test_operator_and_source_match_reference(oracle, nd):
    d = fix(f"operator{nd}d")
    mx = tuple(int(m) for m in d["mx"])
    got = oracle.operator(nd, mx, float(d["h"]), float(d["dt"]), float(d["alpha"]),
                          float(d["eps"]), d["q"])
    assert np.array_equal(got, d["res"])
    src = oracle.source(nd, float(d["alpha"]), d["q"])
    assert np.array_equal(src, d["source"])


@pytest.mark.parametrize("nd", [2, 3])
def test_transfers_match_reference(oracle, nd):
    d = fix(f"transfer{nd}d")
    assert np.array_equal(oracle.restriction(nd, d["a"]), d["restriction"])
    assert np.array_equal(oracle.prolongation_p1(nd, d["c"]), d["prolongation"])


@pytest.mark.parametrize("nd", [2, 3])
def test_setbc_matches_reference(oracle, nd):
    d = fix(f"setbc{nd}d")
    n = 0
    while f"mthbc_{n}" in d:
        got = oracle.setbc(nd, d["q_in"], tuple(int(c) for c in d[f"mthbc_{n}"]))
        assert np.array_equal(got, d[f"q_out_{n}"]), n
        n += 1
    assert n >= 3


def test_interpolate2d_matches_reference(oracle):
    d = fix("interpolate2d")
    mb = tuple(int(v) for v in d["mb"])
    n = 0
    while f"mthbc_{n}" in d:
        mth = tuple(int(c) for c in d[f"mthbc_{n}"])
        for ipass in (0, 1, 2):
            got = oracle.interpolate2d(d["qf_in"], d["qc"], mb, mth, ipass)
            assert np.array_equal(got, d[f"qf_out_{n}_{ipass}"]), (n, ipass)
        n += 1
    assert n >= 3


def test_interpolate3d_matches_reference(oracle):
    d = fix("interpolate3d")
    mb = tuple(int(v) for v in d["mb"])
    n = 0
    while f"mthbc_{n}" in d:
        mth = tuple(int(c) for c in d[f"mthbc_{n}"])
        for ipass in (0, 1, 2):
            got = oracle.interpolate3d(d["qf_in"], d["qc"], mb, mth, ipass)
            assert np.array_equal(got, d[f"qf_out_{n}_{ipass}"]), (n, ipass)
        n += 1
    assert n >= 4


def test_energy2d_matches_reference(oracle):
    d = fix("energy2d")
    got = oracle.energy2d(float(d["h"]), float(d["alpha"]), float(d["eps"]), d["c"])
    assert got == float(d["energy"])


@pytest.mark.parametrize("nd", [2, 3])
def test_errflags_match_reference(oracle, nd):
    d = fix(f"errflags{nd}d")
    got = oracle.errflags(d["qnew"][..., 0], float(d["tol"]))
    assert np.array_equal(got, d["flags"])
    assert 0 < got.sum() < got.size


@pytest.mark.parametrize("nd", [2, 3])
def test_prolongation_mc_matches_reference(oracle, nd):
    d = fix(f"prolong_mc{nd}d")
    assert np.array_equal(oracle.prolong_mc(nd, d["a"]), d["p"])


@pytest.mark.parametrize("n", [0, 1, 2, 3])
def test_new_subgrids_match_reference(oracle, n):
    """Berger-Rigoutsos clustering: the same boxes in the same order."""
    d = fix(f"subgrids_{n}")
    nd = int(d["ndims"])
    got = oracle.new_subgrids(d["flags"], float(d["fill"]), int(d["mgp"]))
    want = d["boxes"]
    assert got.shape[0] == want.shape[0] == int(d["nsubgrids"])
    assert np.array_equal(got[:, :nd, :], want[:, :nd, :])


MG_CASES = ["mg_uniform2d", "mg_uniform3d", "mg_amr2d", "mg_amr3d"]


@pytest.mark.parametrize("name", MG_CASES)
def test_multigrid_composition_matches_reference(oracle, golden_hier, name):
    """The time loop's multigrid solve on a fixed hierarchy: the oracle's
    MultigridIterations (with SetGhost, FillDown, ErrorAFAS and the V-cycle)
    against the reference's own afasroutines.f90 / boundary.f90 composition,
    bit for bit: every patch's q after the steps, V-cycles per step and the
    final residual of each step."""
    hier, d = golden_hier(name)
    nsteps = int(d["nsteps"])
    ref = oracle.run_hier(hier, nsteps)
    assert np.array_equal(ref["nvcycles"], d["nvcycles"]), (ref["nvcycles"], d["nvcycles"])
    last = [d["trace"][s, d["nvcycles"][s] - 1] for s in range(nsteps)]
    assert np.array_equal(ref["residual"], last)
    got = np.concatenate([q.ravel(order="F") for q in ref["q"]])
    assert np.array_equal(got, d["q_out"])


@pytest.mark.parametrize("name", ["mg_uniform2d", "mg_uniform3d", "mg_periodic2d",
                                  "mg_periodic3d"])
def test_uniform_time_loop_matches_reference(oracle, golden_hier, name):
    """orc_run_uniform (its own root and below-root construction) against the
    same fixtures: the whole residual trace of every step and the final q."""
    hier, d = golden_hier(name)
    nd, root = hier.ndims, hier.descs[0]
    nsteps = int(d["nsteps"])
    prob = types.SimpleNamespace(
        ndims=nd, mx=tuple(root["mx"]), xupper=(1.0, 1.0, 1.0), mthbc=tuple(root["mthbc"]),
        minlevel=1, nsmoothingpasses=hier.nsmoothingpasses, maxvcycles=hier.maxvcycles,
        dt=hier.dt, qerrortol=hier.qerrortol, alpha=hier.alpha, eps=hier.eps, nsteps=nsteps)
    assert oracle.lib().orc_minlevel(ctypes.byref(oracle.params_of(prob))) == min(d["level"])
    ref = oracle.run_uniform(prob, nsteps, q0=hier.q0s[0])
    assert np.array_equal(ref["nvcycles"], d["nvcycles"])
    assert np.array_equal(ref["trace"], d["trace"])
    assert np.array_equal(ref["q"][-1].ravel(order="F"), d["q_out"])


def _buffer_fixture(n):
    d = np.load(os.path.join(GOLD, f"ref_buffer_{n}.npz"))
    nd, np_ = int(d["ndims"]), int(d["npatch"])
    descs, fin, fout = [], [], []
    for k in range(np_):
        mg = d[f"mglobal_{k}"]
        mx = [int(mg[n_][1] - mg[n_][0] + 1) for n_ in range(3)]
        descs.append({"level": 1, "parent": 0, "mx": mx, "mbounds": [[1, 1]] * 3,
                      "mglobal": [list(map(int, mg[n_])) for n_ in range(3)],
                      "mthbc": [999] * 6, "dx": 1.0, "xlower": [0.0] * 3})
        shp = tuple(mx[:nd])
        fin.append(d[f"flags_in_{k}"].reshape(shp, order="F"))
        fout.append(d[f"flags_out_{k}"].reshape(shp, order="F"))
    return nd, int(d["ibuffer"]), descs, fin, fout


@pytest.mark.parametrize("n", [0, 1, 2])
def test_buffer_flags_match_reference(oracle, n):
    """BufferAndList + InflateEdgeTags + BufferTaggedCells, interpreted from
    the reference source over a level of three patches (two sharing a face),
    against the oracle's restatement."""
    nd, ib, descs, fin, fout = _buffer_fixture(n)
    got = oracle.buffer_flags(nd, descs, fin, ib)
    for g, w in zip(got, fout):
        assert np.array_equal(g, w)
