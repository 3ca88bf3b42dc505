"""Regridding pieces on the GPU against the oracle (FP64, bit for bit).

* bsam_gpu_errflags: SetErrFlagsUser2D/3D of root and refined patches.
* bsam_gpu_init_patch: InitFields of a refined patch -- the mass-corrected
  prolongation of its parent's state over the footprint and one-cell ring
  (Bi/TriLinProlongationP1MC), qold = q.
The oracle's routines are pinned to the reference source
(tests/test_golden_reference.py).
"""
import numpy as np
import pytest

from bsam_b200 import amr

pytestmark = pytest.mark.gpu

CASES = {
    2: (32, [(1, (9, 5), (24, 20)), (1, (33, 41), (16, 16))]),
    3: (16, [(1, (5, 3, 7), (12, 16, 10))]),
}


def hier(nd):
    n, boxes = CASES[nd]
    return amr.build(n, boxes, eps=0.05, dt=5e-5, qerrortol=1e-9, ndims=nd, field="drop", seed=3)


@pytest.mark.parametrize("nd", [2, 3])
def test_errflags_match_oracle(gpu_lib, oracle, nd):
    h = hier(nd)
    with amr.HierSolver(h) as s:
        for p in h.state_patches():
            q = s.get_q(p)
            for tol in (0.05, 0.2):
                got = s.errflags(p, tol)
                want = oracle.errflags(q[..., 0], tol)
                assert np.array_equal(got.astype(np.int32), want), (p, tol)


@pytest.mark.parametrize("nd", [2, 3])
def test_init_patch_matches_oracle(gpu_lib, oracle, nd):
    h = hier(nd)
    with amr.HierSolver(h) as s:
        s.run(1)  # a state that is not the initial one
        for p, d in enumerate(h.descs):
            if d["level"] < 1:
                continue
            parent = s.get_q(d["parent"])
            sl = tuple(slice(d["mbounds"][k][0] - 1, d["mbounds"][k][1] + 2) for k in range(nd))
            want = oracle.prolong_mc(nd, parent[sl + (slice(None),)])
            s.init_patch(p)
            got = s.get_q(p)
            assert got.shape == want.shape
            assert np.array_equal(got, want), (p, float(np.max(np.abs(got - want))))
            assert np.array_equal(s.get_qold(p), got)


REGRID_CASES = {
    # ndims: (root cells, eps, RegridParams)
    2: (32, 0.02, amr.RegridParams(maxlevel=2, qtolerance=[0.05, 0.05], ibuffer=[1, 1],
                                   desfill=[0.7, 0.7], mgp=[4, 4])),
    3: (16, 0.05, amr.RegridParams(maxlevel=2, qtolerance=[0.15, 0.15], ibuffer=[1, 1],
                                   desfill=[0.7, 0.7], mgp=[2, 2])),
}


@pytest.mark.parametrize("nd", [2, 3])
def test_regrid_run_matches_oracle(gpu_lib, oracle, nd):
    """Time steps with regridding every step (amr.RegridRun: tagging,
    buffering, Berger-Rigoutsos, new-patch prolongation, value transfer, the
    level-by-level ghosts and restrictions of AMR(rootlevel), FillDown,
    MultigridIterations), engine against oracle: the same grids every step,
    the same V-cycle counts, q within 1e-11, and the same after-step
    statistics (composite mass and energy)."""
    n, eps, prm = REGRID_CASES[nd]
    hier = amr.build(n, [], eps=eps, dt=5e-5, qerrortol=1e-9, field="drop", ndims=nd)
    g = amr.GpuBackend(nd, hier.dt, hier.eps, hier.qerrortol)
    o = oracle.OracleBackend(nd, hier.dt, hier.eps, hier.qerrortol)
    try:
        rg = amr.RegridRun(g, hier, prm)
        ro = amr.RegridRun(o, hier, prm)
        for step in range(3):
            nvg, resg = rg.step()
            nvo, reso = ro.step()
            assert rg.descs == ro.descs, f"grids differ at step {step}"
            assert nvg == nvo
            assert resg == pytest.approx(reso, rel=1e-6, abs=1e-15)
            assert max(d["level"] for d in rg.descs) == 2
            # AfterStepStatistics: composite mass and (2D) energy.
            mg, eg = rg.stats()
            mo, eo = ro.stats()
            assert mg == pytest.approx(mo, rel=1e-12)
            assert eg == pytest.approx(eo, rel=1e-12, abs=0 if nd == 2 else 1e-300)
            for (i, qg), (_, qo) in zip(rg.state(), ro.state()):
                d = rg.descs[i]
                inner = tuple(slice(1, m + 1) for m in d["mx"][:nd])
                np.testing.assert_allclose(qg[inner], qo[inner], rtol=0, atol=1e-11)
    finally:
        g.close()
        o.close()


@pytest.mark.parametrize("nd", [2, 3])
def test_write_frame_from_device(gpu_lib, oracle, nd, tmp_path):
    """bsam_host_write_frame (q read back from the device, then WriteQ's
    format) against the oracle's WriteQ text of the same state, after a
    regridding step."""
    n, eps, prm = REGRID_CASES[nd]
    hier = amr.build(n, [], eps=eps, dt=5e-5, qerrortol=1e-9, field="drop", ndims=nd)
    g = amr.GpuBackend(nd, hier.dt, hier.eps, hier.qerrortol)
    try:
        run = amr.RegridRun(g, hier, prm)
        run.step()
        path = str(tmp_path / "m00001.dat")
        g.write_frame(path, 5e-5)
        qs = dict(run.state())
        with open(path) as f:
            assert f.read() == oracle.format_frame(nd, 5e-5, run.descs, qs)
    finally:
        g.close()


@pytest.mark.parametrize("nd", [2, 3])
def test_native_amr_run_matches_oracle(gpu_lib, oracle, nd):
    """The native AMR time-step driver (bsam_amr_step: the whole regrid and
    solve in the host library) against the regrid driver over the oracle:
    the same grids every step, the same V-cycle counts, q within 1e-11."""
    n, eps, prm = REGRID_CASES[nd]
    hier = amr.build(n, [], eps=eps, dt=5e-5, qerrortol=1e-9, field="drop", ndims=nd)
    o = oracle.OracleBackend(nd, hier.dt, hier.eps, hier.qerrortol)
    with amr.AmrRun(hier, prm) as rn:
        try:
            ro = amr.RegridRun(o, hier, prm)
            for step in range(3):
                nvn, _ = rn.step()
                nvo, _ = ro.step()
                assert rn.descs == ro.descs, f"grids differ at step {step}"
                assert nvn == nvo
                mg, _ = rn.stats()
                mo, _ = ro.stats()
                assert mg == pytest.approx(mo, rel=1e-12)
                for (i, qg), (_, qo) in zip(rn.state(), ro.state()):
                    d = rn.descs[i]
                    inner = tuple(slice(1, m + 1) for m in d["mx"][:nd])
                    np.testing.assert_allclose(qg[inner], qo[inner], rtol=0, atol=1e-11)
            # The per-phase host times cover every step.
            prof = rn.profile()
            assert prof["steps"] == 3
            assert all(prof[k] >= 0.0 for k in rn.PHASES) and prof["solve"] > 0.0
            t = rn.table_array()
            assert len(t) == len(rn.descs)
            assert list(t["level"]) == [d["level"] for d in rn.descs]
        finally:
            o.close()


@pytest.mark.parametrize("nd", [2, 3])
@pytest.mark.parametrize("ibuffer", [0, 1, 2])
def test_tag_level_on_device_matches_host_buffering(gpu_lib, nd, ibuffer):
    """bsam_gpu_tag_level (tagging, BufferAndList + InflateEdgeTags and the
    summed-area tables, on the device) against the device's tagging
    buffered by the host library (bsam_host_buffer_flags, pinned to the
    reference's source) and summed on the host, on every level."""
    h = hier(nd)
    with amr.HierSolver(h) as s:
        s.run(1)
        for level in (0, 1):
            idx = [i for i, d in enumerate(h.descs) if d["level"] == level]
            for tol in (0.05, 0.2):
                flags = [s.errflags(p, tol) for p in idx]
                want = amr.buffer_flags(nd, [h.descs[p] for p in idx], flags, ibuffer)
                got = s.tag_level(level, tol, ibuffer)
                for w, g in zip(want, got):
                    assert np.array_equal(amr.summed_area(w), g), (level, tol)
