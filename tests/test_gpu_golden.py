"""The GPU engine against the reference's own multigrid composition.

tests/golden/ref_mg_*.npz hold the result of executing the reference's
MultigridIterations (afasroutines.f90, boundary.f90, the problem module)
from its Fortran source on fixed hierarchies (tests/golden/make_golden.py).
The FP64 form of the engine, driven through the C ABI and the C++ host time
loop, must reproduce them: identical V-cycle counts, q of every patch on every
level >= 0 (ghost rings included) within 1e-11 relative (max norm), final
residuals within 1e-9 relative.
"""
import numpy as np
import pytest

from bsam_b200 import amr

pytestmark = pytest.mark.gpu

RTOL = 1e-11


@pytest.mark.parametrize("name", ["mg_uniform2d", "mg_uniform3d", "mg_amr2d", "mg_amr3d",
                                  "mg_periodic2d", "mg_periodic3d"])
def test_engine_matches_reference_composition(gpu_lib, golden_hier, name):
    hier, d = golden_hier(name)
    nsteps = int(d["nsteps"])
    with amr.HierSolver(hier) as s:
        got = s.run(nsteps)
    assert np.array_equal(got["nvcycles"], d["nvcycles"]), (got["nvcycles"], d["nvcycles"])
    last = np.array([d["trace"][k, d["nvcycles"][k] - 1] for k in range(nsteps)])
    np.testing.assert_allclose(got["residual"], last, rtol=1e-9, atol=0)
    off = 0
    for k, q in enumerate(got["q"]):
        want = d["q_out"][off:off + q.size].reshape(q.shape, order="F")
        off += q.size
        for v in range(2):
            err = float(np.max(np.abs(q[..., v] - want[..., v])) / np.max(np.abs(want[..., v])))
            assert err < RTOL, (name, k, v, err)
    assert off == d["q_out"].size
