"""Known-answer tests and invariants of the CPU oracle.

The reference ships no tests or golden vectors, so these checks follow from
the reference's own formulas (file:line cited per test).
"""
import numpy as np
import pytest

from bsam_b200 import workloads as W


def test_restriction_of_constant(oracle):
    # Restriction2D/3D average 2^d children (gridutilities.f90:104-108, 423-431).
    for nd, shape in ((2, (8, 6, 2)), (3, (4, 6, 8, 2))):
        a = np.full(shape, 0.375, order="F")   # dyadic: every partial sum exact
        r = oracle.restriction(nd, a)
        assert np.all(r == 0.375)
        r = oracle.restriction(nd, np.full(shape, 0.37, order="F"))
        np.testing.assert_allclose(r, 0.37, rtol=4e-16)


def test_restriction_is_mean(oracle):
    rng = np.random.default_rng(0)
    a = rng.random((8, 8, 2))
    r = oracle.restriction(2, np.asfortranarray(a))
    want = 0.25 * (a[1::2, 1::2] + a[0::2, 1::2] + a[1::2, 0::2] + a[0::2, 0::2])
    assert np.array_equal(r, want)


@pytest.mark.parametrize("nd", [2, 3])
def test_prolongation_reproduces_linear(oracle, nd):
    # (Bi|Tri)LinProlongationP1 (gridutilities.f90:137-175, 474-529) is exact on
    # linear fields: coarse centres at (m - 1/2) * 2h map to fine (i - 1/2) h.
    cmx = (4, 6, 5)[:nd]
    grids = np.meshgrid(*[np.arange(c + 2) for c in cmx], indexing="ij")
    coef = (0.5, -0.25, 0.125)
    a = sum(coef[d] * (2.0 * (grids[d] - 0.5)) for d in range(nd)) + 1.0
    a = np.stack([a, 2 * a], axis=-1)
    out = oracle.prolongation_p1(nd, np.asfortranarray(a))
    fg = np.meshgrid(*[np.arange(2 * c + 2) for c in cmx], indexing="ij")
    want = sum(coef[d] * (fg[d] - 0.5) for d in range(nd)) + 1.0
    inner = tuple(slice(1, -1) for _ in range(nd))
    # interior and the ring: the interpolation weights sum to 16 (4^d), exact.
    np.testing.assert_allclose(out[..., 0][inner], want[inner], rtol=0, atol=1e-14)
    np.testing.assert_allclose(out[..., 1][inner], 2 * want[inner], rtol=0, atol=1e-14)


def test_neumann_corners(oracle):
    # SetBC2D copies whole rows face by face (boundary.f90:661-738): every
    # ghost equals its interior mirror, corners the diagonal cell.
    rng = np.random.default_rng(1)
    q = np.zeros((6, 5, 2), order="F")
    q[1:-1, 1:-1] = rng.random((4, 3, 2))
    out = oracle.setbc(2, q, (1, 1, 1, 1))
    assert np.array_equal(out[0, 1:-1], out[1, 1:-1])
    assert np.array_equal(out[-1, 1:-1], out[-2, 1:-1])
    assert np.array_equal(out[1:-1, 0], out[1:-1, 1])
    assert out[0, 0, 0] == out[1, 1, 0] and out[-1, -1, 1] == out[-2, -2, 1]
    assert out[0, -1, 0] == out[1, -2, 0] and out[-1, 0, 1] == out[-2, 1, 1]


def test_user_bc_2d(oracle):
    # UserBC2D (problem.f90:663-693): faces 1,2 -> 2 - q; faces 3,4 -> copy.
    rng = np.random.default_rng(2)
    q = np.zeros((6, 6, 2), order="F")
    q[1:-1, 1:-1] = rng.random((4, 4, 2))
    out = oracle.setbc(2, q, (10, 10, 10, 10))
    assert np.array_equal(out[0, 1:-1], 2.0 - out[1, 1:-1])
    assert np.array_equal(out[1:-1, -1], out[1:-1, -2])
    # corner: face 3 copies the row that face 1 already reflected
    assert out[0, 0, 0] == 2.0 - out[1, 1, 0]


def test_neumann_3d_edges(oracle):
    rng = np.random.default_rng(3)
    q = np.zeros((5, 6, 4, 2), order="F")
    q[1:-1, 1:-1, 1:-1] = rng.random((3, 4, 2, 2))
    out = oracle.setbc(3, q, (1,) * 6)
    assert out[0, 0, 0, 0] == out[1, 1, 1, 0]
    assert out[-1, 0, 2, 1] == out[-2, 1, 2, 1]
    assert np.array_equal(out[2, 3, 0], out[2, 3, 1])


def _random_state(nd, mx, seed):
    rng = np.random.default_rng(seed)
    q = np.zeros(tuple(m + 2 for m in mx) + (2,), order="F")
    inner = tuple(slice(1, m + 1) for m in mx)
    q[inner + (0,)] = 0.5 + 0.1 * rng.standard_normal(mx)
    q[inner + (1,)] = 0.01 * rng.standard_normal(mx)
    f = np.asfortranarray(0.01 * rng.standard_normal(tuple(mx) + (2,)))
    return q, f


@pytest.mark.parametrize("nd", [2, 3])
def test_relax_solves_local_system(oracle, nd):
    # RelaxGrid (problem.f90:164-215, 453-518) is a Newton step of the cell's
    # 2x2 system in (phi, mu) around the old phi.  Since the operator is linear
    # in mu and quadratic-free in the Laplacian, the updated cell satisfies the
    # row-1 equation exactly and the row-2 equation up to the Newton remainder.
    mx = (6, 6, 4)[:nd]
    q, f = _random_state(nd, mx, 5)
    q = oracle.setbc(nd, q, (1,) * (2 * nd))
    h, dt, alpha, eps = 1.0 / 16, 1e-4, 1.0, 0.02
    q1 = oracle.relax_grid(nd, mx, h, dt, alpha, eps, 1, q, f)
    res = oracle.operator(nd, mx, h, dt, alpha, eps, q1)
    idx = (2, 1, 1) if nd == 3 else (1, 1)   # 1-based cell with even i+j(+k)
    c = tuple(i - 1 for i in idx)
    r0 = f[c + (0,)] - res[c + (0,)]
    assert abs(r0) < 1e-12


@pytest.mark.parametrize("nd", [2, 3])
def test_colour_purity(oracle, nd):
    # One colour pass leaves the other colour bit-identical (problem.f90:193, 487).
    mx = (8, 6, 4)[:nd]
    q, f = _random_state(nd, mx, 7)
    q1 = oracle.relax_grid(nd, mx, 1 / 8, 1e-4, 1.0, 0.02, 1, q, f)
    inner = tuple(slice(1, m + 1) for m in mx)
    par = sum(np.meshgrid(*[np.arange(1, m + 1) for m in mx], indexing="ij")) % 2
    for v in range(2):
        a, b = q[inner + (v,)], q1[inner + (v,)]
        assert np.array_equal(a[par == 1], b[par == 1])
        assert not np.array_equal(a[par == 0], b[par == 0])


def test_operator_quadratic(oracle):
    # ULap2D of x^2 + y^2 (undivided, h-scaled) is 4 h^2: check through the
    # operator's second row with phi = quadratic, mu = Dfc(phi).
    mx = (6, 5)
    h = 0.1
    i = (np.arange(mx[0] + 2) - 0.5) * h
    j = (np.arange(mx[1] + 2) - 0.5) * h
    X, Y = np.meshgrid(i, j, indexing="ij")
    phi = X * X + Y * Y
    q = np.zeros(X.shape + (2,), order="F")
    q[..., 0] = phi
    cmh = phi - 0.5
    q[..., 1] = cmh * cmh * cmh
    eps = 0.3
    res = oracle.operator(2, mx, h, 1e-3, 1.0, eps, q)
    np.testing.assert_allclose(res[..., 1], eps * eps / (h * h) * 4 * h * h, rtol=1e-12)


def test_source(oracle):
    rng = np.random.default_rng(9)
    qold = np.asfortranarray(rng.random((6, 5, 2)))
    f = oracle.source(2, 1.0, qold)
    c = qold[1:-1, 1:-1, 0]
    assert np.array_equal(f[..., 0], c)
    assert np.array_equal(f[..., 1], -((c - 0.5) * 1.0 / 4.0))


def test_mass_conserved_and_energy_decays(oracle):
    # Neumann CH conserves h^d sum(c); Eyre's splitting decreases Energy2D
    # (problem.f90:121-132, 330-361).
    prob = W.config1(nsteps=4, n=32)
    r = oracle.run_uniform(prob)
    # Conserved up to the algebraic residual left by the solver (< qerrortol).
    m0 = prob.h ** 2 * prob.c0.sum()
    assert np.all(np.abs(np.diff(np.concatenate([[m0], r["mass"]]))) < prob.qerrortol)
    e = [oracle.energy2d(prob.h, 1.0, prob.eps, prob.q0()[..., 0])]
    e += [oracle.energy2d(prob.h, 1.0, prob.eps, r["q"][s][..., 0]) for s in range(4)]
    assert all(e[s + 1] <= e[s] + 1e-14 for s in range(4))
    assert np.all(r["residual"] < prob.qerrortol)


def test_vcycle_contraction(oracle):
    # Each V(2,2) cycle contracts the residual; once dt/h^2 dominates, the rate
    # is roughly independent of the grid size.
    rates = []
    for n in (64, 128, 256):
        r = oracle.run_uniform(W.config1(nsteps=1, n=n), keep_steps=False)
        tr = r["trace"][0]
        tr = tr[tr > 0]
        rates.append(np.exp(np.mean(np.log(tr[1:] / tr[:-1]))))
    assert all(0 < x < 0.2 for x in rates)
    assert max(rates) / min(rates) < 3.0


def test_3d_converges(oracle):
    r = oracle.run_uniform(W.config3(nsteps=1, n=16), keep_steps=False)
    assert r["nvcycles"][0] < 20 and r["residual"][0] < 1e-8


def test_odd_coarsest(oracle):
    # 96 = 3 * 32: the automatic minlevel stops at 3x3 (bsamroutines.f90:293-298).
    prob = W.config1(nsteps=2, n=96)
    assert oracle.lib().orc_minlevel(oracle.params_of(prob)) == -5
    r = oracle.run_uniform(prob, keep_steps=False)
    assert np.all(r["residual"] < prob.qerrortol)


def test_periodic_mass_conservation_and_ghosts(oracle):
    # Periodic x, Neumann y: the scheme stays conservative, and after a step
    # every periodic ghost column holds the opposite interior column.
    prob = W.config1(nsteps=3, n=32)
    prob.mthbc = (2, 2, 1, 1, 1, 1)
    r = oracle.run_uniform(prob, nsteps=3)
    m0 = prob.h ** 2 * prob.c0.sum()
    assert np.all(np.abs(r["mass"] - m0) < 1e-9)
    q = r["q"][-1]
    assert np.array_equal(q[0, 1:-1], q[32, 1:-1]) and np.array_equal(q[33, 1:-1], q[1, 1:-1])
