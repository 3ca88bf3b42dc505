"""Seeded synthetic inputs for the Cahn-Hilliard workloads.

The reference's own example (problems/simple_cahn-hilliard) is driven by
Fortran namelists and a hard-coded QInit2D (problem.f90:58-101).  The
benchmark workloads here replace QInit with seeded random fields.  Every
array is produced on the host by SplitMix64 so that the CUDA path and the CPU
oracle receive bit-identical inputs.

Variable mapping: the reference potential F(c) = alpha c^2 (c-1)^2 / 4
(problem.f90:769-780) has its wells at c = 0 and c = 1.  A field quoted as
phi in [-1, 1] maps to c = (1 + phi) / 2; errors are reported in c.
"""
from __future__ import annotations

import dataclasses
import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n successive SplitMix64 outputs of the stream `seed`, as uint64."""
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int, a: float, b: float, offset: int = 0) -> np.ndarray:
    """U(a, b) = a + (b - a) * ((x >> 11) * 2^-53), float64."""
    x = splitmix64(seed, n, offset)
    u = (x >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
    return a + (b - a) * u


@dataclasses.dataclass
class Problem:
    """One Cahn-Hilliard solve on a uniform root grid of [0,1]^d."""

    ndims: int
    mx: tuple
    eps: float
    dt: float
    nsteps: int
    qerrortol: float
    alpha: float = 1.0
    maxvcycles: int = 20
    nsmoothingpasses: int = 2
    minlevel: int = 1          # 1 = automatic (lib/bsamroutines.f90:287-301)
    mthbc: tuple = (1, 1, 1, 1, 1, 1)
    c0: np.ndarray | None = None   # interior composition, Fortran order
    xupper: tuple = (1.0, 1.0, 1.0)  # domain [0, xupper]; dx must be equal in all dims
    # Seeded form (c0 = cbar + amp * uniform(seed, cells, -1, 1)): what the
    # device-side initialiser of the batch engine draws.
    seed: int | None = None
    cbar: float = 0.5
    amp: float = 0.0
    # Refined levels regridded every step (served AMR requests, 2D): the
    # initial state is then the circular drop of the AMR workload, seeded by
    # `seed` (bsam_b200.amr.build), not the seeded uniform form above.
    maxlevel: int = 0

    @property
    def h(self) -> float:
        return self.xupper[0] / self.mx[0]

    def q0(self) -> np.ndarray:
        """Root q with ghost ring, Fortran layout (0:mx+1)^d x 2."""
        c0 = self.c0
        if c0 is None:
            cells = int(np.prod(self.mx[:self.ndims]))
            c0 = self.cbar + self.amp * uniform(self.seed, cells, -1.0, 1.0)
        return initial_q(self.ndims, self.mx, c0, self.h, self.eps, self.alpha)


def seeded(ndims: int, n: int, eps: float, nsteps: int, seed: int, cbar: float, amp: float,
           dt: float = 1e-4, qerrortol: float = 1e-8) -> Problem:
    """A problem whose initial composition is cbar + amp * U(-1, 1) from the
    SplitMix64 stream `seed` (drawn lazily; the batch engine can draw it on
    the device)."""
    mx = (n, n, n if ndims == 3 else 1)
    return Problem(ndims=ndims, mx=mx, eps=eps, dt=dt, nsteps=nsteps, qerrortol=qerrortol,
                   seed=seed, cbar=cbar, amp=amp)


def config5(nreq: int, rate: float, seed: int = 5) -> list:
    """Serving stream: Poisson arrivals at `rate` per second; 70 % 2D with
    side in {64, 128, 256, 512}, 30 % 3D with side in {32, 64, 128}; steps
    uniform in 1..50; eps ~ U(0.005, 0.02); dt = 1e-4; c0 = 0.5 + 0.025
    U(-1, 1) (seeded per request); residual 1e-8.  A 2D request has 0, 1 or
    2 refined levels (uniform); one with refined levels starts from the
    circular drop of the AMR workload and regrids every step.  Returns
    (arrival_s, Problem) pairs in arrival order."""
    gaps = -np.log(1.0 - uniform(seed, nreq, 0.0, 1.0)) / rate
    arrival = np.cumsum(gaps)
    is3 = uniform(seed + 1, nreq, 0.0, 1.0) < 0.3
    pick = splitmix64(seed + 2, nreq)
    steps = 1 + (splitmix64(seed + 3, nreq) % np.uint64(50)).astype(np.int64)
    eps = uniform(seed + 4, nreq, 0.005, 0.02)
    levels = (splitmix64(seed + 5, nreq) % np.uint64(3)).astype(np.int64)
    out = []
    for r in range(nreq):
        if is3[r]:
            n, nd = (32, 64, 128)[int(pick[r] % np.uint64(3))], 3
        else:
            n, nd = (64, 128, 256, 512)[int(pick[r] % np.uint64(4))], 2
        p = seeded(nd, n, float(eps[r]), int(steps[r]), seed=7919 * (seed + 1) + r,
                   cbar=0.5, amp=0.025)
        if nd == 2:
            p.maxlevel = int(levels[r])
        out.append((float(arrival[r]), p))
    return out


def _dfc(c, alpha):
    cmh = c - 0.5
    return cmh * cmh * cmh * alpha


def _dfe(c, alpha):
    return (c - 0.5) * alpha / 4.0


def initial_q(ndims, mx, c0, h, eps, alpha) -> np.ndarray:
    """q(0:mx+1, ..., 1:2) with c0 in the interior, Neumann ghosts, and
    mu0 = Dfc(c0) - Dfe(c0) - eps^2/h^2 ULap(c0), the chemical potential
    that makes the operator's second row consistent at c = c_old."""
    shape = tuple(m + 2 for m in mx[:ndims])
    c = np.zeros(shape, order="F")
    inner = tuple(slice(1, m + 1) for m in mx[:ndims])
    c[inner] = np.asarray(c0, dtype=np.float64).reshape(mx[:ndims], order="F")
    # Neumann reflection, applied dimension by dimension (boundary.f90:661-738).
    for d in range(ndims):
        lo = [slice(None)] * ndims
        hi = [slice(None)] * ndims
        lo[d], hi[d] = 0, shape[d] - 1
        s_lo = [slice(None)] * ndims
        s_hi = [slice(None)] * ndims
        s_lo[d], s_hi[d] = 1, shape[d] - 2
        c[tuple(lo)] = c[tuple(s_lo)]
        c[tuple(hi)] = c[tuple(s_hi)]
    lap = -2.0 * ndims * c[inner]
    for d in range(ndims):
        p = list(inner)
        m = list(inner)
        p[d] = slice(2, mx[d] + 2)
        m[d] = slice(0, mx[d])
        lap = lap + c[tuple(p)] + c[tuple(m)]
    mu = np.zeros(shape, order="F")
    mu[inner] = _dfc(c[inner], alpha) - _dfe(c[inner], alpha) - (eps * eps / (h * h)) * lap
    for d in range(ndims):
        lo = [slice(None)] * ndims
        hi = [slice(None)] * ndims
        lo[d], hi[d] = 0, shape[d] - 1
        s_lo = [slice(None)] * ndims
        s_hi = [slice(None)] * ndims
        s_lo[d], s_hi[d] = 1, shape[d] - 2
        mu[tuple(lo)] = mu[tuple(s_lo)]
        mu[tuple(hi)] = mu[tuple(s_hi)]
    q = np.zeros(shape + (2,), order="F")
    q[..., 0] = c
    q[..., 1] = mu
    return q


def config1(nsteps: int = 20, seed: int = 1, n: int = 128) -> Problem:
    """2D 128x128 uniform, eps=0.01, dt=1e-4, V(2,2) to residual 1e-9,
    phi0 = 0.05 U(-1,1) -> c0 = 0.5 + 0.025 U(-1,1)."""
    u = uniform(seed, n * n, -1.0, 1.0)
    return Problem(ndims=2, mx=(n, n, 1), eps=0.01, dt=1e-4, nsteps=nsteps,
                   qerrortol=1e-9, c0=0.5 + 0.025 * u)


def config3(nsteps: int = 20, seed: int = 3, n: int = 128) -> Problem:
    """3D 128^3 uniform, eps=0.02, dt=1e-4, residual 1e-8,
    phi0 = 0.1 + 0.05 U(-1,1) -> c0 = 0.55 + 0.025 U(-1,1)."""
    u = uniform(seed, n * n * n, -1.0, 1.0)
    return Problem(ndims=3, mx=(n, n, n), eps=0.02, dt=1e-4, nsteps=nsteps,
                   qerrortol=1e-8, c0=0.55 + 0.025 * u)


BATCH_SIDES = (64, 96, 128, 192, 256)


def config4(nprob: int = 512, nsteps: int = 10, seed: int = 4) -> list:
    """Batched: sides uniform over BATCH_SIDES, eps ~ U(0.005, 0.02),
    phi0 = m + 0.05 U(-1, 1) with m ~ U(-0.3, 0.3), i.e. in the reference's
    variable c0 = (1 + m)/2 + 0.025 U(-1, 1) (seeded form, drawn per problem
    from its own stream); dt = 1e-4; residual 1e-8."""
    sel = splitmix64(seed, nprob) % np.uint64(len(BATCH_SIDES))
    eps = uniform(seed + 1, nprob, 0.005, 0.02)
    mean = uniform(seed + 2, nprob, -0.3, 0.3)
    out = []
    for p in range(nprob):
        n = BATCH_SIDES[int(sel[p])]
        out.append(seeded(2, n, float(eps[p]), nsteps, seed=1000003 * (seed + 1) + p,
                          cbar=0.5 * (1.0 + float(mean[p])), amp=0.025))
    return out
