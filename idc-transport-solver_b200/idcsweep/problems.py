"""Seeded synthetic problems with the benchmark shapes, on the reference's halo-padded layouts.

* ``lattice``  - the reference's lattice problem (utils/Problems/LatticeProblem.cpp:173-300): 7x7 unit
  blocks on [0,7]^2, absorber blocks sigma_t = 10, sigma_s = 0, elsewhere sigma_t = sigma_s = 1, unit
  isotropic source in [3,4]^2.  Cross sections are projected to piecewise constants and the source to
  Q_p by the reference's 14-point Gauss-Legendre tensor projection with its positivity limiter
  (ComputeProjection, utils/init.cpp:50-300); the angular source is Q/(4 pi) on every ordinate
  (init.cpp:920-925).
* ``lognormal`` - per-cell log-normal sigma_t with a uniform (or fixed) scattering ratio and a given
  isotropic source, the heterogeneous-medium problems of the benchmark configurations.
* ``random_problem`` - small random problems for parity tests (random sources including inflow
  values on the ghost cells).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from numpy.polynomial import legendre as L

from .quadrature import level_symmetric_2d


@dataclass
class Problem:
    nx: int
    ny: int
    p: int
    xi: np.ndarray
    eta: np.ndarray
    w: np.ndarray
    quad: np.ndarray
    sigma_t: np.ndarray          # (nx+2)*(ny+2), times (p+1)^2 Legendre moments when sigma_degree = p
    sigma_s: np.ndarray          # the same layout as sigma_t
    source: np.ndarray           # psi-shaped angular source (nx+2, ny+2, nq, p+1, p+1)
    ax: float = 0.0
    bx: float = 1.0
    ay: float = 0.0
    by: float = 1.0
    dt: float = math.inf
    meta: dict = field(default_factory=dict)
    sigma_degree: int = 0        # 0: one value per cell; p: the cross sections' Legendre moments [cell][u][v]

    @property
    def nq(self):
        return int(self.xi.size)

    @property
    def N(self):
        return (self.p + 1) ** 2

    @property
    def unknowns_per_sweep(self):
        return self.nx * self.ny * self.nq * self.N

    def psi_shape(self):
        return (self.nx + 2, self.ny + 2, self.nq, self.p + 1, self.p + 1)

    def phi_shape(self):
        return (self.nx + 2, self.ny + 2, self.p + 1, self.p + 1)


def _legendre(d, x):
    c = np.zeros(d + 1)
    c[d] = 1.0
    return L.legval(x, c)


def project(f, nx, ny, ax, bx, ay, by, degree, limiter=True, order=14):
    """ComputeProjection (utils/init.cpp:50-300) restated: returns (nx+2, ny+2, P, P) Legendre moments,
    ghost cells zero.  f is vectorised over (x, y)."""
    P = degree + 1
    nodes, weights = L.leggauss(order)
    dx, dy = (bx - ax) / nx, (by - ay) / ny
    out = np.zeros((nx + 2, ny + 2, P, P))
    ic = np.arange(nx)[:, None, None, None]
    jc = np.arange(ny)[None, :, None, None]
    X = ax + ic * dx + (nodes[None, None, :, None] + 1.0) * dx / 2.0
    Y = ay + jc * dy + (nodes[None, None, None, :] + 1.0) * dy / 2.0
    F = f(np.broadcast_to(X, (nx, ny, order, order)), np.broadcast_to(Y, (nx, ny, order, order)))
    for d in range(P):
        for e in range(P):
            wt = (weights[:, None] * weights[None, :] * _legendre(d, nodes)[:, None] * _legendre(e, nodes)[None, :]
                  * (2 * d + 1) * (2 * e + 1) / 4.0)
            out[1:-1, 1:-1, d, e] = np.einsum("ijlm,lm->ij", F, wt)
    if limiter and degree > 0:
        s = np.linspace(-1.0, 1.0, 21)
        Ls = np.stack([_legendre(d, s) for d in range(P)])          # (P, 21)
        for i in range(1, nx + 1):
            for j in range(1, ny + 1):
                c = out[i, j]
                if c[0, 0] < 0.0:
                    continue

                def negative(theta):
                    cc = c * theta
                    cc[0, 0] = c[0, 0]
                    vals = np.einsum("de,dl,em->lm", cc, Ls, Ls)
                    return bool((vals < 0.0).any())

                if not negative(1.0):
                    continue
                lo, hi = 0.0, 1.0
                while hi - lo > 1e-14:
                    mid = 0.5 * (lo + hi)
                    if negative(mid):
                        hi = mid
                    else:
                        lo = mid
                c00 = c[0, 0]
                out[i, j] *= lo
                out[i, j, 0, 0] = c00
    return out


def _lattice_sigma_t(x, y):
    absorber = np.zeros_like(x, dtype=bool)
    blk = lambda a, b, c, d: (x > a) & (x <= b) & (y > c) & (y <= d)
    for (a, b, ys) in ((1, 2, ((1, 2), (3, 4), (5, 6))), (2, 3, ((2, 3), (4, 5))), (3, 4, ((5, 6),)),
                       (4, 5, ((2, 3), (4, 5))), (5, 6, ((1, 2), (3, 4), (5, 6)))):
        for (c, d) in ys:
            absorber |= blk(a, b, c, d)
    return np.where(absorber, 10.0, 1.0)


def _lattice_sigma_s(x, y):
    return np.where(_lattice_sigma_t(x, y) > 5.0, 0.0, 1.0)


def _lattice_source(x, y):
    return np.where((x > 3.0) & (x < 4.0) & (y > 3.0) & (y < 4.0), 1.0, 0.0)


def _isotropic_source(q_moments: np.ndarray, nq: int) -> np.ndarray:
    """(nx+2, ny+2, P, P) source moments -> psi-shaped angular source Q/(4 pi), ghosts included."""
    src = np.repeat((q_moments / (4.0 * math.pi))[:, :, None, :, :], nq, axis=2)
    return np.ascontiguousarray(src)


def lattice(n: int, p: int, sn: int, dt: float = 0.01) -> Problem:
    xi, eta, w, qb = level_symmetric_2d(sn)
    st = project(_lattice_sigma_t, n, n, 0.0, 7.0, 0.0, 7.0, 0, limiter=False)[..., 0, 0]
    ss = project(_lattice_sigma_s, n, n, 0.0, 7.0, 0.0, 7.0, 0, limiter=False)[..., 0, 0]
    q = project(_lattice_source, n, n, 0.0, 7.0, 0.0, 7.0, p)
    return Problem(n, n, p, xi, eta, w, qb, np.ascontiguousarray(st.ravel()), np.ascontiguousarray(ss.ravel()),
                   _isotropic_source(q, xi.size), 0.0, 7.0, 0.0, 7.0, dt, {"kind": "lattice", "sn": sn})


def lognormal(n: int, p: int, sn: int, seed: int, median: float = 1.0, log_sd: float = 1.0,
              c_range=(0.5, 0.999), c_fixed: float | None = None, source: str = "uniform",
              length: float = 7.0, dt: float = math.inf) -> Problem:
    """Log-normal per-cell sigma_t (draws: sigma_t, then c, numpy default_rng(seed)), sigma_s = c sigma_t.
    source: "uniform" (Q = 1 everywhere) or "gaussian" (width 2 cells at (L/3, L/2))."""
    rng = np.random.default_rng(seed)
    xi, eta, w, qb = level_symmetric_2d(sn)
    st = np.zeros((n + 2, n + 2))
    st[1:-1, 1:-1] = median * np.exp(log_sd * rng.standard_normal((n, n)))
    c = np.full((n, n), c_fixed) if c_fixed is not None else rng.uniform(c_range[0], c_range[1], (n, n))
    ss = np.zeros_like(st)
    ss[1:-1, 1:-1] = c * st[1:-1, 1:-1]
    if source == "uniform":
        q = np.zeros((n + 2, n + 2, p + 1, p + 1))
        q[1:-1, 1:-1, 0, 0] = 1.0
    elif source == "gaussian":
        hw = 2.0 * length / n
        cx, cy = length / 3.0, length / 2.0
        q = project(lambda x, y: np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * hw * hw)), n, n, 0.0, length, 0.0,
                    length, p)
    else:
        raise ValueError(source)
    return Problem(n, n, p, xi, eta, w, qb, np.ascontiguousarray(st.ravel()), np.ascontiguousarray(ss.ravel()),
                   _isotropic_source(q, xi.size), 0.0, length, 0.0, length, dt,
                   {"kind": "lognormal", "sn": sn, "seed": seed})


def random_problem(nx: int, ny: int, p: int, sn: int, seed: int, dt: float = math.inf, inflow: bool = True,
                   sigma_range=(0.01, 20.0)) -> Problem:
    """Random cross sections (log-uniform over sigma_range), random scattering ratio in [0, 0.9],
    random angular source, random inflow values on the ghost cells (if inflow)."""
    rng = np.random.default_rng(seed)
    xi, eta, w, qb = level_symmetric_2d(sn)
    nq = xi.size
    lo, hi = np.log(sigma_range[0]), np.log(sigma_range[1])
    st = np.exp(rng.uniform(lo, hi, (nx + 2, ny + 2)))
    ss = st * rng.uniform(0.0, 0.9, (nx + 2, ny + 2))
    src = rng.uniform(-0.5, 1.0, (nx + 2, ny + 2, nq, p + 1, p + 1))
    if not inflow:
        src[0, :] = 0.0
        src[-1, :] = 0.0
        src[:, 0] = 0.0
        src[:, -1] = 0.0
    return Problem(nx, ny, p, xi, eta, w, qb, np.ascontiguousarray(st.ravel()), np.ascontiguousarray(ss.ravel()),
                   np.ascontiguousarray(src), 0.0, 1.0 * nx / max(nx, ny) * 2.0, 0.0, 1.0 * ny / max(nx, ny) * 2.0,
                   dt, {"kind": "random", "sn": sn, "seed": seed})


def smooth_sigma(n: int, p: int, sn: int, seed: int, dt: float = math.inf, c_range=(0.3, 0.8),
                 inflow: bool = True) -> Problem:
    """High-order cross sections (sigma_degree = p): smooth positive sigma_t(x, y) = 1.5 + sin/cos modes of random
    phase (values in [0.4, 2.6]) and sigma_s = c(x, y) sigma_t(x, y) with a smooth scattering ratio in c_range, both
    projected onto the cells' Legendre moments (ComputeProjection); random angular source and inflow values as
    random_problem draws them.  Domain [0, 2]^2."""
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0.0, 2.0 * np.pi, 4)
    xi, eta, w, qb = level_symmetric_2d(sn)
    nq = xi.size

    def st(x, y):
        return 1.5 + 0.6 * np.sin(2.1 * x + ph[0]) * np.cos(1.7 * y + ph[1]) + 0.5 * np.sin(3.3 * x * y + ph[2])

    def cr(x, y):
        return c_range[0] + (c_range[1] - c_range[0]) * 0.5 * (1.0 + np.sin(1.3 * x - 2.2 * y + ph[3]))

    mt = project(st, n, n, 0.0, 2.0, 0.0, 2.0, p, limiter=False)
    ms = project(lambda x, y: cr(x, y) * st(x, y), n, n, 0.0, 2.0, 0.0, 2.0, p, limiter=False)
    src = rng.uniform(-0.5, 1.0, (n + 2, n + 2, nq, p + 1, p + 1))
    if not inflow:
        src[0, :] = 0.0
        src[-1, :] = 0.0
        src[:, 0] = 0.0
        src[:, -1] = 0.0
    return Problem(n, n, p, xi, eta, w, qb, np.ascontiguousarray(mt.ravel()), np.ascontiguousarray(ms.ravel()),
                   np.ascontiguousarray(src), 0.0, 2.0, 0.0, 2.0, dt,
                   {"kind": "smooth-sigma", "sn": sn, "seed": seed}, sigma_degree=p)


def detector_window(P: Problem, cells: int = 16, cx: float = 2.0 / 3.0, cy: float = 0.5) -> np.ndarray:
    """Detector weights c (phi layout) of J = c . phi = the integrated scalar flux over a cells x cells window
    centred at (cx L, cy L): c = dx dy on the (0, 0) moment of the window's cells (the cell integral of the
    Legendre expansion), zero elsewhere."""
    dx, dy = (P.bx - P.ax) / P.nx, (P.by - P.ay) / P.ny
    m = min(cells, P.nx, P.ny)
    i0 = min(max(0, int(round(cx * P.nx - m / 2.0))), P.nx - m)
    j0 = min(max(0, int(round(cy * P.ny - m / 2.0))), P.ny - m)
    c = np.zeros(P.phi_shape())
    c[1 + i0:1 + i0 + m, 1 + j0:1 + j0 + m, 0, 0] = dx * dy
    return c
