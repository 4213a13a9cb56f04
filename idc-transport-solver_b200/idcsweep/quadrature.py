"""Level-symmetric S_N ordinate sets for the 2-D sweep.

The reference ships Chebyshev-Legendre, spherical-triangle and Lebedev sets
(utils/Quadrule/OrdinateSet.cpp:37-59) but no level-symmetric set; the S4/S8/S12/S16 sets
(12/40/84/144 ordinates in 2-D) are generated here.

Construction (the LQ_n family of Lathrop & Carlson, as presented in Lewis & Miller,
"Computational Methods of Neutron Transport", ch. 4):

* one octant holds the points (mu_i, mu_j, mu_k) with i + j + k = N/2 + 2 (1-based), where
  mu_i^2 = mu_1^2 + (i - 1) * 2 (1 - 3 mu_1^2) / (N - 2), so every point lies on the unit sphere;
* points that are permutations of one another share a weight (a symmetry class);
* the class weights integrate the even moments of one direction cosine exactly up to degree N;
  mu_1 is the free parameter that makes that possible (S4, S8, S12 give mu_1 = 0.3500212,
  0.2182179, 0.1672127).  For S16 those conditions leave mu_1 free and it is fitted to all even
  monomials x^2a y^2b z^2c of degree <= 16 instead (``level_symmetric_octant`` has the details).

Values are computed, not tabulated; ``moment_errors`` reports how well each set integrates the
monomials x^2a y^2b z^2c, and the tests check it.

The 2-D set keeps the upper hemisphere (mu > 0) and doubles its weights, the same folding the
reference applies with ``SymmetricReduce`` (OrdinateSet.cpp:1171), so weights sum to 4*pi.  It is
sorted into the reference's quadrant order (OrdinateSet.cpp:658-700, 937): quadrant 0 xi>0,eta>0;
1 xi>0,eta<0; 2 xi<0,eta>0; 3 xi<0,eta<0, and inside a quadrant by decreasing (xi, eta), the order
``OrdinateData::Compare`` (OrdinateSet.cpp:982) produces.
"""
from __future__ import annotations

import functools
import itertools
import math

import numpy as np

__all__ = ["level_symmetric_octant", "level_symmetric_2d", "moment_errors", "SN_COUNTS_2D"]

SN_COUNTS_2D = {2: 4, 4: 12, 6: 24, 8: 40, 10: 60, 12: 84, 14: 112, 16: 144}


def _octant_moment(a: int, b: int, c: int) -> float:
    """(1 / (pi/2)) * integral over the first octant of x^2a y^2b z^2c dOmega."""
    g = math.gamma
    full = 2.0 * g(a + 0.5) * g(b + 0.5) * g(c + 0.5) / g(a + b + c + 1.5)
    return full / 8.0 / (math.pi / 2.0)


def _levels(N: int, mu1: float) -> np.ndarray:
    n = N // 2
    if N == 2:
        return np.array([math.sqrt(1.0 / 3.0)])
    delta = 2.0 * (1.0 - 3.0 * mu1 * mu1) / (N - 2)
    return np.sqrt(mu1 * mu1 + delta * np.arange(n))


def _octant_points(N: int):
    """Index triples (i, j, k), 0-based, and their symmetry class ids."""
    n = N // 2
    triples = [(i, j, k) for i in range(n) for j in range(n) for k in range(n) if i + j + k == n - 1]
    classes = sorted({tuple(sorted(t)) for t in triples})
    cls_id = [classes.index(tuple(sorted(t))) for t in triples]
    return triples, cls_id, len(classes)


def _moment_system(N: int, mu1: float):
    """Least-squares system for the class weights: one row per even monomial x^2a y^2b z^2c with
    a + b + c <= N/2 (rows for permuted exponents coincide by symmetry and are kept once)."""
    triples, cls_id, ncls = _octant_points(N)
    lev = _levels(N, mu1)
    pts = np.array([[lev[i], lev[j], lev[k]] for (i, j, k) in triples])
    n = N // 2
    mons = sorted({tuple(sorted(t)) for t in itertools.product(range(n + 1), repeat=3) if sum(t) <= n})
    M = np.zeros((len(mons), ncls))
    t = np.zeros(len(mons))
    for r, (a, b, c) in enumerate(mons):
        for p, cid in zip(pts, cls_id):
            M[r, cid] += p[0] ** (2 * a) * p[1] ** (2 * b) * p[2] ** (2 * c)
        t[r] = _octant_moment(a, b, c)
    return pts, cls_id, M, t


def _fit(N: int, mu1: float):
    pts, cls_id, M, t = _moment_system(N, mu1)
    w, *_ = np.linalg.lstsq(M, t, rcond=None)
    res = M @ w - t
    return pts, np.array([w[c] for c in cls_id]), float(res @ res)


def _pure_weights(N: int, mu1: float):
    """Class weights from the square system of pure moments x^(2n), n = 0, 2, 3, ..., W (n = 1
    follows from n = 0 because every point lies on the sphere).  None when that system is singular."""
    triples, cls_id, ncls = _octant_points(N)
    lev = _levels(N, mu1)
    pts = np.array([[lev[i], lev[j], lev[k]] for (i, j, k) in triples])
    orders = [0] + list(range(2, ncls + 1))
    M = np.zeros((ncls, ncls))
    for r, m in enumerate(orders):
        for p, cid in zip(pts, cls_id):
            M[r, cid] += p[0] ** (2 * m)
    t = np.array([_octant_moment(m, 0, 0) for m in orders])
    if np.linalg.cond(M) > 1e13:
        return pts, None
    w = np.linalg.solve(M, t)
    return pts, np.array([w[c] for c in cls_id])


def _pure_residual(N: int, mu1: float, n: int) -> float:
    pts, w = _pure_weights(N, mu1)
    if w is None:
        return float("nan")
    return float(np.sum(w * pts[:, 0] ** (2 * n)) - _octant_moment(n, 0, 0))


@functools.lru_cache(maxsize=None)
def level_symmetric_octant(N: int):
    """Returns (mu1, points[M,3], weights[M]) for one octant; weights sum to 1.

    Method A (LQ_n): weights integrate the pure even moments x^(2n), n <= N/2, exactly; with W
    weight classes the square system n = 0, 2..W fixes the weights at a given mu1 and mu1 is the
    root of the residual of moment W + 1.  Used when that moment is still one of the defining ones
    (S4, S6, S8, S10, S12).  Method B (when the defining moments leave mu1 free, S14/S16): weights
    by least squares on all even monomials x^2a y^2b z^2c with a + b + c <= N/2, mu1 minimising
    that residual, weights rescaled so that the zeroth moment is exact."""
    if N < 2 or N % 2:
        raise ValueError(f"S_N order must be even and >= 2, got {N}")
    if N == 2:
        p = np.full((1, 3), math.sqrt(1.0 / 3.0))
        return p[0, 0], p, np.ones(1)
    hi = math.sqrt(1.0 / 3.0)
    grid = np.linspace(1e-3, hi - 1e-3, 1001)
    _, _, ncls = _octant_points(N)

    if ncls + 1 <= N // 2:
        f = lambda m: _pure_residual(N, m, ncls + 1)
        vals = [f(m) for m in grid]
        for a, b, fa, fb in zip(grid[:-1], grid[1:], vals[:-1], vals[1:]):
            if not (np.isfinite(fa) and np.isfinite(fb)) or fa * fb > 0.0:
                continue
            for _ in range(200):  # bisection to machine precision
                c = 0.5 * (a + b)
                fc = f(c)
                if fa * fc <= 0.0:
                    b, fb = c, fc
                else:
                    a, fa = c, fc
            mu1 = 0.5 * (a + b)
            pts, w = _pure_weights(N, mu1)
            if w is not None and w.min() > 0:
                return mu1, pts, w
        raise RuntimeError(f"no level-symmetric S{N} set with positive weights")

    def f(m):
        _, w, r = _fit(N, m)
        return r if w.min() > 0 else np.inf

    vals = np.array([f(m) for m in grid])
    k = int(np.argmin(vals))
    a, b = grid[max(k - 1, 0)], grid[min(k + 1, len(grid) - 1)]
    gr = (math.sqrt(5.0) - 1.0) / 2.0
    for _ in range(120):  # golden-section search on the bracketing grid cell
        c = b - gr * (b - a)
        d = a + gr * (b - a)
        if f(c) < f(d):
            b = d
        else:
            a = c
    mu1 = 0.5 * (a + b)
    pts, w, _ = _fit(N, mu1)
    if w.min() <= 0:
        raise RuntimeError(f"no level-symmetric S{N} set with positive weights")
    return mu1, pts, w / w.sum()


def moment_errors(N: int, max_order: int | None = None) -> dict:
    """Absolute errors of the octant rule on x^2a y^2b z^2c for 2(a+b+c) <= max_order."""
    _, pts, w = level_symmetric_octant(N)
    max_order = N if max_order is None else max_order
    out = {}
    for a, b, c in itertools.product(range(max_order // 2 + 1), repeat=3):
        if 2 * (a + b + c) > max_order:
            continue
        approx = float(np.sum(w * pts[:, 0] ** (2 * a) * pts[:, 1] ** (2 * b) * pts[:, 2] ** (2 * c)))
        out[(a, b, c)] = approx - _octant_moment(a, b, c)
    return out


@functools.lru_cache(maxsize=None)
def _level_symmetric_2d_cached(N: int):
    _, pts, w = level_symmetric_octant(N)
    # first-octant weight fraction -> whole-sphere weight 4*pi/8 per octant, x2 for the +-mu fold
    wq = w * (4.0 * math.pi / 8.0) * 2.0
    xi_l, eta_l, w_l = [], [], []
    bounds = [0]
    for sx, sy in ((+1, +1), (+1, -1), (-1, +1), (-1, -1)):
        q = [(sx * p[0], sy * p[1], ww) for p, ww in zip(pts, wq)]
        q.sort(key=lambda t: (t[0], t[1]), reverse=True)
        xi_l += [t[0] for t in q]
        eta_l += [t[1] for t in q]
        w_l += [t[2] for t in q]
        bounds.append(len(xi_l))
    return (np.array(xi_l), np.array(eta_l), np.array(w_l), np.array(bounds, dtype=np.int64))


def level_symmetric_2d(N: int):
    """2-D level-symmetric S_N set: (xi, eta, w, quad_bounds[5]) in the reference's ordering."""
    xi, eta, w, b = _level_symmetric_2d_cached(N)
    return xi.copy(), eta.copy(), w.copy(), b.copy()
