"""The boundary conditions, high-order cross sections and DG degree 3 on degenerate grids (one cell wide or
high, a single cell), against the reference compiled from its sources (oracle/_ref): the edge cells are then
ghost-cell neighbours on both sides, which is where the reflection, halo-synchronisation and tensor kernels'
index arithmetic meets its limits."""
import os

import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import project, random_problem
from oracle.bindings import REFERENCE_SO, Reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REFERENCE_SO), reason="oracle/_ref/libidcref.so not built")]

GRIDS = [(1, 5), (6, 1), (1, 1), (2, 3)]


@pytest.fixture(scope="module")
def ref():
    return Reference(REFERENCE_SO)


def _ctx(P, reflect=0, periodic=False):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by, sigma_degree=P.sigma_degree)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    if reflect:
        ctx.set_reflecting(reflect)
    if periodic:
        ctx.set_periodic(True)
    return ctx


def _high_order(P, seed):
    """The problem's cross sections replaced by smooth positive ones of degree p (Legendre moments per cell)."""
    rng = np.random.default_rng(seed)
    a, b = rng.uniform(0.5, 2.0, 2)
    st = project(lambda x, y: 1.5 + 0.5 * np.sin(a * x + b * y), P.nx, P.ny, P.ax, P.bx, P.ay, P.by, P.p,
                 limiter=False)
    ss = project(lambda x, y: 0.6 * (1.5 + 0.5 * np.sin(a * x + b * y)), P.nx, P.ny, P.ax, P.bx, P.ay, P.by, P.p,
                 limiter=False)
    P.sigma_t, P.sigma_s, P.sigma_degree = np.ascontiguousarray(st.ravel()), np.ascontiguousarray(ss.ravel()), P.p
    return P


@pytest.mark.parametrize("nx,ny", GRIDS)
@pytest.mark.parametrize("reflect", [abi.EDGE_X_MIN | abi.EDGE_Y_MAX, 15])
def test_reflecting_sweep_and_source_iteration(ref, nx, ny, reflect):
    P = random_problem(nx, ny, 1, 4, seed=7 * nx + ny, dt=0.4, sigma_range=(0.5, 3.0))
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-13, max_its=5000, reflect=reflect) as h:
        want = h.sweep(P.source, P.dt)
        want_si = h.source_iteration(P.source, P.dt)
    with _ctx(P, reflect=reflect) as ctx:
        psi = P.source.copy()
        ctx.sweep(psi, P.dt)
        assert rel_err(psi, want) < 1e-12
        psi = P.source.copy()
        ctx.source_iteration(psi, P.dt, abs_tol=1e-13, max_its=5000)
        assert rel_err(psi[1:-1, 1:-1], want_si[1:-1, 1:-1]) < 1e-11


@pytest.mark.parametrize("nx,ny", GRIDS)
def test_periodic_source_iteration_and_gmres(ref, nx, ny):
    P = random_problem(nx, ny, 1, 4, seed=11 * nx + ny, dt=0.4, sigma_range=(0.5, 3.0))
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-13, max_its=5000, periodic=True) as h:
        want = h.source_iteration(P.source, P.dt)
    with _ctx(P, periodic=True) as ctx:
        psi = P.source.copy()
        ctx.source_iteration(psi, P.dt, abs_tol=1e-13, max_its=5000)
        assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-11
        psi = P.source.copy()
        ctx.gmres_solve(psi, P.dt, abs_tol=1e-13, restart=30, max_its=3000)
        assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-10


@pytest.mark.parametrize("nx,ny", GRIDS)
@pytest.mark.parametrize("p", [2, 3])
def test_high_order_sigma_and_dg3_sweeps(ref, nx, ny, p):
    P = random_problem(nx, ny, p, 4, seed=13 * nx + ny + p, dt=0.4, sigma_range=(0.5, 3.0))
    for high in (False, True):
        if high:
            P = _high_order(P, seed=nx + ny)
        with ref.open(to_oracle(P), P.dt, sigma_degree=P.sigma_degree) as h:
            want = h.sweep(P.source, P.dt)
        with _ctx(P) as ctx:
            psi = P.source.copy()
            phi = np.zeros(P.phi_shape())
            ctx.sweep(psi, P.dt, phi)
        assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-12
        assert rel_err(phi[1:-1, 1:-1], np.tensordot(want[1:-1, 1:-1], P.w, axes=([2], [0]))) < 1e-12
