"""DG degree 3 (P = 4, 16 modes per cell) against the reference compiled from its sources (oracle/_ref) at
Global::DG_degree = 3: it runs on the elimination kernel in FP64 (the lane and modal kernels cover degrees 0-2).
The sweep, Smv and Lmv, source iteration and GMRES (+ DSA), with piecewise-constant and high-order cross
sections and on a periodic grid, and the paths that stay unsupported."""
import os

import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import lognormal, random_problem, smooth_sigma
from oracle.bindings import REFERENCE_SO, Reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REFERENCE_SO), reason="oracle/_ref/libidcref.so not built")]


@pytest.fixture(scope="module")
def ref():
    return Reference(REFERENCE_SO)


def _ctx(P, periodic=False):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by, sigma_degree=P.sigma_degree)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    if periodic:
        ctx.set_periodic(True)
    return ctx


def _phi(P, psi):
    return np.tensordot(psi[1:-1, 1:-1], P.w, axes=([2], [0]))


@pytest.mark.parametrize("kind,sn,dt", [("random", 4, 0.4), ("random", 8, np.inf), ("smooth", 4, 0.5)])
def test_sweep_matches_reference(ref, kind, sn, dt):
    P = (random_problem(9, 7, 3, sn, seed=31 + sn, dt=dt) if kind == "random"
         else smooth_sigma(8, 3, sn, seed=33, dt=dt))
    with ref.open(to_oracle(P), P.dt, sigma_degree=P.sigma_degree) as h:
        want = h.sweep(P.source, P.dt)
    with _ctx(P) as ctx:
        psi = P.source.copy()
        phi = np.zeros(P.phi_shape())
        ctx.sweep(psi, P.dt, phi)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-12
    assert rel_err(phi[1:-1, 1:-1], _phi(P, want)) < 1e-12


@pytest.mark.parametrize("kind", ["random", "smooth"])
def test_smv_lmv_match_reference(ref, kind):
    P = random_problem(7, 6, 3, 4, seed=41) if kind == "random" else smooth_sigma(6, 3, 4, seed=42, dt=0.5)
    rng = np.random.default_rng(4)
    phi = np.zeros(P.phi_shape())
    phi[1:-1, 1:-1] = rng.standard_normal(phi[1:-1, 1:-1].shape)
    y0 = rng.standard_normal(P.psi_shape())
    x = rng.standard_normal(P.psi_shape())
    with ref.open(to_oracle(P), P.dt, sigma_degree=P.sigma_degree) as h:
        smv_want = h.smv(phi, y0, 0.7, 1.3)
        lmv_want = h.lmv(x, y0, 0.9, 0.4)
    with _ctx(P) as ctx:
        y = y0.copy()
        ctx.smv(0.7, 1.3, phi, y)
        assert rel_err(y[1:-1, 1:-1], smv_want[1:-1, 1:-1]) < 1e-13
        y = y0.copy()
        ctx.lmv(0.9, 0.4, x, y)
        assert rel_err(y[1:-1, 1:-1], lmv_want[1:-1, 1:-1]) < 1e-13


@pytest.mark.parametrize("kind,periodic", [("lognormal", False), ("smooth", False), ("lognormal", True)])
def test_source_iteration_and_gmres_match_reference(ref, kind, periodic):
    P = (lognormal(10, 3, 4, seed=12, c_range=(0.3, 0.8), dt=0.5) if kind == "lognormal"
         else smooth_sigma(8, 3, 4, seed=13, dt=0.5, c_range=(0.4, 0.8)))
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-13, max_its=5000, sigma_degree=P.sigma_degree,
                  periodic=periodic) as h:
        want = h.source_iteration(P.source, P.dt)
    phi_want = _phi(P, want)
    with _ctx(P, periodic) as ctx:
        psi = P.source.copy()
        its, err = ctx.source_iteration(psi, P.dt, abs_tol=1e-13, max_its=5000)
        assert err <= 1e-13
        assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-11
        for dsa in (False, True):
            if dsa:
                ctx.set_preconditioner(abi.PRECOND_DSA, 20)
            psi = P.source.copy()
            its, res = ctx.gmres_solve(psi, P.dt, abs_tol=1e-12, restart=30, max_its=3000)
            assert res <= 1e-12
            assert rel_err(_phi(P, psi), phi_want) < 1e-10


def test_unsupported_at_dg_degree_3():
    P = random_problem(6, 5, 3, 4, seed=3, dt=0.5)
    with _ctx(P) as ctx:
        for call in (lambda: ctx.sweep(P.source.copy(), P.dt, None, abi.PREC_FP32),
                     lambda: ctx.sweep(P.source.copy(), P.dt, None, abi.PREC_FP32_REFINED),
                     lambda: ctx.sweep_adjoint(P.source, np.zeros(P.psi_shape()), P.dt),
                     lambda: ctx.idc_integrate(P.source.copy(), P.source, 0.1, 1, 3, 1),
                     lambda: ctx.set_reflecting(abi.EDGE_X_MIN) or ctx.sweep(P.source.copy(), P.dt)):
            with pytest.raises(abi.IdcError) as e:
                call()
            assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        ctx.set_reflecting(0)
        with pytest.raises(abi.IdcError) as e:
            with abi.Batch() as b:
                b.add(ctx)
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED


def test_implicit_idc_matches_reference_integrator(ref):
    """IDC time stepping with implicit scattering at DG degree 3 against the reference's IDCIntegrator."""
    P = random_problem(6, 7, 3, 4, seed=31, dt=0.05, inflow=False, sigma_range=(0.5, 4.0))
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = 0.05
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-14, max_its=100000) as h:
        want = h.idc_steps(psi0, P.source, P.dt, 2, 3, 2, si_abs_tol=1e-14)
    with _ctx(P) as ctx:
        psi = psi0.copy()
        ctx.idc_integrate(psi, P.source, P.dt, 2, 3, 2, abi.SCATTER_IMPLICIT, abi.PREC_FP64, abs_tol=1e-14)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-10
