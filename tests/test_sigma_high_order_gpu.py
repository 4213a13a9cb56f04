"""High-order cross sections (sigma_degree = p: each cell's Legendre moments of sigma_t and sigma_s) against the
reference compiled from its sources (oracle/_ref) with CrossSection objects of DG degree p, as Init builds them
when the deck does not ask for piecewise-constant cross sections: the sweep (CalcA's tensor branch), Smv and Lmv
(their sigma.DG_degree > 0 branches), source iteration and the Peierls GMRES (+ DSA) reaching the reference's
source-iteration fixed point, and the inputs that stay unsupported."""
import os

import numpy as np
import pytest
import torch

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import smooth_sigma
from oracle.bindings import REFERENCE_SO, Reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REFERENCE_SO), reason="oracle/_ref/libidcref.so not built")]


@pytest.fixture(scope="module")
def ref():
    return Reference(REFERENCE_SO)


def _ctx(P):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by, sigma_degree=P.sigma_degree)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    return ctx


def _phi(P, psi):
    return np.tensordot(psi[1:-1, 1:-1], P.w, axes=([2], [0]))


@pytest.mark.parametrize("p,sn,dt", [(1, 4, 0.5), (1, 8, np.inf), (2, 4, 0.3), (2, 6, np.inf)])
def test_sweep_matches_reference(ref, p, sn, dt):
    P = smooth_sigma(9, p, sn, seed=40 + p + sn, dt=dt)
    with ref.open(to_oracle(P), P.dt, sigma_degree=p) as h:
        want = h.sweep(P.source, P.dt)
    with _ctx(P) as ctx:
        psi = P.source.copy()
        phi = np.zeros(P.phi_shape())
        ctx.sweep(psi, P.dt, phi)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-12
    assert rel_err(phi[1:-1, 1:-1], _phi(P, want)) < 1e-12
    # the higher moments matter: the cell averages alone give another sweep
    N = P.N
    avg_t = np.ascontiguousarray(P.sigma_t.reshape(-1, N)[:, 0])
    with abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by) as c0:
        c0.set_ordinates(P.xi, P.eta, P.w, P.quad)
        c0.set_sigma(avg_t, None)
        psi0 = P.source.copy()
        c0.sweep(psi0, P.dt)
    assert rel_err(psi0[1:-1, 1:-1], want[1:-1, 1:-1]) > 1e-4


@pytest.mark.parametrize("p", [1, 2])
def test_smv_lmv_match_reference(ref, p):
    P = smooth_sigma(7, p, 4, seed=60 + p, dt=0.5)
    rng = np.random.default_rng(p)
    phi = np.zeros(P.phi_shape())
    phi[1:-1, 1:-1] = rng.standard_normal(phi[1:-1, 1:-1].shape)
    y0 = rng.standard_normal(P.psi_shape())
    x = rng.standard_normal(P.psi_shape())
    with ref.open(to_oracle(P), P.dt, sigma_degree=p) as h:
        smv_want = h.smv(phi, y0, 0.7, 1.3)
        lmv_want = h.lmv(x, y0, 0.9, 0.4)
    with _ctx(P) as ctx:
        y = y0.copy()
        ctx.smv(0.7, 1.3, phi, y)
        assert rel_err(y[1:-1, 1:-1], smv_want[1:-1, 1:-1]) < 1e-13
        y = y0.copy()
        ctx.lmv(0.9, 0.4, x, y)
        assert rel_err(y[1:-1, 1:-1], lmv_want[1:-1, 1:-1]) < 1e-13


@pytest.mark.parametrize("p,sn", [(1, 8), (2, 4)])
def test_source_iteration_and_gmres_match_reference(ref, p, sn):
    """SISolver::Solve with high-order cross sections, and the Peierls GMRES with and without DSA (whose diffusion
    coefficients are the cell averages) reaching the same fixed point."""
    P = smooth_sigma(12, p, sn, seed=7 + p, dt=0.5, c_range=(0.4, 0.85))
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-13, max_its=5000, sigma_degree=p) as h:
        want = h.source_iteration(P.source, P.dt)
    phi_want = _phi(P, want)
    with _ctx(P) as ctx:
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
            assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-10


def test_unsupported_with_high_order_cross_sections():
    P = smooth_sigma(6, 1, 4, seed=3, dt=0.5)
    with _ctx(P) as ctx:
        for call in (lambda: ctx.sweep(P.source.copy(), P.dt, None, abi.PREC_FP32),
                     lambda: ctx.sweep(P.source.copy(), P.dt, None, abi.PREC_FP32_REFINED),
                     lambda: ctx.gmres_solve(P.source.copy(), P.dt, precision=abi.PREC_FP32_IR),
                     lambda: ctx.idc_integrate(P.source.copy(), P.source, 0.1, 1, 3, 1),
                     lambda: ctx.set_reflecting(abi.EDGE_X_MIN) or ctx.sweep(P.source.copy(), P.dt)):
            with pytest.raises(abi.IdcError) as e:
                call()
            assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        ctx.set_reflecting(0)
        x = torch.zeros(P.psi_shape(), dtype=torch.float64, device="cuda")
        with pytest.raises(abi.IdcError) as e:
            ctx.lmv_transpose(1.0, 0.0, x.data_ptr(), x.data_ptr())
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        with pytest.raises(abi.IdcError) as e:
            with abi.Batch() as b:
                b.add(ctx)
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED


@pytest.mark.parametrize("p", [1, 2])
def test_implicit_idc_matches_reference_integrator(ref, p):
    """IDC time stepping with implicit scattering (GMRES substeps) against the reference's own IDCIntegrator
    (update form, Gauss-Lobatto nodes, SISolver substeps) with degree-p cross sections."""
    P = smooth_sigma(8, p, 4, seed=50 + p, dt=0.05, inflow=False)
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = 0.05
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-14, max_its=100000, sigma_degree=p) as h:
        want = h.idc_steps(psi0, P.source, P.dt, 2, 3, 2, si_abs_tol=1e-14)
    with _ctx(P) as ctx:
        psi = psi0.copy()
        ctx.idc_integrate(psi, P.source, P.dt, 2, 3, 2, abi.SCATTER_IMPLICIT, abi.PREC_FP64, abs_tol=1e-14)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-10
