"""Reflecting boundaries (idc_set_reflecting) against the reference's own sweep with reflecting edges: the
reference compiled from its sources (oracle/_ref) with Global::reflecting_boundaries set as its deck keys
reflect_x_min .. reflect_y_max set it, so SweepPatternUniCartWavefront sweeps the quadrants in sequence (order
3, 2, 1, 0) and OrdinateFlux::ReflectBoundaries refills the ghost cells after each.  A sweep, source
iteration and the Peierls GMRES must reproduce the reference's sweep and source-iteration fixed point."""
import os

import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import lognormal, random_problem
from oracle.bindings import REFERENCE_SO, Reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REFERENCE_SO), reason="oracle/_ref/libidcref.so not built")]


@pytest.fixture(scope="module")
def ref():
    return Reference(REFERENCE_SO)


def _ctx(P, edges):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    ctx.set_reflecting(edges)
    return ctx


def _phi(P, psi):
    return np.tensordot(psi[1:-1, 1:-1], P.w, axes=([2], [0]))


@pytest.mark.parametrize("edges", [abi.EDGE_X_MIN, abi.EDGE_X_MAX, abi.EDGE_Y_MIN, abi.EDGE_Y_MAX,
                                   abi.EDGE_X_MIN | abi.EDGE_Y_MIN, abi.EDGE_X_MAX | abi.EDGE_Y_MAX, 15])
@pytest.mark.parametrize("p,sn,prec,tol", [(0, 4, abi.PREC_FP64, 1e-12), (1, 8, abi.PREC_FP64, 1e-12),
                                           (2, 4, abi.PREC_FP64, 1e-12), (1, 8, abi.PREC_FP32, 1e-5)])
def test_reflecting_sweep_matches_reference(ref, edges, p, sn, prec, tol):
    """One sweep (inflow data on the other edges, and on the reflecting ones before their first reflection,
    as in the reference's in-place array)."""
    P = random_problem(9, 7, p, sn, seed=80 + 3 * p + edges, dt=0.4)
    with ref.open(to_oracle(P), P.dt, reflect=edges) as h:
        want = h.sweep(P.source, P.dt)
    with _ctx(P, edges) as ctx:
        psi = P.source.copy()
        phi = np.zeros(P.phi_shape())
        ctx.sweep(psi, P.dt, phi, prec)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < tol
    assert rel_err(psi, want) < tol   # ghost cells too: inflow kept, reflections as the reference leaves them
    assert rel_err(phi[1:-1, 1:-1], _phi(P, want)) < tol
    vac = P.source.copy()   # the reflections matter: a vacuum sweep differs
    with ref.open(to_oracle(P), P.dt) as h:
        vac = h.sweep(P.source, P.dt)
    assert rel_err(vac[1:-1, 1:-1], want[1:-1, 1:-1]) > 1e-6


@pytest.mark.parametrize("edges", [abi.EDGE_X_MIN, abi.EDGE_X_MIN | abi.EDGE_Y_MIN, abi.EDGE_X_MAX | abi.EDGE_Y_MIN,
                                   abi.EDGE_Y_MAX, 15])
def test_reflecting_source_iteration_and_gmres_match_reference(ref, edges):
    """Source iteration (the reference's SISolver::Solve with reflecting edges: psi from zero, the reflecting
    edges' ghost cells carried from one sweep to the next) reaches the reference's fixed point, and so does the
    Peierls GMRES (+ DSA) whose unknowns include the reflecting edges' ghost values, for edge sets whose
    quadrant order reads a reflection partner before it is swept (x-max, y-max) as well as for those it does
    not (x-min, y-min)."""
    P = lognormal(16, 1, 8, seed=5, c_range=(0.3, 0.8), dt=0.5)
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-13, max_its=5000, reflect=edges) as h:
        want = h.source_iteration(P.source, P.dt)
    phi_want = _phi(P, want)
    with _ctx(P, edges) as ctx:
        psi = P.source.copy()
        its, err = ctx.source_iteration(psi, P.dt, abs_tol=1e-13, max_its=5000)
        assert err <= 1e-13
        assert rel_err(_phi(P, psi), phi_want) < 1e-11
        assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-11
        assert rel_err(psi, want) < 1e-11   # and the ghost cells the reference's psi returns with
        for dsa in (False, True):
            if dsa:
                ctx.set_preconditioner(abi.PRECOND_DSA, 20)
            psi = P.source.copy()
            its, res = ctx.gmres_solve(psi, P.dt, abs_tol=1e-12, restart=30, max_its=3000)
            assert res <= 1e-12
            assert rel_err(_phi(P, psi), phi_want) < 1e-10
            assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-10
        psi = P.source.copy()   # FP32 sweeps: the FP32 operator's accuracy
        ctx.gmres_solve(psi, P.dt, abs_tol=1e-6, restart=30, max_its=3000, precision=abi.PREC_FP32)
        assert rel_err(_phi(P, psi), phi_want) < 1e-4


def test_reflecting_rejections():
    P = random_problem(6, 5, 1, 4, seed=3)
    with _ctx(P, abi.EDGE_X_MIN) as ctx:
        psi = P.source.copy()
        with pytest.raises(abi.IdcError) as e:   # the lane kernel has no cell-refined mode
            ctx.sweep(psi, P.dt, None, abi.PREC_FP32_REFINED)
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        with pytest.raises(abi.IdcError) as e:
            ctx.gmres_solve(P.source.copy(), P.dt, precision=abi.PREC_FP32_IR)
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        with pytest.raises(abi.IdcError) as e:
            ctx.idc_integrate(P.source.copy(), P.source, 0.1, 1, 3, 1, abi.SCATTER_EXPLICIT)   # implicit: supported
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        with pytest.raises(abi.IdcError) as e:
            with abi.Batch() as b:
                b.add(ctx)
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED
    # an ordinate set without reflection partners
    xi, eta, w, q = P.xi.copy(), P.eta.copy(), P.w.copy(), P.quad.copy()
    xi[0] *= 0.999
    with abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by) as ctx:
        ctx.set_ordinates(xi, eta, w, q)
        with pytest.raises(abi.IdcError) as e:
            ctx.set_reflecting(abi.EDGE_X_MIN)
        assert e.value.code == abi.IDC_ERR_ARG
