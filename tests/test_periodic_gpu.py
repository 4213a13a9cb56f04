"""Periodic boundaries (idc_set_periodic) against the reference compiled from its sources (oracle/_ref) with
Global::periodic set, as its deck key `periodic` sets it: a sweep reads the ghost cells as given; the reference's
SISolver::Solve synchronises the halos from the opposite edges at the start of every iteration after the first
and copies the source into the interior only, so its fixed point is the periodic problem's solution.  Source
iteration and the Peierls GMRES (+ DSA) must reach it; Lmv takes the opposite edges' cells as its upwind
neighbours across an edge."""
import os

import numpy as np
import pytest
import torch

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import lognormal, random_problem, smooth_sigma
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
    ctx.set_periodic(True)
    return ctx


def _phi(P, psi):
    return np.tensordot(psi[1:-1, 1:-1], P.w, axes=([2], [0]))


def _sync(a):
    """The halos of a psi-shaped array from the opposite interior edges (corners untouched)."""
    a = a.copy()
    a[0, 1:-1] = a[-2, 1:-1]
    a[-1, 1:-1] = a[1, 1:-1]
    a[1:-1, 0] = a[1:-1, -2]
    a[1:-1, -1] = a[1:-1, 1]
    return a


@pytest.mark.parametrize("p,sn,dt", [(0, 4, 0.5), (1, 8, np.inf), (2, 4, 0.3)])
def test_sweep_reads_ghosts_as_given(ref, p, sn, dt):
    P = random_problem(9, 7, p, sn, seed=90 + p, dt=dt)
    with ref.open(to_oracle(P), P.dt, periodic=True) as h:
        want = h.sweep(P.source, P.dt)
    with _ctx(P) as ctx:
        psi = P.source.copy()
        ctx.sweep(psi, P.dt)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-12


@pytest.mark.parametrize("kind,p,sn", [("lognormal", 1, 8), ("lognormal", 2, 4), ("smooth", 1, 4)])
def test_source_iteration_and_gmres_match_reference(ref, kind, p, sn):
    """The reference's SISolver::Solve on a periodic grid (with piecewise-constant and high-order cross sections);
    our source iteration reaches its fixed point, and GMRES with and without DSA, whose unknowns include the
    edges' incoming ghost values, reaches the same one."""
    if kind == "smooth":
        P = smooth_sigma(12, p, sn, seed=21, dt=0.5, c_range=(0.4, 0.8))
    else:
        P = lognormal(14, p, sn, seed=8 + p, c_range=(0.3, 0.8), dt=0.5)
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-13, max_its=5000, periodic=True,
                  sigma_degree=P.sigma_degree) as h:
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
    # the periodic coupling matters: the vacuum problem's fixed point is another
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-13, max_its=5000, sigma_degree=P.sigma_degree) as h:
        vac = h.source_iteration(P.source, P.dt)
    assert rel_err(_phi(P, vac), phi_want) > 1e-4


def test_lmv_wraps_across_edges(ref):
    P = random_problem(8, 6, 1, 4, seed=5)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(P.psi_shape())
    with ref.open(to_oracle(P), P.dt, periodic=True) as h:
        want = h.lmv(_sync(x), None, 0.8, 0.0)
    with _ctx(P) as ctx:
        y = np.zeros(P.psi_shape())
        ctx.lmv(0.8, 0.0, x, y)   # x's own ghost values are not used
    assert rel_err(y[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-13


def test_periodic_rejections():
    P = random_problem(6, 5, 1, 4, seed=3)
    with _ctx(P) as ctx:
        for call in (lambda: ctx.set_reflecting(abi.EDGE_X_MIN),
                     lambda: ctx.gmres_solve(P.source.copy(), P.dt, precision=abi.PREC_FP32_IR),
                     lambda: ctx.idc_integrate(P.source.copy(), P.source, 0.1, 1, 3, 1)):
            with pytest.raises(abi.IdcError) as e:
                call()
            assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        x = torch.zeros(P.psi_shape(), dtype=torch.float64, device="cuda")
        with pytest.raises(abi.IdcError) as e:
            ctx.lmv_transpose(1.0, 0.0, x.data_ptr(), x.data_ptr())
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        with pytest.raises(abi.IdcError) as e:
            with abi.Batch() as b:
                b.add(ctx)
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED
        ctx.set_periodic(False)   # off again: a plain context
        ctx.set_reflecting(abi.EDGE_X_MIN)
        with pytest.raises(abi.IdcError) as e:
            ctx.set_periodic(True)
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED
