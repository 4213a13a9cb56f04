"""Implicit solvers on the GPU against the reference's own source-iteration fixed point.

GMRES (Peierls form) has no reference run here (PETSc is absent), so its parity is on the converged
solution: the reference's SISolver result stored in the golden fixtures (SI to 1e-12) and the CPU
restatement's SI at tight tolerance."""
import glob
import os

import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import lattice, lognormal, random_problem

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def context_for(P):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    return ctx


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_REFINED, abi.PREC_FP32_IR])
def test_gmres_reaches_reference_si_fixed_point(path, prec):
    z = np.load(path)
    P = lambda: None
    with abi.SweepContext(int(z["nx"]), int(z["ny"]), int(z["p"]), float(z["ax"]), float(z["bx"]), float(z["ay"]),
                          float(z["by"])) as ctx:
        ctx.set_ordinates(z["xi"], z["eta"], z["w"], z["quad"])
        ctx.set_sigma(z["sigma_t"], z["sigma_s"])
        psi = z["source"].copy()
        its, res = ctx.gmres_solve(psi, float(z["dt"]), abs_tol=1e-13, restart=30, max_its=500, precision=prec)
        assert res <= 1e-13
        assert rel_err(psi, z["si_psi"]) < 1e-10


@pytest.mark.parametrize("dsa", [False, True])
def test_fp32_krylov_with_fp64_refinement_meets_the_fp64_tolerance(dsa):
    """IDC_PREC_FP32_IR: FP32 sweeps in the Krylov iterations, FP64 residuals and solution: the same
    solution as the FP64 solve to the tolerance, although an FP32 sweep alone is accurate to ~1e-7 only."""
    P = lognormal(64, 2, 8, seed=4, c_range=(0.5, 0.99))
    out = {}
    with context_for(P) as ctx:
        if dsa:
            ctx.set_preconditioner(abi.PRECOND_DSA, 20)
        for prec in (abi.PREC_FP64, abi.PREC_FP32_IR):
            psi = P.source.copy()
            its, res = ctx.gmres_solve(psi, P.dt, abs_tol=1e-10, restart=30, max_its=2000, precision=prec)
            assert res <= 1e-10
            out[prec] = psi
        one = P.source.copy()
        ctx.sweep(one, P.dt, None, abi.PREC_FP32)
        two = P.source.copy()
        ctx.sweep(two, P.dt, None, abi.PREC_FP64)
    assert rel_err(out[abi.PREC_FP32_IR], out[abi.PREC_FP64]) < 1e-9
    assert 1e-9 < rel_err(one, two) < 1e-5   # a single FP32 sweep is FP32-accurate


def test_gmres_matches_restatement_si_on_lattice(restatement):
    P = lattice(24, 1, 8, dt=0.01)
    o = to_oracle(P)
    ref, _, _ = restatement.source_iteration(o, P.source, P.dt, abs_tol=1e-13, max_its=2000)
    with context_for(P) as ctx:
        psi = P.source.copy()
        its, res = ctx.gmres_solve(psi, P.dt, abs_tol=1e-12, restart=30, max_its=500)
        si = P.source.copy()
        its_si, err_si = ctx.source_iteration(si, P.dt, abs_tol=1e-13, max_its=2000)
    assert rel_err(psi, ref) < 1e-9
    assert rel_err(si, ref) < 1e-11
    assert its < its_si


def test_gmres_not_converged_is_reported():
    P = lognormal(32, 1, 8, seed=3, c_range=(0.99, 0.999))
    with context_for(P) as ctx:
        psi = P.source.copy()
        with pytest.raises(abi.IdcError) as e:
            ctx.gmres_solve(psi, np.inf, abs_tol=1e-14, restart=5, max_its=3)
        assert e.value.code == abi.IDC_ERR_NOT_CONVERGED


def test_sweep_out_matches_in_place():
    P = random_problem(20, 17, 2, 8, seed=9, dt=0.3)
    with context_for(P) as ctx:
        a = P.source.copy()
        pa = np.zeros(P.phi_shape())
        ctx.sweep(a, P.dt, pa)
        b = np.full_like(P.source, 7.0)
        pb = np.zeros(P.phi_shape())
        ctx.sweep_out(P.source, b, P.dt, pb)
    interior = (slice(1, -1), slice(1, -1))
    assert np.array_equal(a[interior], b[interior])
    assert np.all(b[0] == 7.0) and np.all(b[:, -1] == 7.0)    # result ghosts untouched
    assert np.array_equal(pa, pb)                               # fixed-order moment reduction


@pytest.mark.parametrize("path", GOLDEN[:4], ids=[os.path.basename(p) for p in GOLDEN[:4]])
def test_gmres_dsa_reaches_reference_si_fixed_point(path):
    z = np.load(path)
    with abi.SweepContext(int(z["nx"]), int(z["ny"]), int(z["p"]), float(z["ax"]), float(z["bx"]), float(z["ay"]),
                          float(z["by"])) as ctx:
        ctx.set_ordinates(z["xi"], z["eta"], z["w"], z["quad"])
        ctx.set_sigma(z["sigma_t"], z["sigma_s"])
        ctx.set_preconditioner(abi.PRECOND_DSA, 30)
        psi = z["source"].copy()
        its, res = ctx.gmres_solve(psi, float(z["dt"]), abs_tol=1e-13, restart=30, max_its=500)
        assert res <= 1e-13
        assert rel_err(psi, z["si_psi"]) < 1e-10


@pytest.mark.parametrize("p,sn,c", [(1, 8, (0.95, 0.999)), (2, 8, (0.5, 0.999))])
def test_dsa_reduces_gmres_iterations(p, sn, c):
    """Scattering-dominated log-normal media: the DSA-preconditioned flexible GMRES converges to the same
    solution in fewer iterations."""
    P = lognormal(64, p, sn, seed=2, c_range=c)
    out = {}
    for kind in (abi.PRECOND_NONE, abi.PRECOND_DSA):
        with context_for(P) as ctx:
            ctx.set_preconditioner(kind, 30)
            psi = P.source.copy()
            its, res = ctx.gmres_solve(psi, P.dt, abs_tol=1e-10, restart=30, max_its=3000)
            out[kind] = (its, psi)
    assert out[abi.PRECOND_DSA][0] < out[abi.PRECOND_NONE][0]
    assert rel_err(out[abi.PRECOND_DSA][1], out[abi.PRECOND_NONE][1]) < 1e-8


def test_set_preconditioner_rejects_bad_arguments():
    P = lognormal(8, 1, 4, seed=1)
    with context_for(P) as ctx:
        with pytest.raises(abi.IdcError):
            ctx.set_preconditioner(7, 30)
        with pytest.raises(abi.IdcError):
            ctx.set_preconditioner(abi.PRECOND_DSA, 0)


@pytest.mark.parametrize("dsa", [False, True])
def test_solves_are_bitwise_reproducible(dsa):
    """Every reduction of the solvers (dot products, Krylov norms, the SI distance, the DSA inner products)
    adds its partial sums in a fixed order, so repeating a solve gives bitwise the same result."""
    P = lognormal(40, 1, 8, seed=12, c_range=(0.5, 0.99))
    with context_for(P) as ctx:
        if dsa:
            ctx.set_preconditioner(abi.PRECOND_DSA, 20)
        outs = []
        for _ in range(2):
            a = P.source.copy()
            its_g, res_g = ctx.gmres_solve(a, P.dt, abs_tol=1e-10)
            b = P.source.copy()
            its_s, err_s = ctx.source_iteration(b, P.dt, abs_tol=1e-8, max_its=2000)
            outs.append((a, b, its_g, res_g, its_s, err_s))
    (a0, b0, *r0), (a1, b1, *r1) = outs
    assert np.array_equal(a0, a1) and np.array_equal(b0, b1)
    assert r0 == r1
