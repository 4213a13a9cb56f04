"""The adjoint of IDC's correction sweeps (idc_adjoint_idc).

* The transposed transport operator, L^T (idc_lmv_transpose), is pinned by <L^T a, b> = <a, L b> against the
  forward Lmv, itself pinned to the reference's TransportOperator::Lmv.
* The gradients of a detector response J = c . phi(psi^N) after N implicit-scattering IDC steps (every
  substep a GMRES solve; the forward integrator is pinned to the reference's IDCIntegrator) with respect to
  the per-cell sigma_t, sigma_s, the isotropic source moments and the initial angular flux, against central
  differences of the GPU's own IDC time stepping on seeded cells: h = 1e-4 |value| for the cross sections,
  a tenth of the largest value for the source and the initial flux (J is linear in both, so the difference is
  exact up to rounding, and a large step keeps the solves' rounding small against it).
* Recomputing each step's stages from checkpoints reproduces the forward pass exactly, so the checkpoint
  interval does not change a bit of the gradients.
"""
import numpy as np
import pytest
import torch

from idcsweep import abi
from idcsweep.problems import detector_window, lognormal, random_problem

pytestmark = pytest.mark.gpu


def _ctx(P):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    return ctx


@pytest.mark.parametrize("p,sn", [(0, 4), (1, 8), (2, 4)])
def test_lmv_transpose_is_the_adjoint_of_lmv(p, sn):
    P = random_problem(9, 7, p, sn, seed=70 + p)
    rng = np.random.default_rng(5 + p)
    a, b = np.zeros(P.psi_shape()), np.zeros(P.psi_shape())
    a[1:-1, 1:-1] = rng.standard_normal(a[1:-1, 1:-1].shape)
    b[1:-1, 1:-1] = rng.standard_normal(b[1:-1, 1:-1].shape)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    la, lb = torch.zeros_like(da), torch.zeros_like(db)
    with _ctx(P) as ctx:
        ctx.lmv(1.0, 0.0, db.data_ptr(), lb.data_ptr(), loc=abi.LOC_DEVICE)
        ctx.lmv_transpose(1.0, 0.0, da.data_ptr(), la.data_ptr())
    lhs = float((la[1:-1, 1:-1] * db[1:-1, 1:-1]).sum())
    rhs = float((da[1:-1, 1:-1] * lb[1:-1, 1:-1]).sum())
    scale = float((la.abs()[1:-1, 1:-1] * db.abs()[1:-1, 1:-1]).sum())
    assert abs(lhs - rhs) <= 1e-13 * scale
    assert float(la[0].abs().sum() + la[-1].abs().sum() + la[:, 0].abs().sum() + la[:, -1].abs().sum()) == 0.0


def _J(ctx, P, c, sigma_t, sigma_s, source, psi0, dt, steps, M, K, tol):
    ctx.set_sigma(sigma_t, sigma_s)
    psi = psi0.copy()
    ctx.idc_integrate(psi, source, dt, steps, M, K, abi.SCATTER_IMPLICIT, abi.PREC_FP64, abs_tol=tol, max_its=3000)
    phi = np.zeros(P.phi_shape())
    ctx.pmv(1.0, 0.0, psi, phi)
    return float((c * phi).sum())


@pytest.mark.parametrize("M,K,cells", [(3, 2, 6), (4, 3, 4)])
def test_idc_adjoint_matches_central_differences(M, K, cells):
    P = lognormal(10, 1, 4, seed=31, median=2.0, log_sd=0.7, c_fixed=0.8, source="gaussian")
    c = detector_window(P, cells=3)
    rng = np.random.default_rng(8)
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = rng.uniform(0.0, 1.0, psi0[1:-1, 1:-1].shape)
    dt, steps, tol = 0.1, 3, 1e-13
    gt, gs = np.zeros(P.sigma_t.shape), np.zeros(P.sigma_s.shape)
    gq, gp = np.zeros(P.phi_shape()), np.zeros(P.psi_shape())
    with _ctx(P) as ctx:
        J, solves = ctx.adjoint_idc(psi0, P.source, c, dt, steps, M, K, checkpoint_every=2, dsigma_t=gt, dsigma_s=gs,
                                    dsource=gq, dpsi0=gp, abs_tol=tol)
        # forward 3 steps, the first segment's second input again, each step's stages again, and the adjoint
        # solves of 3 steps: 10 x (K + 1)(M - 1)
        assert solves == 10 * (K + 1) * (M - 1)
        J0 = _J(ctx, P, c, P.sigma_t, P.sigma_s, P.source, psi0, dt, steps, M, K, tol)
        assert abs(J - J0) <= 1e-12 * abs(J0)
        picks = rng.choice(P.nx * P.ny, size=cells, replace=False)
        qs = float(np.abs(P.source).max())
        ps = float(np.abs(psi0).max())
        got, fd = {"sigma_t": [], "sigma_s": [], "source": [], "psi0": []}, {"sigma_t": [], "sigma_s": [],
                                                                              "source": [], "psi0": []}
        for cell in picks:
            i, j = 1 + cell // P.ny, 1 + cell % P.ny
            idx = i * (P.ny + 2) + j
            for name, arr, grad in (("sigma_t", P.sigma_t, gt), ("sigma_s", P.sigma_s, gs)):
                h = 1e-4 * abs(arr[idx])
                up, dn = arr.copy(), arr.copy()
                up[idx] += h
                dn[idx] -= h
                st_u, ss_u = (up, P.sigma_s) if name == "sigma_t" else (P.sigma_t, up)
                st_d, ss_d = (dn, P.sigma_s) if name == "sigma_t" else (P.sigma_t, dn)
                f = (_J(ctx, P, c, st_u, ss_u, P.source, psi0, dt, steps, M, K, tol) -
                     _J(ctx, P, c, st_d, ss_d, P.source, psi0, dt, steps, M, K, tol)) / (2 * h)
                got[name].append(grad[idx])
                fd[name].append(f)
            k = int(rng.integers(0, (P.p + 1) ** 2))
            d, e = divmod(k, P.p + 1)
            h = 0.1 * qs   # the isotropic source moment k of the cell: moment / (4 pi) on every ordinate
            up, dn = P.source.copy(), P.source.copy()
            up[i, j, :, d, e] += h / (4 * np.pi)
            dn[i, j, :, d, e] -= h / (4 * np.pi)
            f = (_J(ctx, P, c, P.sigma_t, P.sigma_s, up, psi0, dt, steps, M, K, tol) -
                 _J(ctx, P, c, P.sigma_t, P.sigma_s, dn, psi0, dt, steps, M, K, tol)) / (2 * h)
            got["source"].append(gq[i, j, d, e])
            fd["source"].append(f)
            q = int(rng.integers(0, P.nq))
            h = 0.1 * ps
            up, dn = psi0.copy(), psi0.copy()
            up[i, j, q, d, e] += h
            dn[i, j, q, d, e] -= h
            f = (_J(ctx, P, c, P.sigma_t, P.sigma_s, P.source, up, dt, steps, M, K, tol) -
                 _J(ctx, P, c, P.sigma_t, P.sigma_s, P.source, dn, dt, steps, M, K, tol)) / (2 * h)
            got["psi0"].append(gp[i, j, q, d, e])
            fd["psi0"].append(f)
        ctx.set_sigma(P.sigma_t, P.sigma_s)
    for name in got:
        a, f = np.asarray(got[name]), np.asarray(fd[name])
        scale = max(np.abs(f).max(), 1e-300)
        assert np.abs(a - f).max() <= 1e-6 * scale, (name, np.abs(a - f).max() / scale)
        big = np.abs(f) > 1e-3 * scale   # entries above the round-off floor: each within 1e-5 relative
        assert np.all(np.abs(a[big] - f[big]) <= 1e-5 * np.abs(f[big])), name


def test_idc_adjoint_checkpoint_interval_is_bitwise_neutral():
    P = lognormal(12, 1, 4, seed=9, median=2.0, log_sd=0.7, c_fixed=0.9, source="gaussian")
    c = detector_window(P, cells=4)
    psi0 = np.zeros(P.psi_shape())
    outs = []
    with _ctx(P) as ctx:
        ctx.set_preconditioner(abi.PRECOND_DSA, 20)
        for ck in (1, 2, 0):
            gt, gq, gp = np.zeros(P.sigma_t.shape), np.zeros(P.phi_shape()), np.zeros(P.psi_shape())
            J, _ = ctx.adjoint_idc(psi0, P.source, c, 0.1, 4, 3, 2, checkpoint_every=ck, dsigma_t=gt, dsource=gq,
                                   dpsi0=gp)
            outs.append((J, gt, gq, gp))
    for J, gt, gq, gp in outs[1:]:
        assert J == outs[0][0]
        assert np.array_equal(gt, outs[0][1]) and np.array_equal(gq, outs[0][2]) and np.array_equal(gp, outs[0][3])
