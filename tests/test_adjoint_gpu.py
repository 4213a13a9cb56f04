"""Discrete adjoint on the GPU: the transposed sweep against the oracle's, the transpose identity at full
size, and the adjoint gradients against the CPU FP64 adjoint (tests/adjoint_ref.py) and central finite
differences of the GPU forward solve."""
import numpy as np
import pytest

from adjoint_ref import forward, gradient
from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import detector_window, lognormal, random_problem

pytestmark = pytest.mark.gpu


def context_for(P, tiling=(0, 0)):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    ctx.set_tiling(*tiling)
    return ctx


@pytest.mark.parametrize("p", [0, 1, 2])
@pytest.mark.parametrize("tiling", [(0, 0), (4, 8), (1, 3)])
@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-12), (abi.PREC_FP32_REFINED, 1e-8)])
def test_transposed_sweep_matches_oracle(restatement, p, tiling, prec, tol):
    P = random_problem(11, 9, p, 8, seed=40 + p, dt=0.3)
    OP = to_oracle(P)
    want = restatement.sweep_adjoint(OP, P.source, P.dt).reshape(P.psi_shape())
    with context_for(P, tiling) as ctx:
        got = np.zeros(P.psi_shape())
        mom = np.zeros(P.phi_shape())
        ctx.sweep_adjoint(P.source, got, P.dt, mom, precision=prec)
    assert rel_err(got[1:-1, 1:-1], want[1:-1, 1:-1]) < tol
    assert rel_err(mom[1:-1, 1:-1], want[1:-1, 1:-1].sum(axis=2)) < tol
    assert np.all(mom[0] == 0) and np.all(mom[:, -1] == 0)


@pytest.mark.parametrize("n,p,sn", [(96, 2, 8), (128, 1, 12)])
def test_transpose_identity_on_the_gpu(n, p, sn):
    """<L^-T a, b> == <a, L^-1 b> on interior cells (zero inflow), sweeps on the GPU."""
    P = lognormal(n, p, sn, seed=3)
    rng = np.random.default_rng(1)
    a = np.zeros(P.psi_shape())
    b = np.zeros(P.psi_shape())
    a[1:-1, 1:-1] = rng.uniform(-1, 1, a[1:-1, 1:-1].shape)
    b[1:-1, 1:-1] = rng.uniform(-1, 1, b[1:-1, 1:-1].shape)
    with context_for(P) as ctx:
        la = np.zeros_like(a)
        lb = np.zeros_like(b)
        ctx.sweep_adjoint(a, la, P.dt)
        ctx.sweep_out(b, lb, P.dt)
    lhs = (la[1:-1, 1:-1] * b[1:-1, 1:-1]).sum()
    rhs = (a[1:-1, 1:-1] * lb[1:-1, 1:-1]).sum()
    assert abs(lhs - rhs) <= 1e-11 * abs(rhs)


def _adjoint_problem(n=12, p=1, sn=4, seed=5):
    P = lognormal(n, p, sn, seed=seed, median=2.0, log_sd=0.7, c_fixed=0.9, source="gaussian")
    return P, detector_window(P, cells=4)


@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-10), (abi.PREC_FP32_REFINED, 1e-8)])
def test_adjoint_gradient_matches_cpu_adjoint(restatement, prec, tol):
    P, c = _adjoint_problem()
    OP = to_oracle(P)
    psi = forward(restatement, OP, P.source.reshape(OP.psi_shape()).copy(), P.dt)
    g_t, g_s, g_q = gradient(restatement, OP, psi, c, P.dt)
    with context_for(P) as ctx:
        d_t = np.zeros((P.nx + 2) * (P.ny + 2))
        d_s = np.zeros_like(d_t)
        d_q = np.zeros(P.phi_shape())
        its, res = ctx.adjoint_grad(psi, c, d_t, d_s, d_q, dt=P.dt, abs_tol=1e-14, precision=prec)
    assert res <= 1e-14
    assert rel_err(d_t.reshape(g_t.shape), g_t) < tol
    assert rel_err(d_s.reshape(g_s.shape), g_s) < tol
    assert rel_err(d_q, g_q) < tol


def test_adjoint_gradient_with_transposed_dsa():
    """The transposed DSA right preconditioner leaves the gradients as they are and cuts the adjoint
    GMRES iterations (scattering ratio 0.9 on an optically thick problem)."""
    from idcsweep.problems import detector_window, lognormal
    P = lognormal(48, 1, 8, seed=3, median=2.0, log_sd=0.7, c_fixed=0.95, source="gaussian")
    c = detector_window(P, cells=8)
    out = {}
    with context_for(P) as ctx:
        psi = P.source.copy()
        ctx.gmres_solve(psi, P.dt, abs_tol=1e-13, restart=30, max_its=3000)
        for kind in (abi.PRECOND_NONE, abi.PRECOND_DSA):
            ctx.set_preconditioner(kind, 30)
            d = [np.zeros((P.nx + 2) * (P.ny + 2)), np.zeros((P.nx + 2) * (P.ny + 2)), np.zeros(P.phi_shape())]
            its, res = ctx.adjoint_grad(psi, c, *d, dt=P.dt, abs_tol=1e-13)
            assert res <= 1e-13
            out[kind] = (its, d)
    (i0, d0), (i1, d1) = out[abi.PRECOND_NONE], out[abi.PRECOND_DSA]
    assert i1 < i0
    for a_, b_ in zip(d0, d1):
        assert rel_err(b_, a_) < 1e-9


def test_adjoint_gradient_matches_finite_differences_of_gpu_solves():
    P, c = _adjoint_problem(n=16)
    src0 = P.source.copy()

    def J(sigma_t, sigma_s, src):
        with abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by) as ctx:
            ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
            ctx.set_sigma(sigma_t, sigma_s)
            psi = src.copy()
            ctx.gmres_solve(psi, P.dt, abs_tol=1e-14, restart=30, max_its=2000)
            phi = np.zeros(P.phi_shape())
            ctx.pmv(1.0, 0.0, psi, phi)
        return float((c * phi).sum()), psi

    _, psi = J(P.sigma_t, P.sigma_s, src0)
    with context_for(P) as ctx:
        d_t = np.zeros((P.nx + 2) * (P.ny + 2))
        d_s = np.zeros_like(d_t)
        d_q = np.zeros(P.phi_shape())
        ctx.adjoint_grad(psi, c, d_t, d_s, d_q, dt=P.dt, abs_tol=1e-14)
    rng = np.random.default_rng(7)
    for _ in range(4):
        i, j = (int(v) for v in rng.integers(1, P.nx + 1, 2))
        k = i * (P.ny + 2) + j
        h = 1e-4 * P.sigma_t[k]
        st_p, st_m = P.sigma_t.copy(), P.sigma_t.copy()
        st_p[k] += h
        st_m[k] -= h
        fd = (J(st_p, P.sigma_s, src0)[0] - J(st_m, P.sigma_s, src0)[0]) / (2 * h)
        assert abs(fd - d_t[k]) <= 1e-6 * np.abs(d_t).max()
        h = 1e-4 * P.sigma_s[k]
        ss_p, ss_m = P.sigma_s.copy(), P.sigma_s.copy()
        ss_p[k] += h
        ss_m[k] -= h
        fd = (J(P.sigma_t, ss_p, src0)[0] - J(P.sigma_t, ss_m, src0)[0]) / (2 * h)
        assert abs(fd - d_s[k]) <= 1e-6 * np.abs(d_s).max()
        h = 1e-3
        s_p, s_m = src0.copy(), src0.copy()
        s_p[i, j, :, 0, 0] += h / (4 * np.pi)
        s_m[i, j, :, 0, 0] -= h / (4 * np.pi)
        fd = (J(P.sigma_t, P.sigma_s, s_p)[0] - J(P.sigma_t, P.sigma_s, s_m)[0]) / (2 * h)
        assert abs(fd - d_q[i, j, 0, 0]) <= 1e-6 * np.abs(d_q).max()


def test_adjoint_rejects_unrefined_fp32():
    P, c = _adjoint_problem(n=8)
    with context_for(P) as ctx:
        with pytest.raises(abi.IdcError) as e:
            ctx.sweep_adjoint(P.source, np.zeros(P.psi_shape()), P.dt, precision=abi.PREC_FP32)
        assert e.value.code == abi.IDC_ERR_UNSUPPORTED


@pytest.mark.parametrize("p,sn", [(1, 4), (2, 8)])
@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-9), (abi.PREC_FP32_REFINED, 1e-8)])
def test_transient_adjoint_matches_cpu_adjoint(restatement, p, sn, prec, tol):
    """Implicit-Euler steps: the GPU's checkpointed backward adjoint (idc_adjoint_transient) against the CPU
    FP64 transient adjoint on the restatement (tests/adjoint_ref.py), J included."""
    from adjoint_ref import transient_gradient
    P = lognormal(10, p, sn, seed=21 + p, median=2.0, log_sd=0.7, c_fixed=0.8, source="gaussian")
    OP = to_oracle(P)
    c = detector_window(P, cells=3)
    rng = np.random.default_rng(6)
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = rng.uniform(0.0, 1.0, psi0[1:-1, 1:-1].shape)
    dt, steps = 0.2, 4
    J_ref, gt_ref, gs_ref, gq_ref, gp_ref = transient_gradient(restatement, OP, psi0, P.source.copy(), c, dt, steps)
    gt, gs = np.zeros(P.sigma_t.shape), np.zeros(P.sigma_s.shape)
    gq, gp = np.zeros(P.phi_shape()), np.zeros(P.psi_shape())
    with context_for(P) as ctx:
        J, solves = ctx.adjoint_transient(psi0, P.source, c, dt, steps, checkpoint_every=2, dsigma_t=gt,
                                          dsigma_s=gs, dsource=gq, dpsi0=gp, abs_tol=1e-13, precision=prec)
    assert solves == 3 * steps   # forward, recomputation (two segments of two), adjoint
    assert abs(J - J_ref) <= tol * abs(J_ref)
    gt, gs = gt.reshape(P.nx + 2, P.ny + 2), gs.reshape(P.nx + 2, P.ny + 2)
    for got, want in ((gt, gt_ref), (gs, gs_ref), (gq, gq_ref), (gp, gp_ref)):
        assert rel_err(got[1:-1, 1:-1], want[1:-1, 1:-1]) < tol


def test_transient_adjoint_checkpoint_interval_is_bitwise_neutral():
    """Recomputing the states from checkpoints reproduces the forward pass exactly, so every checkpoint
    interval gives bitwise the same gradients."""
    P = lognormal(24, 1, 8, seed=9, median=2.0, log_sd=0.7, c_fixed=0.9, source="gaussian")
    c = detector_window(P, cells=4)
    psi0 = np.zeros(P.psi_shape())
    outs = []
    with context_for(P) as ctx:
        ctx.set_preconditioner(abi.PRECOND_DSA, 20)
        for K in (1, 3, 7, 0):
            gt, gq = np.zeros(P.sigma_t.shape), np.zeros(P.phi_shape())
            J, _ = ctx.adjoint_transient(psi0, P.source, c, 0.1, 7, checkpoint_every=K, dsigma_t=gt, dsource=gq)
            outs.append((J, gt, gq))
    for J, gt, gq in outs[1:]:
        assert J == outs[0][0]
        assert np.array_equal(gt, outs[0][1]) and np.array_equal(gq, outs[0][2])
