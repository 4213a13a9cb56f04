"""Parity at the benchmark configurations' full sizes.

* The reference's own CPU-runnable case (64x64 lattice on [0,7]^2, Q1, S8, one implicit-Euler step of
  dt = 0.01 from zero flux, source iteration to 1e-10): the GPU's idc_source_iteration against the
  reference's SISolver::Solve, whose result is the committed fixture tests/golden/config/
  config0_lattice64_q1_s8.npz (tests/golden/make_golden.py).
* The adjoint configuration (128x128, Q1, S8, log-normal sigma_t with median 2 and log-sd 0.7, c = 0.9,
  Gaussian source at the left third, detector = the scalar flux over a 16x16-cell window at the right
  third): the GPU adjoint gradients with respect to sigma_t, sigma_s and the source against central finite
  differences of GPU forward solves on 64 seeded cells, step h = 1e-4 |value| (for the source, to which J
  is linear, 1e-4 of the largest source value).
"""
import os

import numpy as np
import pytest

from conftest import rel_err
from idcsweep import abi
from idcsweep.problems import detector_window, lattice, lognormal

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GOLDEN0 = os.path.join(os.path.dirname(__file__), "golden", "config", "config0_lattice64_q1_s8.npz")


def _ctx(P):
    c = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    c.set_ordinates(P.xi, P.eta, P.w, P.quad)
    c.set_sigma(P.sigma_t, P.sigma_s)
    return c


@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-12), (abi.PREC_FP32_REFINED, 1e-8)])
def test_config0_source_iteration_matches_reference(prec, tol):
    z = np.load(GOLDEN0)
    P = lattice(64, 1, 8, dt=0.01)
    # the fixture's inputs are the ones this build generates
    assert np.array_equal(P.sigma_t, z["sigma_t"]) and np.array_equal(P.sigma_s, z["sigma_s"])
    assert P.source.sum() == z["source_sum"] and np.abs(P.source).sum() == z["source_abs_sum"]
    with _ctx(P) as c:
        psi = P.source.copy()
        its, change = c.source_iteration(psi, P.dt, abs_tol=float(z["si_tol"]), max_its=5000, precision=prec)
        phi = np.zeros(P.phi_shape())
        c.pmv(1.0, 0.0, psi, phi)
    assert change <= float(z["si_tol"])
    assert rel_err(phi, z["phi"]) < tol
    cells = z["cells"]
    assert rel_err(psi[cells[:, 0], cells[:, 1]], z["psi_cells"]) < tol


def test_config3_adjoint_gradients_match_central_differences():
    P = lognormal(128, 1, 8, seed=0, median=2.0, log_sd=0.7, c_fixed=0.9, source="gaussian")
    c_host = detector_window(P, cells=16)
    dev = "cuda"
    c_det = torch.from_numpy(c_host).to(dev)
    src0 = torch.from_numpy(P.source).to(dev)
    psi = torch.empty_like(src0)
    phi = torch.zeros(P.phi_shape(), dtype=torch.float64, device=dev)
    tol = 1e-13

    with _ctx(P) as ctx:
        ctx.set_preconditioner(abi.PRECOND_DSA, 30)

        def J(sigma_t, sigma_s, src):
            ctx.set_sigma(sigma_t, sigma_s)
            psi.copy_(src)
            ctx.gmres_solve(psi.data_ptr(), P.dt, abs_tol=tol, restart=30, max_its=3000, loc=abi.LOC_DEVICE)
            ctx.pmv(1.0, 0.0, psi.data_ptr(), phi.data_ptr(), loc=abi.LOC_DEVICE)
            return float((c_det * phi).sum().item())

        J(P.sigma_t, P.sigma_s, src0)   # psi of the unperturbed problem
        g_t = torch.zeros((P.nx + 2) * (P.ny + 2), dtype=torch.float64, device=dev)
        g_s = torch.zeros_like(g_t)
        g_q = torch.zeros(P.phi_shape(), dtype=torch.float64, device=dev)
        its, res = ctx.adjoint_grad(psi.data_ptr(), c_det.data_ptr(), g_t.data_ptr(), g_s.data_ptr(),
                                    g_q.data_ptr(), dt=P.dt, abs_tol=tol, loc=abi.LOC_DEVICE)
        assert res <= tol
        g_t, g_s, g_q = g_t.cpu().numpy(), g_s.cpu().numpy(), g_q.cpu().numpy()

        q_scale = float(np.abs(P.source[..., 0, 0]).max()) * 4 * np.pi
        rng = np.random.default_rng(2024)
        cells = rng.choice(P.nx * P.ny, size=64, replace=False)
        fd = {"t": [], "s": [], "q": []}
        adj = {"t": [], "s": [], "q": []}
        for cell in cells:
            i, j = 1 + int(cell // P.ny), 1 + int(cell % P.ny)
            k = i * (P.ny + 2) + j
            for name, arr in (("t", P.sigma_t), ("s", P.sigma_s)):
                h = 1e-4 * abs(arr[k])
                plus, minus = arr.copy(), arr.copy()
                plus[k] += h
                minus[k] -= h
                if name == "t":
                    d = (J(plus, P.sigma_s, src0) - J(minus, P.sigma_s, src0)) / (2 * h)
                    adj["t"].append(g_t[k])
                else:
                    d = (J(P.sigma_t, plus, src0) - J(P.sigma_t, minus, src0)) / (2 * h)
                    adj["s"].append(g_s[k])
                fd[name].append(d)
            # the isotropic source moment q_00 of the cell (angular source q_00 / (4 pi) on every ordinate).  J
            # is linear in it, so central differences are exact up to round-off for any step; the step is
            # 1e-4 of the largest source value (the Gaussian source is ~0 in most sampled cells, where
            # 1e-4 |value| would leave only round-off)
            h = 1e-4 * q_scale
            s_p, s_m = src0.clone(), src0.clone()
            s_p[i, j, :, 0, 0] += h / (4 * np.pi)
            s_m[i, j, :, 0, 0] -= h / (4 * np.pi)
            fd["q"].append((J(P.sigma_t, P.sigma_s, s_p) - J(P.sigma_t, P.sigma_s, s_m)) / (2 * h))
            adj["q"].append(g_q[i, j, 0, 0])
    for name, full in (("t", g_t), ("s", g_s), ("q", g_q)):
        a, f = np.array(adj[name]), np.array(fd[name])
        scale = np.abs(full).max()
        assert np.abs(a - f).max() <= 1e-6 * scale, (name, np.abs(a - f).max() / scale)
        big = np.abs(a) > 1e-3 * scale   # entries well above the round-off floor: each within 1e-6 relative
        assert np.all(np.abs(a[big] - f[big]) <= 1e-6 * np.abs(a[big])), name
