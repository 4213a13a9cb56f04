"""FP64 CPU discrete adjoint of the transport problem on the oracle restatement (test infrastructure).

The forward problem is the reference's: (L - S P) psi = q with L^{-1} the sweep (SweepOperator::Apply)
and S, P the scattering broadcast and the moment reduction (TransportOperator::Smv / Pmv), solved by
the reference's source iteration (SISolver::Solve).  For J = c . P psi the adjoint is
(L - S P)^T lam = P^T c; with mu = c + S^T lam it reads mu = c + S^T L^{-T} P^T mu, solved here by the
same fixed-point iteration with the oracle's transposed sweep.  Gradients per cell:
dJ/dsigma_t = -sum lam psi, dJ/dsigma_s = sum_k Lam_k phi_k / (4 pi), dJ/dq_k = Lam_k / (4 pi),
Lam = sum_q lam_q, for the isotropic source moments q (angular source q / (4 pi))."""
import numpy as np


def forward(R, OP, source, dt, tol=1e-14, max_its=20000):
    psi, its, err = R.source_iteration(OP, source, dt, abs_tol=tol, max_its=max_its)
    return psi.reshape(OP.psi_shape())


def functional(R, OP, psi, c):
    return float((c * R.pmv(OP, psi)).sum())


def adjoint(R, OP, c, dt, tol=1e-15, max_its=20000):
    """Returns (lam, Lam) on the halo layouts (interior cells meaningful)."""
    nq = OP.nq
    w = np.asarray(OP.w)
    ss = np.asarray(OP.sigma_s).reshape(OP.nx + 2, OP.ny + 2)
    mu = c.copy()
    for _ in range(max_its):
        src = np.zeros(OP.psi_shape())
        src[1:-1, 1:-1] = w[None, None, :, None, None] * mu[1:-1, 1:-1, None, :, :]
        lam = R.sweep_adjoint(OP, src, dt).reshape(OP.psi_shape())
        Lam = np.zeros(OP.phi_shape())
        Lam[1:-1, 1:-1] = lam[1:-1, 1:-1].sum(axis=2)
        mu_new = c.copy()
        mu_new[1:-1, 1:-1] += ss[1:-1, 1:-1, None, None] / (4.0 * np.pi) * Lam[1:-1, 1:-1]
        done = np.abs(mu_new - mu).max() <= tol * max(np.abs(mu_new).max(), 1e-300)
        mu = mu_new
        if done:
            break
    src = np.zeros(OP.psi_shape())
    src[1:-1, 1:-1] = w[None, None, :, None, None] * mu[1:-1, 1:-1, None, :, :]
    lam = R.sweep_adjoint(OP, src, dt).reshape(OP.psi_shape())
    Lam = np.zeros(OP.phi_shape())
    Lam[1:-1, 1:-1] = lam[1:-1, 1:-1].sum(axis=2)
    return lam, Lam


def gradient(R, OP, psi, c, dt):
    lam, Lam = adjoint(R, OP, c, dt)
    phi = R.pmv(OP, psi).reshape(OP.phi_shape())
    nx, ny = OP.nx, OP.ny
    g_t = np.zeros((nx + 2, ny + 2))
    g_s = np.zeros((nx + 2, ny + 2))
    g_q = np.zeros(OP.phi_shape())
    g_t[1:-1, 1:-1] = -(lam[1:-1, 1:-1] * psi[1:-1, 1:-1]).sum(axis=(2, 3, 4))
    g_s[1:-1, 1:-1] = (Lam[1:-1, 1:-1] * phi[1:-1, 1:-1]).sum(axis=(2, 3)) / (4.0 * np.pi)
    g_q[1:-1, 1:-1] = Lam[1:-1, 1:-1] / (4.0 * np.pi)
    return g_t, g_s, g_q
