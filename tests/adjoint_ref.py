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


# ---- implicit-Euler time stepping: (1/dt + L - S P) psi^{n+1} = psi^n / dt + Q, J = c . P psi^N ----------

def step_source(psi, Q, dt):
    """psi / dt + Q on interior cells, Q's ghost cells (the inflow) elsewhere."""
    src = Q.copy()
    src[1:-1, 1:-1] += psi[1:-1, 1:-1] / dt
    return src


def forward_transient(R, OP, psi0, Q, dt, steps):
    """All states psi^0 .. psi^steps, each step solved by the reference's source iteration."""
    states = [psi0]
    for _ in range(steps):
        states.append(forward(R, OP, step_source(states[-1], Q, dt), dt))
    return states


def adjoint_psi(R, OP, b, dt, tol=1e-15, max_its=20000):
    """(L' - S P)^T lam = b for a psi-sized b (interior cells): nu = S^T lam is the fixed point of
    nu = S^T L'^{-T} (b + P^T nu), then lam = L'^{-T} (b + P^T nu).  Returns (lam, Lam = sum_q lam_q)."""
    w = np.asarray(OP.w)
    ss = np.asarray(OP.sigma_s).reshape(OP.nx + 2, OP.ny + 2)
    nu = np.zeros(OP.phi_shape())

    def solve(nu):
        src = np.zeros(OP.psi_shape())
        src[1:-1, 1:-1] = b[1:-1, 1:-1] + w[None, None, :, None, None] * nu[1:-1, 1:-1, None, :, :]
        lam = R.sweep_adjoint(OP, src, dt).reshape(OP.psi_shape())
        Lam = np.zeros(OP.phi_shape())
        Lam[1:-1, 1:-1] = lam[1:-1, 1:-1].sum(axis=2)
        return lam, Lam

    for _ in range(max_its):
        lam, Lam = solve(nu)
        nu_new = np.zeros(OP.phi_shape())
        nu_new[1:-1, 1:-1] = ss[1:-1, 1:-1, None, None] / (4.0 * np.pi) * Lam[1:-1, 1:-1]
        done = np.abs(nu_new - nu).max() <= tol * max(np.abs(nu_new).max(), 1e-300)
        nu = nu_new
        if done:
            break
    return solve(nu)


def transient_gradient(R, OP, psi0, Q, c, dt, steps):
    """Gradients of J = c . P psi^steps with respect to sigma_t, sigma_s, the isotropic source moments and
    psi^0 (interior cells), by the backward adjoint steps A^T lam^N = P^T c, A^T lam^n = lam^{n+1} / dt."""
    states = forward_transient(R, OP, psi0, Q, dt, steps)
    w = np.asarray(OP.w)
    nx, ny = OP.nx, OP.ny
    g_t = np.zeros((nx + 2, ny + 2))
    g_s = np.zeros((nx + 2, ny + 2))
    g_q = np.zeros(OP.phi_shape())
    b = np.zeros(OP.psi_shape())
    b[1:-1, 1:-1] = w[None, None, :, None, None] * c[1:-1, 1:-1, None, :, :]
    lam = None
    for n in range(steps, 0, -1):
        if lam is not None:
            b = np.zeros(OP.psi_shape())
            b[1:-1, 1:-1] = lam[1:-1, 1:-1] / dt
        lam, Lam = adjoint_psi(R, OP, b, dt)
        psi = states[n]
        phi = R.pmv(OP, psi).reshape(OP.phi_shape())
        g_t[1:-1, 1:-1] -= (lam[1:-1, 1:-1] * psi[1:-1, 1:-1]).sum(axis=(2, 3, 4))
        g_s[1:-1, 1:-1] += (Lam[1:-1, 1:-1] * phi[1:-1, 1:-1]).sum(axis=(2, 3)) / (4.0 * np.pi)
        g_q[1:-1, 1:-1] += Lam[1:-1, 1:-1] / (4.0 * np.pi)
    g_p = np.zeros(OP.psi_shape())
    g_p[1:-1, 1:-1] = lam[1:-1, 1:-1] / dt
    return functional(R, OP, states[-1], c), g_t, g_s, g_q, g_p
