"""IDC time stepping restated on the oracle operators (test infrastructure).

Non-hybrid update form of IDCIntegrator::Step_Nonhybrid (time_integrators/RKDG/idc.cpp:846-955) with
ComputeResiduals / ComputeSource (:1657-1740) on Gauss-Lobatto nodes (SetNodes, :2305-2381):
implicit substeps solved by the restatement's source iteration (the reference's SISolver), or the IMEX
variant (one sweep per substep, scattering lagged to the previous node and corrected)."""
import numpy as np
from numpy.polynomial import legendre as L


def lobatto(M):
    """Gauss-Lobatto nodes on [0, 1] and W[i, j] = int_{t_{i-1}}^{t_i} l_j (i >= 1), int_0^1 l_j (i = 0)."""
    c = np.zeros(M)
    c[-1] = 1.0
    inner = np.sort(L.legroots(L.legder(c))) if M > 2 else np.array([])
    t = np.concatenate([[0.0], 0.5 * (inner + 1.0), [1.0]])
    W = np.zeros((M, M))
    for j in range(M):
        y = np.zeros(M)
        y[j] = 1.0
        coef = np.polynomial.polynomial.polyfit(t, y, M - 1)
        integ = np.polynomial.polynomial.polyint(coef)
        F = lambda x: np.polynomial.polynomial.polyval(x, integ)
        W[0, j] = F(1.0) - F(0.0)
        for i in range(1, M):
            W[i, j] = F(t[i]) - F(t[i - 1])
    return t, W


def _interior(P, a):
    out = np.zeros_like(a)
    out[1:-1, 1:-1] = a[1:-1, 1:-1]
    return out


def idc_steps(R, OP, psi0, Q, dt, steps, M=4, K=3, scattering="explicit", si_tol=1e-14, zero_ghosts=False):
    """psi after `steps` IDC steps.  psi0, Q: halo psi arrays (Q's ghost cells = inflow).

    zero_ghosts=True zeroes the ghost cells of every step's result, as IDCIntegrator::Step_Nonhybrid does
    (`initial_condition.ZeroDensity( OpDomain::Boundary )`, idc.cpp:949-950), so that the residual of the
    next step's first stage sees vacuum inflow.  With inflow data that makes the reference's multi-step
    result first order in time; the default keeps the inflow values (the GPU integrator's behaviour).  On
    vacuum boundaries both give the same result."""
    t, W = lobatto(M)
    shp = OP.psi_shape()
    psi = psi0.reshape(shp).copy()
    Q = Q.reshape(shp)
    pmv = lambda x: R.pmv(OP, x).reshape(OP.phi_shape())
    lmv = lambda x: R.lmv(OP, x).reshape(shp)
    smv = lambda phi, x, alpha=1.0: R.smv(OP, phi, x, alpha=alpha, beta=1.0).reshape(shp)

    def src_with_ghosts(interior_sum):
        s = Q.copy()
        s[1:-1, 1:-1] += interior_sum[1:-1, 1:-1]
        return s

    def solve(src, hdt):
        if scattering == "implicit":
            out, _, _ = R.source_iteration(OP, src, hdt, abs_tol=si_tol, max_its=100000)
            return out.reshape(shp)
        raise AssertionError

    for _ in range(steps):
        stages = [psi] + [Q.copy() for _ in range(M - 1)]
        phis = [pmv(psi)] + [None] * (M - 1)
        for n in range(1, M):   # prediction
            h = t[n] - t[n - 1]
            src = src_with_ghosts(stages[n - 1] / (h * dt))
            if scattering == "implicit":
                stages[n] = solve(src, h * dt)
            else:
                stages[n] = R.sweep(OP, smv(phis[n - 1], src), h * dt).reshape(shp)
            phis[n] = pmv(stages[n])
        for _p in range(K):
            res = [smv(phis[l], lmv(stages[l]), alpha=-1.0) for l in range(M)]
            phis_old = [f.copy() for f in phis]
            for n in range(1, M):
                h = t[n] - t[n - 1]
                acc = stages[n - 1] / (h * dt)
                for l in range(M):
                    acc = acc + ((1.0 if n == l else 0.0) - W[n, l] / h) * res[l]
                src = src_with_ghosts(acc)
                if scattering == "implicit":
                    stages[n] = solve(src, h * dt)
                else:
                    phi_s = phis[n - 1] - phis_old[n - 1] + phis_old[n]
                    stages[n] = R.sweep(OP, smv(phi_s, src), h * dt).reshape(shp)
                phis[n] = pmv(stages[n])
        psi = stages[M - 1]
        if zero_ghosts:
            psi = psi.copy()
            psi[0], psi[-1], psi[:, 0], psi[:, -1] = 0.0, 0.0, 0.0, 0.0
    return psi
