"""The oracle's transposed sweep and the CPU adjoint gradient, pinned without a GPU.

The transposed sweep is checked as the transpose of the (reference-pinned) forward sweep on interior
cells, and the adjoint gradient against central finite differences of the reference's own source
iteration on the restatement."""
import numpy as np
import pytest

from adjoint_ref import forward, functional, gradient
from conftest import to_oracle
from idcsweep.problems import detector_window, lognormal, random_problem


def _interior_random(OP, rng):
    a = np.zeros(OP.psi_shape())
    a[1:-1, 1:-1] = rng.uniform(-1.0, 1.0, a[1:-1, 1:-1].shape)
    return a


@pytest.mark.parametrize("p", [0, 1, 2])
@pytest.mark.parametrize("dt", [np.inf, 0.05])
def test_oracle_transposed_sweep_is_the_transpose(restatement, p, dt):
    P = random_problem(7, 5, p, 4, seed=11 + p, dt=dt, inflow=False)
    OP = to_oracle(P)
    rng = np.random.default_rng(3)
    a, b = _interior_random(OP, rng), _interior_random(OP, rng)
    lhs = (restatement.sweep_adjoint(OP, a, dt).reshape(OP.psi_shape())[1:-1, 1:-1] * b[1:-1, 1:-1]).sum()
    rhs = (a[1:-1, 1:-1] * restatement.sweep(OP, b, dt).reshape(OP.psi_shape())[1:-1, 1:-1]).sum()
    assert abs(lhs - rhs) <= 1e-12 * abs(rhs)


def test_oracle_adjoint_gradient_matches_central_differences(restatement):
    P = lognormal(8, 1, 4, seed=5, median=2.0, log_sd=0.7, c_fixed=0.9, source="gaussian")
    OP = to_oracle(P)
    c = detector_window(P, cells=3)
    src = P.source.reshape(OP.psi_shape()).copy()
    psi = forward(restatement, OP, src, P.dt)
    g_t, g_s, g_q = gradient(restatement, OP, psi, c, P.dt)
    st0, ss0 = OP.sigma_t.copy(), OP.sigma_s.copy()
    rng = np.random.default_rng(0)
    for _ in range(3):
        i, j = (int(v) for v in rng.integers(1, 9, 2))
        k = i * (P.ny + 2) + j
        # sigma_t (sigma_s fixed)
        h = 1e-4 * st0[k]
        vals = []
        for sgn in (1, -1):
            OP.sigma_t = st0.copy()
            OP.sigma_t[k] += sgn * h
            vals.append(functional(restatement, OP, forward(restatement, OP, src, P.dt), c))
        OP.sigma_t = st0.copy()
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g_t[i, j]) <= 1e-6 * abs(g_t).max()
        # sigma_s
        h = 1e-4 * ss0[k]
        vals = []
        for sgn in (1, -1):
            OP.sigma_s = ss0.copy()
            OP.sigma_s[k] += sgn * h
            vals.append(functional(restatement, OP, forward(restatement, OP, src, P.dt), c))
        OP.sigma_s = ss0.copy()
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g_s[i, j]) <= 1e-6 * abs(g_s).max()
        # isotropic source moment (0, 0): the angular source changes by h / (4 pi) on every ordinate
        h = 1e-3
        vals = []
        for sgn in (1, -1):
            s2 = src.copy()
            s2[i, j, :, 0, 0] += sgn * h / (4 * np.pi)
            vals.append(functional(restatement, OP, forward(restatement, OP, s2, P.dt), c))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g_q[i, j, 0, 0]) <= 1e-6 * abs(g_q).max()


def test_oracle_transient_adjoint_matches_central_differences(restatement):
    """Implicit-Euler steps on the restatement: the backward adjoint gradients against central differences
    of the forward time stepping (sigma_t, sigma_s, source moment, initial flux)."""
    from adjoint_ref import forward_transient, transient_gradient
    P = lognormal(6, 1, 4, seed=8, median=2.0, log_sd=0.7, c_fixed=0.8, source="gaussian")
    OP = to_oracle(P)
    c = detector_window(P, cells=2)
    Q = P.source.reshape(OP.psi_shape()).copy()
    rng = np.random.default_rng(4)
    psi0 = np.zeros(OP.psi_shape())
    psi0[1:-1, 1:-1] = rng.uniform(0.0, 1.0, psi0[1:-1, 1:-1].shape)
    dt, steps = 0.2, 3
    J, g_t, g_s, g_q, g_p = transient_gradient(restatement, OP, psi0, Q, c, dt, steps)

    def J_of(psi0_, Q_):
        return functional(restatement, OP, forward_transient(restatement, OP, psi0_, Q_, dt, steps)[-1], c)

    assert abs(J_of(psi0, Q) - J) <= 1e-13 * abs(J)
    st0, ss0 = OP.sigma_t.copy(), OP.sigma_s.copy()
    for i, j in ((2, 3), (5, 1), (4, 6)):
        k = i * (P.ny + 2) + j
        for arr, g in ((st0, g_t), (ss0, g_s)):
            h = 1e-4 * arr[k]
            vals = []
            for sgn in (1, -1):
                pert = arr.copy()
                pert[k] += sgn * h
                if arr is st0:
                    OP.sigma_t = pert
                else:
                    OP.sigma_s = pert
                vals.append(J_of(psi0, Q))
            OP.sigma_t, OP.sigma_s = st0.copy(), ss0.copy()
            assert abs((vals[0] - vals[1]) / (2 * h) - g[i, j]) <= 1e-6 * abs(g).max()
        h = 1e-3
        vals = []
        for sgn in (1, -1):
            Q2 = Q.copy()
            Q2[i, j, :, 0, 0] += sgn * h / (4 * np.pi)
            vals.append(J_of(psi0, Q2))
        assert abs((vals[0] - vals[1]) / (2 * h) - g_q[i, j, 0, 0]) <= 1e-6 * abs(g_q).max()
        vals = []
        for sgn in (1, -1):
            p2 = psi0.copy()
            p2[i, j, 3, 1, 0] += sgn * h
            vals.append(J_of(p2, Q))
        assert abs((vals[0] - vals[1]) / (2 * h) - g_p[i, j, 3, 1, 0]) <= 1e-6 * abs(g_p).max()
