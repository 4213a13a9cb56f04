"""The restated IDC (tests/idc_ref.py) without a GPU: Lobatto weights integrate polynomials exactly, and
the restated IMEX and implicit IDC reach fourth order in time on the oracle's operators."""
import numpy as np
import pytest

from conftest import to_oracle
from idc_ref import idc_steps, lobatto
from idcsweep.problems import random_problem


@pytest.mark.parametrize("M", [2, 3, 4, 5])
def test_lobatto_weights_integrate_polynomials(M):
    t, W = lobatto(M)
    for deg in range(M):
        f = t ** deg
        assert abs(W[0] @ f - 1.0 / (deg + 1)) < 1e-14
        for i in range(1, M):
            assert abs(W[i] @ f - (t[i] ** (deg + 1) - t[i - 1] ** (deg + 1)) / (deg + 1)) < 1e-14


@pytest.mark.parametrize("scattering", ["explicit", "implicit"])
def test_restated_idc_is_fourth_order(restatement, scattering):
    P = random_problem(4, 4, 1, 4, seed=9, inflow=True, sigma_range=(0.5, 2.0))
    OP = to_oracle(P)
    T = 0.4
    psi0 = P.source.copy()   # ghost cells: the same inflow as the source (no jump in time at t = 0)
    psi0[1:-1, 1:-1] = 0.1
    sols = {m: idc_steps(restatement, OP, psi0, P.source, T / m, m, M=4, K=3, scattering=scattering,
                         si_tol=1e-15)[1:-1, 1:-1] for m in (2, 4, 8, 64)}
    e = [np.abs(sols[m] - sols[64]).max() for m in (2, 4, 8)]
    orders = [np.log2(e[k] / e[k + 1]) for k in range(2)]
    assert orders[-1] > 3.5 and min(orders) > 3.0, (e, orders)


# The restated IDC against the reference's own IDCIntegrator (oracle/_ref: IDCIntegrator::Create + Step,
# non-hybrid update form, Gauss-Lobatto nodes, SISolver substeps), both with substeps converged to 1e-14.
@pytest.mark.parametrize("case", [
    dict(kind="lattice", n=8, p=1, sn=4, M=4, K=3, steps=3),
    dict(kind="lattice", n=10, p=0, sn=8, M=3, K=2, steps=2),
    dict(kind="random", n=6, p=2, sn=8, M=4, K=3, steps=2, inflow=False),
    dict(kind="random", n=5, p=1, sn=4, M=5, K=4, steps=2, inflow=False),
    dict(kind="random", n=5, p=1, sn=4, M=2, K=1, steps=3, inflow=False),
])
def test_restated_idc_matches_reference_integrator(restatement, reference, case):
    from idcsweep.problems import lattice
    if case["kind"] == "lattice":
        P = lattice(case["n"], case["p"], case["sn"], dt=0.01)
    else:
        P = random_problem(case["n"], case["n"] + 1, case["p"], case["sn"], seed=31, dt=0.05,
                           inflow=case["inflow"], sigma_range=(0.5, 4.0))
    OP = to_oracle(P)
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = 0.05
    want = idc_steps(restatement, OP, psi0, P.source, P.dt, case["steps"], M=case["M"], K=case["K"],
                     scattering="implicit", si_tol=1e-14)
    with reference.open(OP, P.dt, abs_tol=1e-14, max_its=100000) as h:
        got = h.idc_steps(psi0, P.source, P.dt, case["steps"], case["M"], case["K"], si_abs_tol=1e-14)
    scale = np.abs(got[1:-1, 1:-1]).max()
    assert np.abs(got[1:-1, 1:-1] - want[1:-1, 1:-1]).max() / scale < 1e-12


def test_restated_idc_with_inflow_matches_reference_integrator(restatement, reference):
    """Inflow on the ghost cells: the reference zeroes the ghost cells of each step's result (so a later
    step's first-stage residual sees vacuum inflow); restated with zero_ghosts=True it agrees, and the
    first step agrees either way."""
    P = random_problem(6, 5, 1, 8, seed=3, dt=0.05, inflow=True, sigma_range=(0.5, 4.0))
    OP = to_oracle(P)
    psi0 = np.zeros(P.psi_shape())
    with reference.open(OP, P.dt, abs_tol=1e-14, max_its=100000) as h:
        one = h.idc_steps(psi0, P.source, P.dt, 1, 4, 3, si_abs_tol=1e-14)
        three = h.idc_steps(psi0, P.source, P.dt, 3, 4, 3, si_abs_tol=1e-14)
    for steps, got in ((1, one), (3, three)):
        want = idc_steps(restatement, OP, psi0, P.source, P.dt, steps, M=4, K=3, scattering="implicit",
                         si_tol=1e-14, zero_ghosts=True)
        assert np.abs(got - want).max() / np.abs(got).max() < 1e-12
    keep = idc_steps(restatement, OP, psi0, P.source, P.dt, 1, M=4, K=3, scattering="implicit", si_tol=1e-14)
    assert np.abs(one[1:-1, 1:-1] - keep[1:-1, 1:-1]).max() / np.abs(one).max() < 1e-12
