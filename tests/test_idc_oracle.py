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
