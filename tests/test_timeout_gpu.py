"""Failure detection on the GPU without a fault: every device-side wait of the sweep kernels is bounded.

idc_set_spin_limit shortens the bound to a few polls, so the waits of a multi-row-block sweep (the item
below polling for the traces of the item above, the warps of a thread block waiting on one another) give
up long before their producers arrive.  The kernel then records the failure in the device error word,
every warp leaves, and the call returns IDC_ERR_TIMEOUT; nothing hangs and the context stays usable.
After the default bound is restored, the next calls on the same context must give the same results as a
context that never failed: the trace buffers that the abandoned sweep left half written are re-armed.
"""
import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import random_problem

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def _ctx(P):
    c = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    c.set_ordinates(P.xi, P.eta, P.w, P.quad)
    c.set_sigma(P.sigma_t, P.sigma_s)
    return c


def _expect_timeout(fn):
    with pytest.raises(abi.IdcError) as e:
        fn()
    assert e.value.code == abi.IDC_ERR_TIMEOUT, e.value


def test_sweep_wait_gives_up_and_context_recovers(restatement):
    # 96 rows: several row blocks, so the items below poll for the traces of the items above
    P = random_problem(64, 96, 2, 8, seed=77, dt=0.1)
    ref = restatement.sweep(to_oracle(P), P.source, P.dt)
    with _ctx(P) as c:
        c.set_spin_limit(2)
        for _ in range(2):   # twice: a failed sweep must not leave state that breaks the next failure either
            psi = P.source.copy()
            _expect_timeout(lambda: c.sweep(psi, P.dt, None, abi.PREC_FP64))
        c.set_spin_limit(0)   # the default bound
        for prec, tol in ((abi.PREC_FP64, TOL64), (abi.PREC_FP32_REFINED, 1e-8)):
            psi = P.source.copy()
            phi = np.zeros(P.phi_shape())
            c.sweep(psi, P.dt, phi, prec)
            assert rel_err(psi, ref) < tol
            assert rel_err(phi, restatement.pmv(to_oracle(P), ref)) < tol


def test_gmres_dsa_timeout_then_bitwise_recovery():
    """A GMRES + DSA solve whose sweeps and DSA grid barriers give up, then the same solve with the default
    bound, bitwise equal to the solve on a context that never failed."""
    P = random_problem(48, 72, 1, 8, seed=78)
    with _ctx(P) as c:
        c.set_preconditioner(abi.PRECOND_DSA, 10)
        src = P.source.copy()
        its_ref, _ = c.gmres_solve(src, P.dt, abs_tol=1e-10, restart=20, max_its=500)
    with _ctx(P) as c:
        c.set_preconditioner(abi.PRECOND_DSA, 10)
        c.set_spin_limit(2)
        bad = P.source.copy()
        _expect_timeout(lambda: c.gmres_solve(bad, P.dt, abs_tol=1e-10, restart=20, max_its=500))
        c.set_spin_limit(0)
        psi = P.source.copy()
        its, _ = c.gmres_solve(psi, P.dt, abs_tol=1e-10, restart=20, max_its=500)
    assert its == its_ref
    assert np.array_equal(psi, src)
