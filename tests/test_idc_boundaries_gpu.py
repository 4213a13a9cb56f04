"""IDC time stepping with implicit scattering on reflecting edges and on a periodic grid against the reference's
own IDCIntegrator (update form, Gauss-Lobatto nodes, SISolver substeps) built and run with
Global::reflecting_boundaries / Global::periodic set: every substep solve reaches the boundary condition's fixed
point (the boundary-unknown GMRES), the initial stage is reflected (or its halos synchronised) at every step as
Step_Nonhybrid does, and the residuals read the reflections or periodic images the solves leave."""
import os

import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import random_problem
from oracle.bindings import REFERENCE_SO, Reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REFERENCE_SO), reason="oracle/_ref/libidcref.so not built")]


@pytest.fixture(scope="module")
def ref():
    return Reference(REFERENCE_SO)


def _periodic_images(a):
    a = a.copy()
    a[0, 1:-1] = a[-2, 1:-1]
    a[-1, 1:-1] = a[1, 1:-1]
    a[1:-1, 0] = a[1:-1, -2]
    a[1:-1, -1] = a[1:-1, 1]
    return a


@pytest.mark.parametrize("mode", [abi.EDGE_X_MIN, abi.EDGE_X_MIN | abi.EDGE_Y_MIN, 15, "periodic"])
def test_implicit_idc_with_boundaries_matches_reference_integrator(ref, mode):
    P = random_problem(7, 8, 1, 4, seed=61, dt=0.05, inflow=False, sigma_range=(0.5, 4.0))
    rng = np.random.default_rng(2)
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = 0.05 + 0.01 * rng.standard_normal(psi0[1:-1, 1:-1].shape)
    periodic = mode == "periodic"
    if periodic:
        psi0 = _periodic_images(psi0)
    reflect = 0 if periodic else mode
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-14, max_its=100000, reflect=reflect, periodic=periodic) as h:
        want = h.idc_steps(psi0, P.source, P.dt, 2, 3, 2, si_abs_tol=1e-14)
    with abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by) as ctx:
        ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
        ctx.set_sigma(P.sigma_t, P.sigma_s)
        if periodic:
            ctx.set_periodic(True)
        else:
            ctx.set_reflecting(reflect)
        psi = psi0.copy()
        ctx.idc_integrate(psi, P.source, P.dt, 2, 3, 2, abi.SCATTER_IMPLICIT, abi.PREC_FP64, abs_tol=1e-14)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-10
    # the boundary condition matters: the vacuum integrator gives another result
    with ref.open(to_oracle(P), P.dt, abs_tol=1e-14, max_its=100000) as h:
        vac = h.idc_steps(psi0, P.source, P.dt, 2, 3, 2, si_abs_tol=1e-14)
    assert rel_err(vac[1:-1, 1:-1], want[1:-1, 1:-1]) > 1e-4
