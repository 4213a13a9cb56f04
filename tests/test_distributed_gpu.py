"""The ordinate-partitioned solver's GPU backend (libidcsweep on this rank's GPU) on one rank: it gives
the same solution as the single-context GMRES."""
import numpy as np
import pytest

from conftest import rel_err
from idcsweep import abi
from idcsweep.distributed import DistributedTransport, GpuBackend, partition_ordinates
from idcsweep.problems import lognormal

pytestmark = pytest.mark.gpu


def test_gpu_backend_one_rank_matches_context_gmres():
    P = lognormal(24, 1, 8, seed=4)
    idx = partition_ordinates(P.quad, 1, 0)
    be = GpuBackend(P, idx, device=0)
    try:
        dt = DistributedTransport(be)
        phi, psi, its, res = dt.gmres(be.local_source(P.source), P.dt, abs_tol=1e-12, restart=30)
        phi2, psi2, its2, err2 = dt.source_iteration(be.local_source(P.source), P.dt, abs_tol=1e-12, max_its=3000)
    finally:
        be.close()
    with abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by) as ctx:
        ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
        ctx.set_sigma(P.sigma_t, P.sigma_s)
        want = P.source.copy()
        ctx.gmres_solve(want, P.dt, abs_tol=1e-12, restart=30, max_its=3000)
    assert res <= 1e-12
    assert rel_err(psi.cpu().numpy()[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-9
    assert rel_err(psi2.cpu().numpy()[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-9
