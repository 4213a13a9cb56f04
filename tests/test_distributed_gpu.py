"""The ordinate-partitioned solver's GPU backend (libidcsweep on this rank's GPU) on one rank: it gives
the same solution as the single-context GMRES."""
import threading

import numpy as np
import pytest
import torch

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


def _threaded_allreduce(n_ranks):
    """An in-process stand-in for an all-reduce over ranks that are threads of this process: each rank
    leaves its partial sums, all wait, and each adds them in rank order (bitwise the same sums everywhere),
    as an NCCL all-reduce gives every rank the same result.  The exchange is on the host: no kernel waits
    for another."""
    import torch
    from idcsweep.distributed import _DeviceVector

    barrier = threading.Barrier(n_ranks, timeout=120)
    slots = [None] * n_ranks

    def make(rank):
        def fn(ptr, n):
            t = torch.as_tensor(_DeviceVector(ptr, n), device="cuda:0")
            slots[rank] = t.cpu()
            barrier.wait()
            total = slots[0].clone()
            for r in range(1, n_ranks):
                total += slots[r]
            barrier.wait()
            t.copy_(total.to("cuda:0"))
            torch.cuda.synchronize()
            return 0
        return fn

    return make


@pytest.mark.parametrize("dsa", [False, True])
def test_device_gmres_over_two_ranks_with_allreduce_hook(dsa):
    """Two ranks (threads, each a context with half of every quadrant's ordinates) run the library's GMRES
    (+ DSA) with the all-reduce hook: both take the same iterations and get bitwise the same moments, and each
    rank's psi is the full-quadrature solve's psi at its ordinates."""
    P = lognormal(20, 2, 8, seed=31)
    make = _threaded_allreduce(2)
    backends = [GpuBackend(P, partition_ordinates(P.quad, 2, r), device=0) for r in range(2)]
    results, errors = [None, None], []
    try:
        if dsa:
            for be in backends:
                be.ctx.set_preconditioner(abi.PRECOND_DSA, 20)

        def run(r):
            try:
                results[r] = DistributedTransport(backends[r]).gmres_device(
                    backends[r].local_source(P.source), P.dt, abs_tol=1e-11, restart=30, max_its=2000,
                    hook=make(r))
            except Exception as e:   # reported below
                errors.append(e)

        threads = [threading.Thread(target=run, args=(r,)) for r in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    finally:
        for be in backends:
            be.close()
    assert not errors, errors
    with abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by) as ctx:
        ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
        ctx.set_sigma(P.sigma_t, P.sigma_s)
        if dsa:
            ctx.set_preconditioner(abi.PRECOND_DSA, 20)
        want = P.source.copy()
        want_its, _ = ctx.gmres_solve(want, P.dt, abs_tol=1e-11, restart=30, max_its=2000)
    (phi0, psi0, its0, res0), (phi1, psi1, its1, res1) = results
    assert its0 == its1 and res0 == res1 and res0 <= 1e-11
    assert abs(its0 - want_its) <= 1
    assert torch.equal(phi0, phi1)
    for r, psi in enumerate((psi0, psi1)):
        idx = partition_ordinates(P.quad, 2, r)
        assert rel_err(psi.cpu().numpy()[1:-1, 1:-1], want[1:-1, 1:-1][:, :, idx]) < 1e-8
