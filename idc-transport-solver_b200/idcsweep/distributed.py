"""Ordinate-partitioned transport solves across GPUs: one process per GPU, torch.distributed plumbing
(NCCL on GPUs, gloo on CPU).

A sweep needs no data from other ordinates, so each rank sweeps a slice of every quadrant's ordinates
(contiguous, balanced) and forms partial moments phi_g = sum_{q in slice} w_q psi_q; one all-reduce (sum)
of phi (nx+2)(ny+2)N doubles -- 4.7 MB at 256^2, Q2 -- completes the moments.  That all-reduce is the path's
only exchange: the scattering source of the next sweep is rebuilt locally from the replicated phi, and
the Krylov vectors (moment-sized) are replicated, so the Arnoldi process runs redundantly and identically
on every rank (all-reduce results are identical on all ranks).  The reference's multi-rank parallelism
is spatial KBA over MPI (SweepPatternUniCartKBA*); the ordinate split replaces it on a single node.

A backend does the local sweeps: GpuBackend (libidcsweep on this rank's GPU) in production; tests
inject a CPU backend to run the same control flow under gloo without a GPU.
"""
from __future__ import annotations

import math

import numpy as np
import torch
import torch.distributed as dist


def partition_ordinates(quad, world: int, rank: int) -> np.ndarray:
    """Indices of this rank's ordinates: chunk `rank` of `world` near-equal contiguous chunks of each
    quadrant's range [quad[k], quad[k+1])."""
    idx = []
    for k in range(4):
        lo, hi = int(quad[k]), int(quad[k + 1])
        n = hi - lo
        b = lo + (n * rank) // world
        e = lo + (n * (rank + 1)) // world
        idx.extend(range(b, e))
    return np.asarray(idx, dtype=np.int64)


def local_quadrature(xi, eta, w, quad, idx):
    """The ordinate subset `idx` with its own quadrant bounds."""
    xi_l, eta_l, w_l = np.asarray(xi)[idx], np.asarray(eta)[idx], np.asarray(w)[idx]
    counts = [int(((idx >= quad[k]) & (idx < quad[k + 1])).sum()) for k in range(4)]
    q = np.zeros(5, dtype=np.int64)
    q[1:] = np.cumsum(counts)
    return xi_l, eta_l, w_l, q


class _DeviceVector:
    """A float64 vector of n entries at a raw device address, for torch.as_tensor without a copy."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def torch_allreduce_hook(device, group=None):
    """The all-reduce hook of idc_set_allreduce over torch.distributed (NCCL): sums the moment array in place on
    every rank and returns once the sums are there."""
    dev = torch.device(device)

    def fn(ptr: int, n: int) -> int:
        t = torch.as_tensor(_DeviceVector(ptr, n), device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        torch.cuda.current_stream(dev).synchronize()
        return 0

    return fn


class GpuBackend:
    """Sweeps of this rank's ordinates on its GPU through libidcsweep (device tensors)."""

    def __init__(self, P, idx, device: int = 0):
        from .abi import SweepContext
        self.P, self.idx, self.device = P, idx, torch.device(f"cuda:{device}")
        xi, eta, w, q = local_quadrature(P.xi, P.eta, P.w, P.quad, idx)
        self.nq_local = int(len(idx))
        self.ctx = SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by, device=device)
        self.ctx.set_ordinates(xi, eta, w, q)
        self.ctx.set_sigma(P.sigma_t, P.sigma_s)

    def zeros_phi(self):
        return torch.zeros(self.P.phi_shape(), dtype=torch.float64, device=self.device)

    def local_source(self, source):
        return torch.as_tensor(np.ascontiguousarray(source[:, :, self.idx]), device=self.device)

    def sweep(self, src, phi_scatter, dt, precision, want_psi=False):
        """Partial moments of L^{-1}(src + S phi_scatter) over this rank's ordinates (and the local psi)."""
        phi = self.zeros_phi()
        psi = torch.empty((self.P.nx + 2, self.P.ny + 2, self.nq_local, self.P.p + 1, self.P.p + 1),
                          dtype=torch.float64, device=self.device) if want_psi else None
        self.ctx.sweep_fused(None if src is None else src.data_ptr(), None if psi is None else psi.data_ptr(), dt,
                             None if phi_scatter is None else phi_scatter.data_ptr(), 1.0, phi.data_ptr(), precision)
        return (phi, psi) if want_psi else phi

    def close(self):
        self.ctx.close()


class DistributedTransport:
    """Source iteration and Peierls-form GMRES on ordinate-partitioned ranks (replicated phi)."""

    def __init__(self, backend, group=None):
        self.b, self.group = backend, group

    def _reduce(self, t):
        if dist.is_initialized():
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t

    def moments(self, src, phi_scatter, dt, precision=0):
        return self._reduce(self.b.sweep(src, phi_scatter, dt, precision))

    @staticmethod
    def _interior_dist(a, b):
        return float(torch.sqrt(((a[1:-1, 1:-1] - b[1:-1, 1:-1]) ** 2).sum()))

    def source_iteration(self, src, dt, abs_tol=1e-10, max_its=500, precision=0):
        """SISolver::Solve (linear_solvers/Abstract/ImplicitSolver/SISolver.cpp:190-254), absolute l2
        stopping rule on phi.  Returns (phi, local psi, iterations, error)."""
        phi = self.b.zeros_phi()
        err, its = math.inf, 0
        psi = None
        while its < max_its and err > abs_tol:
            its += 1
            part, psi = self.b.sweep(src, phi, dt, precision, want_psi=True)
            new = self._reduce(part)
            err = self._interior_dist(new, phi)
            phi = new
        return phi, psi, its, err

    def gmres(self, src, dt, abs_tol=1e-10, restart=30, max_its=3000, precision=0):
        """(I - P L^{-1} S) phi = P L^{-1} Q by GMRES(restart) from zero, stopping on the residual
        2-norm <= abs_tol (PETScPeierlsSolver, PETScPeierlsSolver.cpp:423-572); then the local
        psi = L^{-1}(S phi + Q).  Returns (phi, local psi, iterations, residual)."""
        b = self.moments(src, None, dt, precision)
        shape = b.shape
        bv = b.reshape(-1)
        A = lambda v: v - self.moments(None, v.reshape(shape), dt, precision).reshape(-1)
        x = torch.zeros_like(bv)
        r = bv.clone()
        beta = float(torch.linalg.vector_norm(r))
        its, resid = 0, beta
        while resid > abs_tol and its < max_its:
            V = [r / beta]
            H = np.zeros((restart + 1, restart))
            g = np.zeros(restart + 1)
            g[0] = beta
            cs, sn = np.zeros(restart), np.zeros(restart)
            k = 0
            for j in range(restart):
                w = A(V[j])
                for _ in range(2):   # CGS2
                    h = torch.stack([torch.dot(v, w) for v in V])
                    w = w - sum(hi * v for hi, v in zip(h, V))
                    H[:j + 1, j] += h.cpu().numpy()
                hn = float(torch.linalg.vector_norm(w))
                H[j + 1, j] = hn
                for i in range(j):
                    a, c = H[i, j], H[i + 1, j]
                    H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * c, -sn[i] * a + cs[i] * c
                rr = math.hypot(H[j, j], H[j + 1, j])
                cs[j], sn[j] = (H[j, j] / rr, H[j + 1, j] / rr) if rr > 0 else (1.0, 0.0)
                H[j, j], H[j + 1, j] = rr, 0.0
                g[j + 1], g[j] = -sn[j] * g[j], cs[j] * g[j]
                resid = abs(g[j + 1])
                its += 1
                k = j + 1
                if resid <= abs_tol or hn == 0.0 or its >= max_its:
                    break
                V.append(w / hn)
            y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
            x = x + sum(float(yi) * v for yi, v in zip(y, V[:k]))
            if resid <= abs_tol or its >= max_its:
                break
            r = bv - A(x)
            beta = float(torch.linalg.vector_norm(r))
            resid = beta
            if beta == 0.0:
                break
        phi = x.reshape(shape)
        _, psi = self.b.sweep(src, phi, dt, precision, want_psi=True)
        return phi, psi, its, resid

    def gmres_device(self, src, dt, abs_tol=1e-10, restart=30, max_its=3000, precision=0, hook=None):
        """The same solve by the library's GMRES on this rank's context (GpuBackend only): the partial moments
        of every sweep are completed by an all-reduce hook (idc_set_allreduce), so the Arnoldi process, the
        DSA preconditioner if the context has one, and the stopping test run on the device, identically on
        every rank, with one host synchronisation per Krylov step.  `hook` defaults to torch.distributed's
        all-reduce.  Returns (phi, local psi, iterations, residual)."""
        ctx = self.b.ctx
        ctx.set_allreduce(hook if hook is not None else torch_allreduce_hook(self.b.device, self.group))
        try:
            psi = src.clone()
            its, res = ctx.gmres_solve(psi.data_ptr(), dt, abs_tol=abs_tol, restart=restart, max_its=max_its,
                                       precision=precision, loc=1)
        finally:
            ctx.set_allreduce(None)
        phi = self.b.zeros_phi()
        ctx.pmv(1.0, 0.0, psi.data_ptr(), phi.data_ptr(), loc=1)
        if hook is None:
            self._reduce(phi)
        else:
            hook(phi.data_ptr(), phi.numel())
        return phi, psi, its, res
