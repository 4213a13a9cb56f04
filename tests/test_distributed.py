"""Ordinate-partitioned solves (idcsweep.distributed) as world_size-2 gloo process groups on CPU: the
partition covers every ordinate once, and distributed source iteration and GMRES reproduce the
single-process solution, with each rank's local psi equal to its slice of the full one.  The local sweeps
use a CPU backend built on the oracle restatement (test infrastructure); the GPU backend is the same
interface over libidcsweep."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import to_oracle
from idcsweep.distributed import DistributedTransport, local_quadrature, partition_ordinates
from idcsweep.problems import random_problem


def test_partition_covers_each_ordinate_once():
    quad = np.array([0, 7, 10, 21, 24])
    for world in (1, 2, 3, 4, 8):
        parts = [partition_ordinates(quad, world, r) for r in range(world)]
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(24))
        sizes = [len(p) for p in parts]
        assert max(sizes) - min(sizes) <= 4   # at most one extra per quadrant


def test_local_quadrature_bounds():
    from idcsweep.quadrature import level_symmetric_2d
    xi, eta, w, quad = level_symmetric_2d(8)
    idx = partition_ordinates(quad, 3, 1)
    xl, el, wl, ql = local_quadrature(xi, eta, w, quad, idx)
    assert ql[0] == 0 and ql[4] == len(idx)
    for k in range(4):
        s = slice(ql[k], ql[k + 1])
        assert np.all((xl[s] < 0) == (k >= 2)) and np.all((el[s] < 0) == bool(k & 1))


class OracleBackend:
    def __init__(self, P, idx):
        from oracle.bindings import Restatement, Problem as OP
        self.R = Restatement()
        xi, eta, w, q = local_quadrature(P.xi, P.eta, P.w, P.quad, idx)
        self.OP = OP(P.nx, P.ny, P.p, xi, eta, w, q, P.sigma_t, P.sigma_s, P.ax, P.bx, P.ay, P.by)
        self.P, self.idx = P, idx

    def zeros_phi(self):
        return torch.zeros(self.P.phi_shape(), dtype=torch.float64)

    def local_source(self, source):
        return torch.from_numpy(np.ascontiguousarray(source[:, :, self.idx]))

    def sweep(self, src, phi_scatter, dt, precision, want_psi=False):
        s = np.zeros(self.OP.psi_shape()) if src is None else src.numpy().copy()
        if phi_scatter is not None:
            s = self.R.smv(self.OP, phi_scatter.numpy(), s, alpha=1.0, beta=1.0)
        psi = self.R.sweep(self.OP, s, dt).reshape(self.OP.psi_shape())
        phi = torch.from_numpy(self.R.pmv(self.OP, psi).reshape(self.P.phi_shape()))
        return (phi, torch.from_numpy(psi)) if want_psi else phi


def _worker(rank, world, port, out_dir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        P = random_problem(7, 6, 1, 8, seed=21, dt=0.5)
        idx = partition_ordinates(P.quad, world, rank)
        be = OracleBackend(P, idx)
        dt_ = DistributedTransport(be)
        src = be.local_source(P.source)
        phi_si, psi_si, its, err = dt_.source_iteration(src, P.dt, abs_tol=1e-13, max_its=2000)
        phi_g, psi_g, its_g, res_g = dt_.gmres(src, P.dt, abs_tol=1e-13, restart=20)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), idx=idx, phi_si=phi_si.numpy(), psi_si=psi_si.numpy(),
                 phi_g=phi_g.numpy(), psi_g=psi_g.numpy(), res_g=res_g)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_solves_match_single_process(restatement):
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d), nprocs=world, join=True, start_method="spawn")
        res = [np.load(os.path.join(d, f"r{r}.npz")) for r in range(world)]
    P = random_problem(7, 6, 1, 8, seed=21, dt=0.5)
    OP = to_oracle(P)
    psi_ref, _, _ = restatement.source_iteration(OP, P.source, P.dt, abs_tol=1e-14, max_its=5000)
    psi_ref = psi_ref.reshape(P.psi_shape())
    phi_ref = restatement.pmv(OP, psi_ref).reshape(P.phi_shape())
    scale = np.abs(phi_ref).max()
    for r in res:
        assert np.abs(r["phi_si"] - phi_ref).max() < 1e-11 * scale
        assert np.abs(r["phi_g"] - phi_ref).max() < 1e-11 * scale
        assert float(r["res_g"]) <= 1e-13
        want = psi_ref[1:-1, 1:-1][:, :, r["idx"]]
        assert np.abs(r["psi_si"][1:-1, 1:-1] - want).max() < 1e-10 * np.abs(psi_ref).max()
        assert np.abs(r["psi_g"][1:-1, 1:-1] - want).max() < 1e-10 * np.abs(psi_ref).max()
    assert np.array_equal(res[0]["phi_g"], res[1]["phi_g"])   # replicated, identical on every rank
