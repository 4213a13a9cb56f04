"""Generates the golden fixtures in this folder by running the REFERENCE solver (crockatt/
idc-transport-solver compiled from its own sources by oracle/Makefile.ref, driven through
oracle/ref_driver.cpp) on small seeded problems.

    python tests/golden/make_golden.py

Each fixture in this folder holds the problem inputs (grid, ordinates, cross sections, angular source,
dt) and the reference's outputs: the in-place sweep (SweepOperator::Apply), phi = Pmv(psi), Lmv(source), Smv and
the source-iteration solution (SISolver::Solve).  The reference publishes no test vectors of its own,
so these are the pins for the CPU restatement (tests/test_oracle_golden.py) and the CUDA path
(tests/test_sweep_gpu.py).  config/ holds the reference's results on full-size benchmark problems
(config/config0_lattice64_q1_s8.npz: its own 64x64 lattice case solved by SISolver::Solve), for the GPU
tests at those sizes.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "idc-transport-solver_b200"))

from idcsweep.problems import random_problem, lattice  # noqa: E402
from oracle.bindings import Reference, Problem as OP  # noqa: E402

CASES = [
    # name, builder
    ("rand_1x1_p1_s4", lambda: random_problem(1, 1, 1, 4, seed=11)),
    ("rand_2x3_p1_s4_dt", lambda: random_problem(2, 3, 1, 4, seed=12, dt=0.01)),
    ("rand_1x5_p2_s8", lambda: random_problem(1, 5, 2, 8, seed=13)),
    ("rand_6x1_p0_s8_dt", lambda: random_problem(6, 1, 0, 8, seed=14, dt=0.5)),
    ("rand_3x2_p2_s8", lambda: random_problem(3, 2, 2, 8, seed=15)),
    ("rand_2x4_p1_s12_dt", lambda: random_problem(2, 4, 1, 12, seed=16, dt=0.02)),
    ("rand_2x2_p2_s16", lambda: random_problem(2, 2, 2, 16, seed=17, inflow=False)),
    ("lattice_8_p1_s8_dt", lambda: lattice(8, 1, 8, dt=0.01)),
]


def config0(ref):
    """The reference's own CPU-runnable case at full size: 64x64 lattice on [0,7]^2, Q1, S8, one implicit-Euler
    step of dt = 0.01 from zero flux, source iteration to 1e-10 (absolute l2 change of phi, SISolver::Solve).
    The fixture keeps the inputs' cross sections, the source's checksum, the reference's phi and its psi on
    64 seeded cells (the whole psi would be 5.6 MB)."""
    P = lattice(64, 1, 8, dt=0.01)
    o = OP(P.nx, P.ny, P.p, P.xi, P.eta, P.w, P.quad, P.sigma_t, P.sigma_s, P.ax, P.bx, P.ay, P.by)
    with ref.open(o, P.dt, abs_tol=1e-10, max_its=5000) as h:
        psi = h.source_iteration(P.source, P.dt)
        phi = h.pmv(psi)
    rng = np.random.default_rng(64)
    cells = np.stack([rng.integers(1, P.nx + 1, 64), rng.integers(1, P.ny + 1, 64)], axis=1)
    np.savez_compressed(
        os.path.join(HERE, "config", "config0_lattice64_q1_s8.npz"), nx=P.nx, ny=P.ny, p=P.p, dt=P.dt,
        sigma_t=P.sigma_t, sigma_s=P.sigma_s, source_sum=P.source.sum(), source_abs_sum=np.abs(P.source).sum(),
        si_tol=1e-10, phi=phi, cells=cells, psi_cells=psi[cells[:, 0], cells[:, 1]])
    print("wrote config0_lattice64_q1_s8", phi.shape)


def main():
    ref = Reference()
    os.makedirs(os.path.join(HERE, "config"), exist_ok=True)
    config0(ref)
    for name, build in CASES:
        P = build()
        o = OP(P.nx, P.ny, P.p, P.xi, P.eta, P.w, P.quad, P.sigma_t, P.sigma_s, P.ax, P.bx, P.ay, P.by)
        with ref.open(o, P.dt, abs_tol=1e-12, max_its=2000) as h:
            psi = h.sweep(P.source, P.dt)
            phi = h.pmv(psi)
            lmv = h.lmv(P.source)
            smv = h.smv(phi, P.source, 0.75, 1.0)
            si = h.source_iteration(P.source, P.dt)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), nx=P.nx, ny=P.ny, p=P.p, ax=P.ax, bx=P.bx, ay=P.ay, by=P.by,
            dt=P.dt, xi=P.xi, eta=P.eta, w=P.w, quad=P.quad, sigma_t=P.sigma_t, sigma_s=P.sigma_s,
            source=P.source, psi=psi, phi=phi, lmv=lmv, smv=smv, si_psi=si, si_tol=1e-12)
        print("wrote", name, P.source.shape)


if __name__ == "__main__":
    main()
