"""Generates the golden fixtures in this folder by running the REFERENCE solver (crockatt/
idc-transport-solver compiled from its own sources by oracle/Makefile.ref, driven through
oracle/ref_driver.cpp) on small seeded problems.

    python tests/golden/make_golden.py

Each fixture holds the problem inputs (grid, ordinates, cross sections, angular source, dt) and the
reference's outputs: the in-place sweep (SweepOperator::Apply), phi = Pmv(psi), Lmv(source), Smv and
the source-iteration solution (SISolver::Solve).  The reference publishes no test vectors of its own,
so these are the pins for the CPU restatement (tests/test_oracle_golden.py) and the CUDA path
(tests/test_sweep_gpu.py).
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


def main():
    ref = Reference()
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
