"""Pins the CPU restatement (oracle/sweep_oracle.c) against the reference solver compiled from its own
sources (oracle/Makefile.ref): sweep, Pmv, Smv, Lmv and source iteration on seeded problems."""
import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idcsweep.problems import lattice, random_problem

CASES = [
    (1, 1, 0, 2, np.inf), (1, 1, 1, 4, 0.01), (2, 3, 1, 4, np.inf), (1, 9, 2, 8, np.inf), (9, 1, 1, 8, 0.1),
    (5, 4, 2, 8, np.inf), (4, 6, 1, 12, 0.02), (3, 5, 2, 16, np.inf), (8, 8, 1, 16, np.inf),
]


@pytest.mark.parametrize("nx,ny,p,sn,dt", CASES)
def test_restatement_matches_reference(restatement, reference, nx, ny, p, sn, dt):
    P = random_problem(nx, ny, p, sn, seed=100 * nx + ny, dt=dt)
    o = to_oracle(P)
    with reference.open(o, dt) as h:
        psi_ref = h.sweep(P.source, dt)
        phi_ref = h.pmv(psi_ref)
        lmv_ref = h.lmv(P.source)
        smv_ref = h.smv(phi_ref, P.source, 0.6, 1.4)
    psi = restatement.sweep(o, P.source, dt)
    phi = restatement.pmv(o, psi)
    assert rel_err(psi, psi_ref) < 1e-14
    assert rel_err(phi, phi_ref) < 1e-14
    assert rel_err(restatement.lmv(o, P.source), lmv_ref) < 1e-14
    assert rel_err(restatement.smv(o, phi, P.source, 0.6, 1.4), smv_ref) < 1e-14


def test_source_iteration_matches_reference(restatement, reference):
    P = lattice(12, 1, 8, dt=0.01)
    o = to_oracle(P)
    with reference.open(o, P.dt, abs_tol=1e-12, max_its=500) as h:
        ref = h.source_iteration(P.source, P.dt)
    psi, its, err = restatement.source_iteration(o, P.source, P.dt, abs_tol=1e-12, max_its=500)
    assert err <= 1e-12 and its > 1
    assert rel_err(psi, ref) < 1e-13
