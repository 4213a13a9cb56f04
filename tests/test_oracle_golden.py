"""The CPU restatement against the golden fixtures that the reference produced (tests/golden/make_golden.py)."""
import glob
import os

import numpy as np
import pytest

from conftest import rel_err
from oracle.bindings import Problem as OP

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load(path):
    z = np.load(path)
    P = OP(int(z["nx"]), int(z["ny"]), int(z["p"]), z["xi"], z["eta"], z["w"], z["quad"], z["sigma_t"],
           z["sigma_s"], float(z["ax"]), float(z["bx"]), float(z["ay"]), float(z["by"]))
    return P, z


def test_fixtures_present():
    assert len(GOLDEN) >= 8


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_restatement_reproduces_golden(restatement, path):
    P, z = load(path)
    dt = float(z["dt"])
    psi = restatement.sweep(P, z["source"], dt)
    assert rel_err(psi, z["psi"]) < 1e-14
    assert rel_err(restatement.pmv(P, psi), z["phi"]) < 1e-14
    assert rel_err(restatement.lmv(P, z["source"]), z["lmv"]) < 1e-14
    assert rel_err(restatement.smv(P, z["phi"], z["source"], 0.75, 1.0), z["smv"]) < 1e-14
    si, its, err = restatement.source_iteration(P, z["source"], dt, abs_tol=float(z["si_tol"]), max_its=2000)
    assert rel_err(si, z["si_psi"]) < 1e-12
