import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "idc-transport-solver_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def restatement():
    from oracle.bindings import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle.bindings import Reference, reference_available
    if not reference_available():
        pytest.skip("reference library oracle/_ref/libidcref.so not built (needs the reference sources)")
    return Reference()


def to_oracle(P):
    """idcsweep.problems.Problem -> oracle.bindings.Problem."""
    from oracle.bindings import Problem as OP
    return OP(P.nx, P.ny, P.p, P.xi, P.eta, P.w, P.quad, P.sigma_t, P.sigma_s, P.ax, P.bx, P.ay, P.by)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / (scale if scale > 0 else 1.0))
