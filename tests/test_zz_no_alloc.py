"""idc_sweep_noalloc, the sweep for callers that cannot allocate device memory (a code that owns all of
HBM through its own arena, or a loop that cannot pay for cudaMalloc's implicit synchronisation).

The entry point takes only caller-owned device pointers and keeps its scratch in a fixed device array;
this test (the caller) owns the buffers through torch.  Its results must match the context-based entry
point idc_sweep on two calls in a row -- the second on a different grid, so a stale queue head, error
word or progress flag left in the shared array by the first call would show.  Collected last so that a
run stopping at the first failure has already run every other test."""
import numpy as np
import pytest

from conftest import rel_err
from idcsweep import abi
from idcsweep.problems import random_problem

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL64 = 1e-12


def _context_result(P):
    with abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by) as ctx:
        ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
        ctx.set_sigma(P.sigma_t, P.sigma_s)
        psi = P.source.copy()
        phi = np.zeros(P.phi_shape())
        ctx.sweep(psi, P.dt, phi, abi.PREC_FP64)
    return psi, phi


def _noalloc_result(P):
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()
    xi, eta, w, st, src = d(P.xi), d(P.eta), d(P.w), d(P.sigma_t), d(P.source)
    # NaN everywhere: every interior value must be written by the call, the ghost cells left alone
    out = torch.full_like(src, float("nan"))
    phi = torch.full(P.phi_shape(), float("nan"), dtype=torch.float64, device="cuda")   # must be cleared by the call
    torch.cuda.synchronize()
    rc = abi.sweep_noalloc(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by, xi.data_ptr(), eta.data_ptr(), w.data_ptr(),
                           P.nq, P.quad, st.data_ptr(), src.data_ptr(), out.data_ptr(), P.dt, phi.data_ptr(),
                           abi.PREC_FP64, device=0, stream=None)
    assert rc == abi.IDC_OK, rc
    assert torch.equal(src, d(P.source))                # the source is not modified
    out = out.cpu().numpy()
    interior = np.zeros(out.shape[:2], bool)
    interior[1:-1, 1:-1] = True
    assert np.isnan(out[~interior]).all()               # ghost cells of the result are not written
    out[~interior] = P.source[~interior]                # ... and take the inflow values for the comparison
    return out, phi.cpu().numpy()


def test_noalloc_matches_sweep_on_two_calls_in_a_row():
    first = random_problem(37, 29, 2, 8, seed=404, dt=0.05)
    second = random_problem(64, 80, 1, 16, seed=405)   # more work items than the first call
    for P in (first, second):
        ref_psi, ref_phi = _context_result(P)
        psi, phi = _noalloc_result(P)
        assert not np.isnan(psi).any() and not np.isnan(phi).any()
        assert rel_err(psi, ref_psi) < TOL64
        assert rel_err(phi, ref_phi) < TOL64


def test_noalloc_phi_repeats_bitwise():
    """phi_out is summed over the ordinates in a fixed order, so two calls give the same bits."""
    P = random_problem(40, 33, 2, 12, seed=406)
    psi1, phi1 = _noalloc_result(P)
    psi2, phi2 = _noalloc_result(P)
    assert np.array_equal(phi1, phi2)
    assert np.array_equal(psi1, psi2)


def test_noalloc_rejects_oversized_problems():
    P = random_problem(2, 3, 0, 2, seed=1)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()
    xi, eta, w = d(P.xi), d(P.eta), d(P.w)
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    # S2 has one ordinate per quadrant: 16 rows per item, so 4 * 70000/16 items exceed the fixed scratch
    rc = abi.sweep_noalloc(2, 70000, 0, 0.0, 1.0, 0.0, 1.0, xi.data_ptr(), eta.data_ptr(), w.data_ptr(), P.nq,
                           P.quad, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr())
    assert rc == abi.IDC_ERR_ARG
    msg = abi.load_library().idc_last_error_message().decode()
    assert "work items" in msg and str(abi.IDC_NOALLOC_MAX_ITEMS) in msg, msg
