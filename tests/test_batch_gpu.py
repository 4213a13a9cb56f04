"""Batched sweeps (several problems in one launch per DG degree) and the autotuner: psi is bitwise the
per-problem sweep's (cell arithmetic does not depend on the tiling), phi agrees to rounding."""
import numpy as np
import pytest
import torch

from conftest import rel_err
from idcsweep import abi
from idcsweep.problems import lognormal, random_problem

pytestmark = pytest.mark.gpu


def _ctx(P):
    c = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    c.set_ordinates(P.xi, P.eta, P.w, P.quad)
    c.set_sigma(P.sigma_t, P.sigma_s)
    return c


def _problems():
    return [random_problem(9, 7, 1, 4, seed=1), random_problem(16, 20, 2, 8, seed=2), lognormal(24, 1, 12, seed=3),
            random_problem(5, 13, 2, 4, seed=4, dt=0.2), lognormal(12, 2, 16, seed=5), random_problem(1, 6, 1, 8, seed=6)]


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_REFINED])
def test_batched_sweep_matches_individual_sweeps(prec):
    probs = _problems()
    dts = {P.dt for P in probs}
    ctxs = [_ctx(P) for P in probs]
    try:
        for dt in dts:
            sel = [k for k, P in enumerate(probs) if P.dt == dt]
            srcs = [torch.from_numpy(probs[k].source).cuda() for k in sel]
            outs = [torch.zeros_like(s) for s in srcs]
            phis = [torch.zeros(probs[k].phi_shape(), dtype=torch.float64, device="cuda") for k in sel]
            with abi.Batch() as b:
                for k in sel:
                    b.add(ctxs[k])
                b.sweep([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], [f.data_ptr() for f in phis], dt,
                        prec)
                b.sweep([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], [f.data_ptr() for f in phis], dt,
                        prec)   # reuse (re-armed traces)
            for j, k in enumerate(sel):
                want = torch.zeros_like(srcs[j])
                wphi = torch.zeros_like(phis[j])
                ctxs[k].sweep_out(srcs[j].data_ptr(), want.data_ptr(), dt, wphi.data_ptr(), prec, loc=abi.LOC_DEVICE)
                assert torch.equal(outs[j][1:-1, 1:-1], want[1:-1, 1:-1])
                assert rel_err(phis[j].cpu().numpy(), wphi.cpu().numpy()) < 1e-14
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("seg", [4, 8, 16])
def test_batched_lane_shapes_match_individual_sweeps(seg):
    """The lane kernel run over a batch (tile shape (seg, 0), FP64): every member's psi bitwise its own sweep's,
    phi to rounding, with a reused batch and members of both degrees."""
    probs = [P for P in _problems() if P.dt == np.inf]
    ctxs = [_ctx(P) for P in probs]
    try:
        srcs = [torch.from_numpy(P.source).cuda() for P in probs]
        outs = [torch.zeros_like(s) for s in srcs]
        phis = [torch.zeros(P.phi_shape(), dtype=torch.float64, device="cuda") for P in probs]
        with abi.Batch() as b:
            for c in ctxs:
                b.add(c)
            for p in (1, 2):
                b.set_shape(p, abi.PREC_FP64, seg, 0)
                assert b.get_shape(p, abi.PREC_FP64) == (seg, 0)
            for _ in range(2):
                b.sweep([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], [f.data_ptr() for f in phis],
                        np.inf)
            with pytest.raises(abi.IdcError) as e:   # the lane kernel has no FP32 form
                b.set_shape(1, abi.PREC_FP32_REFINED, seg, 0)
            assert e.value.code == abi.IDC_ERR_ARG
        for j, c in enumerate(ctxs):
            want = torch.zeros_like(srcs[j])
            wphi = torch.zeros_like(phis[j])
            c.sweep_out(srcs[j].data_ptr(), want.data_ptr(), np.inf, wphi.data_ptr(), loc=abi.LOC_DEVICE)
            assert torch.equal(outs[j][1:-1, 1:-1], want[1:-1, 1:-1])
            assert rel_err(phis[j].cpu().numpy(), wphi.cpu().numpy()) < 1e-14
    finally:
        for c in ctxs:
            c.close()


def test_batched_gmres_on_lane_shapes():
    """Batched GMRES + DSA with the lane kernel's shapes (converged members skipped inside its launches): the
    members' own solutions."""
    probs = [random_problem(12, 9, 1, 4, seed=31), lognormal(40, 2, 8, seed=32, c_range=(0.3, 0.99)),
             lognormal(24, 1, 12, seed=33, c_range=(0.5, 0.95))]
    tol = 1e-10
    ctxs = [_ctx(P) for P in probs]
    try:
        want = []
        for P, c in zip(probs, ctxs):
            c.set_preconditioner(abi.PRECOND_DSA, 20)
            psi = P.source.copy()
            c.gmres_solve(psi, P.dt, abs_tol=tol, restart=10, max_its=2000)
            want.append(psi)
        psis = [torch.from_numpy(P.source).cuda() for P in probs]
        with abi.Batch() as b:
            for c in ctxs:
                b.add(c)
            b.set_shape(1, abi.PREC_FP64, 16, 0)
            b.set_shape(2, abi.PREC_FP64, 8, 0)
            its, res = b.gmres_solve([x.data_ptr() for x in psis], np.inf, abs_tol=tol, restart=10, max_its=2000)
        for k in range(len(probs)):
            assert res[k] <= tol
            assert rel_err(psis[k].cpu().numpy(), want[k]) < 1e-8
    finally:
        for c in ctxs:
            c.close()


def test_autotuners_keep_results():
    probs = _problems()[:3]
    ctxs = [_ctx(P) for P in probs]
    try:
        srcs = [torch.from_numpy(P.source).cuda() for P in probs]
        outs = [torch.zeros_like(s) for s in srcs]
        with abi.Batch() as b:
            for c in ctxs:
                b.add(c)
            b.autotune([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], np.inf)
            b.sweep([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], None, np.inf)
        for j, c in enumerate(ctxs):
            seg, wn = c.autotune(srcs[j].data_ptr(), np.inf)
            assert seg in (4, 8, 16, 32) and 0 <= wn <= 7   # wn = 0: the lane kernel
            want = torch.zeros_like(srcs[j])
            c.sweep_out(srcs[j].data_ptr(), want.data_ptr(), np.inf, None, loc=abi.LOC_DEVICE)
            assert torch.equal(outs[j][1:-1, 1:-1], want[1:-1, 1:-1])
    finally:
        for c in ctxs:
            c.close()


def test_batched_sweep_complete_on_return():
    """Every degree group has finished when the batched sweep returns: the results are read at once on
    another stream, with the largest problem in the last group to launch (the highest degree)."""
    probs = [random_problem(24, 24, 1, 4, seed=11), lognormal(160, 2, 16, seed=12)]
    ctxs = [_ctx(P) for P in probs]
    try:
        srcs = [torch.from_numpy(P.source).cuda() for P in probs]
        outs = [torch.zeros_like(s) for s in srcs]
        phis = [torch.zeros(P.phi_shape(), dtype=torch.float64, device="cuda") for P in probs]
        want = []
        for j, c in enumerate(ctxs):
            w = torch.zeros_like(srcs[j])
            c.sweep_out(srcs[j].data_ptr(), w.data_ptr(), np.inf, None, loc=abi.LOC_DEVICE)
            want.append(w.cpu())
        with abi.Batch() as b:
            for c in ctxs:
                b.add(c)
            for _ in range(3):
                for o in outs:
                    o.zero_()
                torch.cuda.synchronize()
                b.sweep([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], [f.data_ptr() for f in phis],
                        np.inf)
                got = [o.cpu() for o in outs]   # torch's stream: ordered after the sweep only by its return
                for j in range(len(probs)):
                    assert torch.equal(got[j][1:-1, 1:-1], want[j][1:-1, 1:-1])
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("dsa", [False, True])
def test_batched_gmres_matches_single_solves(dsa):
    """Every member's Peierls GMRES (+ DSA) solved together, one batched sweep per Krylov step with converged
    members skipped: the same solutions as the members' own solves to the tolerance."""
    probs = [random_problem(12, 9, 1, 4, seed=21), lognormal(40, 2, 8, seed=22, c_range=(0.3, 0.99)),
             lognormal(24, 1, 12, seed=23, c_range=(0.5, 0.95)), random_problem(7, 16, 2, 4, seed=24, inflow=False)]
    tol = 1e-10
    ctxs = [_ctx(P) for P in probs]
    try:
        for c in ctxs:
            if dsa:
                c.set_preconditioner(abi.PRECOND_DSA, 20)
        want, want_its = [], []
        for P, c in zip(probs, ctxs):
            psi = P.source.copy()
            its, res = c.gmres_solve(psi, P.dt, abs_tol=tol, restart=10, max_its=2000)
            want.append(psi)
            want_its.append(its)
        psis = [torch.from_numpy(P.source).cuda() for P in probs]
        with abi.Batch() as b:
            for c in ctxs:
                b.add(c)
            its, res = b.gmres_solve([x.data_ptr() for x in psis], np.inf, abs_tol=tol, restart=10, max_its=2000)
        for k, P in enumerate(probs):
            assert res[k] <= tol
            assert abs(its[k] - want_its[k]) <= 1
            assert rel_err(psis[k].cpu().numpy(), want[k]) < 1e-8
    finally:
        for c in ctxs:
            c.close()
