"""The CUDA sweep through the C ABI against the oracle: golden fixtures made by the reference, the CPU
restatement on edge-case grids, and size-independent properties at the benchmark sizes.

Tolerances: FP64 path 1e-12 relative (max abs difference / max abs value) in psi and phi, the bar
the reference's CPU sweep is held to; FP32 cell solves with FP64 refinement 1e-8 relative in phi (the
mixed-precision target); unrefined FP32 5e-4 (it only shows that refinement matters)."""
import glob
import os

import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idcsweep import abi
from idcsweep.problems import lattice, lognormal, random_problem

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
TOL64 = 1e-12
TOL_REFINED = 1e-8


def context_for(P):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    return ctx


class _G:
    def __init__(self, z):
        self.nx, self.ny, self.p = int(z["nx"]), int(z["ny"]), int(z["p"])
        self.ax, self.bx, self.ay, self.by = float(z["ax"]), float(z["bx"]), float(z["ay"]), float(z["by"])
        self.xi, self.eta, self.w, self.quad = z["xi"], z["eta"], z["w"], z["quad"]
        self.sigma_t, self.sigma_s, self.source, self.dt = z["sigma_t"], z["sigma_s"], z["source"], float(z["dt"])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_golden_fp64(path):
    z = np.load(path)
    P = _G(z)
    with context_for(P) as ctx:
        psi = P.source.copy()
        phi = np.zeros(z["phi"].shape)
        ctx.sweep(psi, P.dt, phi, abi.PREC_FP64)
        assert rel_err(psi, z["psi"]) < TOL64
        assert rel_err(phi, z["phi"]) < TOL64
        # operators
        phi2 = np.zeros_like(phi)
        ctx.pmv(1.0, 0.0, z["psi"], phi2)
        assert rel_err(phi2, z["phi"]) < 1e-13
        y = P.source.copy()
        ctx.smv(0.75, 1.0, z["phi"], y)
        assert rel_err(y, z["smv"]) < 1e-13
        y = np.zeros_like(P.source)
        ctx.lmv(1.0, 0.0, P.source, y)
        assert rel_err(y, z["lmv"]) < 1e-13
        # source iteration
        si = P.source.copy()
        its, err = ctx.source_iteration(si, P.dt, abs_tol=float(z["si_tol"]), max_its=2000)
        assert err <= float(z["si_tol"])
        assert rel_err(si, z["si_psi"]) < 1e-11


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_golden_fp32_refined(path):
    z = np.load(path)
    P = _G(z)
    with context_for(P) as ctx:
        psi = P.source.copy()
        phi = np.zeros(z["phi"].shape)
        ctx.sweep(psi, P.dt, phi, abi.PREC_FP32_REFINED)
        assert rel_err(phi, z["phi"]) < TOL_REFINED
        assert rel_err(psi, z["psi"]) < TOL_REFINED


EDGE = [
    # nx, ny, p, sn, dt, (G, R) tiling or None
    (1, 1, 0, 2, np.inf, None), (1, 1, 2, 16, 0.01, None), (1, 17, 1, 8, np.inf, None), (17, 1, 1, 8, np.inf, None),
    (2, 3, 2, 4, 0.05, None), (7, 5, 1, 12, np.inf, (5, 3)), (9, 13, 2, 8, np.inf, (3, 2)),
    (16, 16, 1, 16, np.inf, (7, 4)), (33, 19, 2, 16, 0.1, None), (40, 40, 1, 8, np.inf, (10, 1)),
    (12, 30, 0, 12, np.inf, (21, 15)), (25, 7, 2, 8, 1.0, (1, 1)),
]


@pytest.mark.parametrize("nx,ny,p,sn,dt,tiling", EDGE)
def test_edge_cases_against_restatement(restatement, nx, ny, p, sn, dt, tiling):
    P = random_problem(nx, ny, p, sn, seed=nx * 31 + ny * 7 + p, dt=dt)
    o = to_oracle(P)
    ref = restatement.sweep(o, P.source, dt)
    ref_phi = restatement.pmv(o, ref)
    with context_for(P) as ctx:
        if tiling:
            ctx.set_tiling(*tiling)
        for prec, tol in ((abi.PREC_FP64, TOL64), (abi.PREC_FP32_REFINED, TOL_REFINED), (abi.PREC_FP32, 5e-4)):
            psi = P.source.copy()
            phi = np.zeros(P.phi_shape())
            ctx.sweep(psi, dt, phi, prec)
            assert rel_err(phi, ref_phi) < tol, prec
            if prec != abi.PREC_FP32:
                assert rel_err(psi, ref) < tol, prec
            # ghost cells of psi are inputs: untouched
            assert np.array_equal(psi[0], P.source[0]) and np.array_equal(psi[-1], P.source[-1])
            assert np.array_equal(psi[:, 0], P.source[:, 0]) and np.array_equal(psi[:, -1], P.source[:, -1])
            assert not phi[0].any() and not phi[-1].any() and not phi[:, 0].any() and not phi[:, -1].any()


def test_source_iteration_lattice(restatement):
    P = lattice(16, 1, 8, dt=0.01)
    o = to_oracle(P)
    ref, its_ref, _ = restatement.source_iteration(o, P.source, P.dt, abs_tol=1e-10, max_its=500)
    with context_for(P) as ctx:
        psi = P.source.copy()
        its, err = ctx.source_iteration(psi, P.dt, abs_tol=1e-10, max_its=500)
    assert err <= 1e-10
    assert abs(its - its_ref) <= 1
    assert rel_err(psi, ref) < 1e-10


def test_tiling_does_not_change_psi():
    P = random_problem(24, 20, 2, 8, seed=5)
    out = []
    with context_for(P) as ctx:
        for t in (None, (10, 1), (3, 7), (1, 16), (10, 32)):
            ctx.set_tiling(*(t or (0, 0)))
            psi = P.source.copy()
            ctx.sweep(psi, np.inf, None, abi.PREC_FP64)
            out.append(psi)
    for o in out[1:]:
        assert np.array_equal(o, out[0])


@pytest.mark.parametrize("p,sn,dt", [(2, 16, np.inf), (1, 12, 0.05), (0, 4, 1.0)])
def test_lane_and_modal_kernels_agree_on_every_tile_shape(restatement, p, sn, dt):
    """The lane-pipelined kernel (warps = 0) and the modal kernel (warps >= 1) do the same cell arithmetic:
    psi is bitwise the same for every tile shape of either; phi differs only in the order of its sums."""
    P = random_problem(37, 45, p, sn, seed=70 + p, dt=dt)
    ref = restatement.sweep(to_oracle(P), P.source, P.dt)
    shapes = [(4, 0), (8, 0), (16, 0), (4, 4), (8, 3), (16, 2), (32, 1), (0, 0)]
    outs = []
    with context_for(P) as ctx:
        for shape in shapes:
            ctx.set_tile_shape(*shape)
            psi = P.source.copy()
            phi = np.zeros(P.phi_shape())
            ctx.sweep(psi, P.dt, phi, abi.PREC_FP64)
            outs.append((psi, phi))
    assert rel_err(outs[0][0], ref) < 1e-12
    for psi, phi in outs[1:]:
        assert np.array_equal(psi, outs[0][0])
        assert rel_err(phi, outs[0][1]) < 1e-14


@pytest.mark.parametrize("p,sn,dt", [(2, 16, np.inf), (1, 8, 0.2), (0, 4, np.inf)])
def test_moments_only_sweep_matches_per_ordinate_sweep(restatement, p, sn, dt):
    """The Krylov iterations' sweep (no source array, psi not stored, moments of the fused scattering source
    out) runs on the lane kernel without per-ordinate transforms (modal sources per cell and quadrant, moments
    summed in the packed basis); its moments must match the per-ordinate path (modal kernel) and P L^-1 S
    of the restatement."""
    torch = pytest.importorskip("torch")
    P = random_problem(33, 29, p, sn, seed=90 + p, dt=dt, inflow=False)
    rng = np.random.default_rng(3)
    x = np.zeros(P.phi_shape())
    x[1:-1, 1:-1] = rng.uniform(0.1, 1.0, x[1:-1, 1:-1].shape)
    xd = torch.from_numpy(x).cuda()
    outs = []
    for shape in ((4, 0), (8, 0), (16, 0), (4, 4)):   # lane kernel (moments-only path) and modal kernel
        with context_for(P) as ctx:
            ctx.set_tile_shape(*shape)
            phi = torch.zeros(P.phi_shape(), dtype=torch.float64, device="cuda")
            ctx.sweep_fused(None, None, P.dt, xd.data_ptr(), 1.0, phi.data_ptr())
            outs.append(phi.cpu().numpy())
    OP = to_oracle(P)
    src = restatement.smv(OP, x, np.zeros(P.psi_shape()), 1.0, 0.0)   # S x on interior cells
    want = restatement.pmv(OP, restatement.sweep(OP, src, P.dt))
    for phi in outs:
        assert rel_err(phi, want) < 1e-12
        assert rel_err(phi, outs[-1]) < 1e-13


def test_bad_ordinates_rejected():
    P = random_problem(4, 4, 1, 4, seed=1)
    with abi.SweepContext(4, 4, 1) as ctx:
        xi = P.xi.copy()
        xi[0] = -xi[0]            # wrong sign for quadrant 0
        with pytest.raises(abi.IdcError) as e:
            ctx.set_ordinates(xi, P.eta, P.w, P.quad)
        assert e.value.code == abi.IDC_ERR_ARG
        with pytest.raises(abi.IdcError) as e:
            ctx.sweep(P.source.copy())
        assert e.value.code == abi.IDC_ERR_STATE


# ---- benchmark sizes: size-independent properties on device-resident data ----------------------------

torch = pytest.importorskip("torch")


def _device_problem(P):
    src = torch.from_numpy(P.source).cuda()
    return src


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_REFINED])
def test_full_size_residual_and_moments(prec):
    """256x256, Q2, S16 (the mixed-precision benchmark shape): the computed psi satisfies the discrete
    transport equation, checked by the FP64 Lmv operator: |q - (L + 1/dt) psi| / |q| small; the fused
    phi equals Pmv(psi)."""
    P = lognormal(256, 2, 16, seed=0)
    with context_for(P) as ctx:
        q = _device_problem(P)
        psi = q.clone()
        phi = torch.zeros(P.phi_shape(), dtype=torch.float64, device="cuda")
        ctx.sweep(psi.data_ptr(), P.dt, phi.data_ptr(), prec, loc=abi.LOC_DEVICE)
        lpsi = torch.zeros_like(psi)
        ctx.lmv(1.0, 0.0, psi.data_ptr(), lpsi.data_ptr(), loc=abi.LOC_DEVICE)
        interior = (slice(1, -1), slice(1, -1))
        r = (q - lpsi)[interior]
        rel = (r.abs().max() / q[interior].abs().max()).item()
        assert rel < (1e-11 if prec == abi.PREC_FP64 else 1e-7), rel
        phi2 = torch.zeros_like(phi)
        ctx.pmv(1.0, 0.0, psi.data_ptr(), phi2.data_ptr(), loc=abi.LOC_DEVICE)
        assert ((phi - phi2).abs().max() / phi2.abs().max()).item() < 1e-14


def test_full_size_linearity_and_precision_agreement():
    """512x512, Q1, S12 (the IDC benchmark shape): L^{-1}(2 q1 + q2) = 2 L^{-1} q1 + L^{-1} q2, and the
    FP32-refined sweep agrees with the FP64 sweep to the mixed-precision bar."""
    P = lattice(512, 1, 12, dt=0.005)
    with context_for(P) as ctx:
        q1 = torch.from_numpy(P.source).cuda()
        g = torch.Generator(device="cuda").manual_seed(3)
        q2 = torch.rand(q1.shape, dtype=torch.float64, device="cuda", generator=g)
        a, b, c = q1.clone(), q2.clone(), (2 * q1 + q2)
        for t in (a, b, c):
            ctx.sweep(t.data_ptr(), P.dt, None, abi.PREC_FP64, loc=abi.LOC_DEVICE)
        lin = ((c - (2 * a + b)).abs().max() / c.abs().max()).item()
        assert lin < 1e-12, lin
        phi64 = torch.zeros(P.phi_shape(), dtype=torch.float64, device="cuda")
        phi32 = torch.zeros_like(phi64)
        x, y = q1.clone(), q1.clone()
        ctx.sweep(x.data_ptr(), P.dt, phi64.data_ptr(), abi.PREC_FP64, loc=abi.LOC_DEVICE)
        ctx.sweep(y.data_ptr(), P.dt, phi32.data_ptr(), abi.PREC_FP32_REFINED, loc=abi.LOC_DEVICE)
        assert ((phi32 - phi64).abs().max() / phi64.abs().max()).item() < TOL_REFINED


@pytest.mark.parametrize("count", [1, 2, 5])
def test_sweep_out_many_host_matches_single_sweeps(count):
    """The overlapped host-array form gives each step exactly what idc_sweep_out gives it (bitwise psi
    and phi), with different sources per step and the callers' ghost cells untouched."""
    P = random_problem(13, 11, 2, 8, seed=21)
    rng = np.random.default_rng(5)
    srcs = [P.source * (1.0 + 0.1 * k) + 0.01 * rng.standard_normal(P.source.shape) for k in range(count)]
    with context_for(P) as ctx:
        want, wphi = [], []
        for s in srcs:
            r = np.full_like(s, 7.0)
            f = np.zeros(P.phi_shape())
            ctx.sweep_out(s, r, P.dt, f)
            want.append(r)
            wphi.append(f)
        outs = [np.full_like(s, 7.0) for s in srcs]
        phis = [np.zeros(P.phi_shape()) for _ in srcs]
        ctx.sweep_out_many(srcs, outs, phis, P.dt)
        for k in range(count):
            assert np.array_equal(outs[k], want[k])   # ghost cells keep the 7.0 fill in both
            assert np.array_equal(phis[k], wphi[k])
