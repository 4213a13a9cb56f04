"""IDC time stepping on the GPU against the restated reference IDC (tests/idc_ref.py) on the oracle's
operators, graph replay against plain launches, and the temporal order of accuracy."""
import numpy as np
import pytest

from conftest import rel_err, to_oracle
from idc_ref import idc_steps
from idcsweep import abi
from idcsweep.problems import lattice, random_problem

pytestmark = pytest.mark.gpu


def context_for(P):
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    return ctx


def _problem(n=10, p=1):
    P = lattice(n, p, 4, dt=0.01)
    psi0 = np.zeros(P.psi_shape())
    return P, psi0


@pytest.mark.parametrize("use_graph", [False, True])
@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-12), (abi.PREC_FP32_REFINED, 1e-9)])
def test_imex_idc_matches_restated_reference(restatement, use_graph, prec, tol):
    P, psi0 = _problem()
    want = idc_steps(restatement, to_oracle(P), psi0, P.source, P.dt, 3, M=4, K=3, scattering="explicit")
    with context_for(P) as ctx:
        psi = psi0.copy()
        sweeps = ctx.idc_integrate(psi, P.source, P.dt, 3, 4, 3, abi.SCATTER_EXPLICIT, prec, use_graph=use_graph)
    assert sweeps == 3 * 3 * 4
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < tol


def test_implicit_idc_matches_restated_reference(restatement):
    P, psi0 = _problem(n=8)
    want = idc_steps(restatement, to_oracle(P), psi0, P.source, P.dt, 2, M=3, K=2, scattering="implicit")
    with context_for(P) as ctx:
        psi = psi0.copy()
        ctx.idc_integrate(psi, P.source, P.dt, 2, 3, 2, abi.SCATTER_IMPLICIT, abi.PREC_FP64, abs_tol=1e-14)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-10


def test_graph_replay_is_bitwise_plain_launches():
    P = lattice(32, 1, 8, dt=0.005)
    out = []
    for g in (False, True):
        with context_for(P) as ctx:
            psi = np.zeros(P.psi_shape())
            ctx.idc_integrate(psi, P.source, P.dt, 5, 4, 3, abi.SCATTER_EXPLICIT, abi.PREC_FP64, use_graph=g)
            out.append(psi)
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("scattering", [abi.SCATTER_EXPLICIT, abi.SCATTER_IMPLICIT])
def test_idc_fourth_order_in_time(scattering):
    """4 Lobatto nodes + 3 corrections: the error at T against a 16x finer run falls ~16x per halving of dt."""
    P = random_problem(4, 4, 1, 4, seed=9, inflow=True, sigma_range=(0.5, 2.0))
    T = 0.4
    src = P.source.copy()
    psi0 = P.source.copy()   # ghost cells: the same inflow as the source (no jump in time at t = 0)
    psi0[1:-1, 1:-1] = 0.1
    sols = {}
    with context_for(P) as ctx:
        for m in (2, 4, 8, 64):
            psi = psi0.copy()
            ctx.idc_integrate(psi, src, T / m, m, 4, 3, scattering, abi.PREC_FP64, abs_tol=1e-14)
            sols[m] = psi[1:-1, 1:-1]
    e = [np.abs(sols[m] - sols[64]).max() for m in (2, 4, 8)]
    orders = [np.log2(e[k] / e[k + 1]) for k in range(2)]
    assert orders[-1] > 3.5 and min(orders) > 3.0, (e, orders)


def test_idc_rejects_bad_arguments():
    P, psi0 = _problem(n=6)
    with context_for(P) as ctx:
        for kw in ({"dt": np.inf}, {"num_nodes": 1}, {"scattering": 5}):
            args = dict(dt=P.dt, num_nodes=4, scattering=abi.SCATTER_EXPLICIT)
            args.update(kw)
            with pytest.raises(abi.IdcError):
                ctx.idc_integrate(psi0.copy(), P.source, args["dt"], 1, args["num_nodes"], 3, args["scattering"])


@pytest.mark.parametrize("p,M,prec,tol", [
    (2, 4, abi.PREC_FP64, 1e-12),     # Q2
    (1, 2, abi.PREC_FP64, 1e-12), (1, 3, abi.PREC_FP64, 1e-12), (1, 5, abi.PREC_FP64, 1e-12),
    (1, 6, abi.PREC_FP64, 1e-12),     # more nodes than the fused correction kernel takes
    (1, 4, abi.PREC_FP32, 5e-3),      # unrefined FP32 sweeps: sources combined into a scratch array first
])
def test_imex_idc_degrees_nodes_precisions(restatement, p, M, prec, tol):
    """IMEX-IDC against the restated reference for every way a substep's source is formed: in the sweep
    (fused correction sources plus psi_{n-1} / (h dt)), combined into a scratch array first, or by the
    separate residual and source kernels."""
    P, psi0 = _problem(n=9, p=p)
    want = idc_steps(restatement, to_oracle(P), psi0, P.source, P.dt, 2, M=M, K=2, scattering="explicit")
    with context_for(P) as ctx:
        psi = psi0.copy()
        sweeps = ctx.idc_integrate(psi, P.source, P.dt, 2, M, 2, abi.SCATTER_EXPLICIT, prec, use_graph=True)
    assert sweeps == 2 * 3 * (M - 1)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < tol


@pytest.mark.parametrize("case", [
    dict(kind="lattice", n=10, p=1, sn=4, M=4, K=3, steps=3),
    dict(kind="random", n=7, p=2, sn=8, M=4, K=3, steps=2),
    dict(kind="random", n=6, p=1, sn=12, M=3, K=2, steps=2),
])
def test_implicit_idc_matches_reference_integrator(reference, case):
    """The GPU's implicit IDC (GMRES substeps to 1e-14) against the reference's own IDCIntegrator (oracle/_ref:
    IDCIntegrator::Step, update form, Gauss-Lobatto nodes, SISolver substeps to 1e-14), vacuum boundaries."""
    if case["kind"] == "lattice":
        P = lattice(case["n"], case["p"], case["sn"], dt=0.01)
    else:
        P = random_problem(case["n"], case["n"] + 1, case["p"], case["sn"], seed=31, dt=0.05, inflow=False,
                           sigma_range=(0.5, 4.0))
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = 0.05
    with reference.open(to_oracle(P), P.dt, abs_tol=1e-14, max_its=100000) as h:
        want = h.idc_steps(psi0, P.source, P.dt, case["steps"], case["M"], case["K"], si_abs_tol=1e-14)
    with context_for(P) as ctx:
        psi = psi0.copy()
        ctx.idc_integrate(psi, P.source, P.dt, case["steps"], case["M"], case["K"], abi.SCATTER_IMPLICIT,
                          abi.PREC_FP64, abs_tol=1e-14)
    assert rel_err(psi[1:-1, 1:-1], want[1:-1, 1:-1]) < 1e-10


def test_implicit_idc_with_inflow_stepwise_matches_reference_integrator(reference):
    """With inflow data the reference zeroes the ghost cells of each step's result; one GPU step per call
    with the ghost cells zeroed in between reproduces its multi-step result."""
    P = random_problem(6, 5, 1, 8, seed=3, dt=0.05, inflow=True, sigma_range=(0.5, 4.0))
    psi0 = np.zeros(P.psi_shape())
    with reference.open(to_oracle(P), P.dt, abs_tol=1e-14, max_its=100000) as h:
        want = h.idc_steps(psi0, P.source, P.dt, 3, 4, 3, si_abs_tol=1e-14)
    psi = psi0.copy()
    with context_for(P) as ctx:
        for _ in range(3):
            ctx.idc_integrate(psi, P.source, P.dt, 1, 4, 3, abi.SCATTER_IMPLICIT, abi.PREC_FP64, abs_tol=1e-14)
            psi[0], psi[-1], psi[:, 0], psi[:, -1] = 0.0, 0.0, 0.0, 0.0
    assert rel_err(psi, want) < 1e-10
