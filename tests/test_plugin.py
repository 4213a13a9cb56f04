"""The drop-in boundary seen from the reference's side: the reference solver, compiled from its own
sources, with the GPU sweep pattern plugged into its factory (oracle/sweep_pattern_gpu.cpp, deck key
`sweep_pattern gpu-wavefront`, oracle/_ref/libidcref_gpu.so).  The reference's own SweepOperator::Apply,
SISolver::Solve and IDCIntegrator::Step run unchanged on top of it; their results must match the same
reference code with its CPU wavefront pattern."""
import os

import numpy as np
import pytest

from conftest import gpu_available, rel_err, to_oracle
from idcsweep.problems import lattice, lognormal, random_problem, smooth_sigma
from oracle.bindings import REFERENCE_GPU_SO, Reference

pytestmark = pytest.mark.skipif(not os.path.exists(REFERENCE_GPU_SO),
                                reason="oracle/_ref/libidcref_gpu.so not built (needs the reference sources)")


@pytest.fixture(scope="module")
def plugged():
    return Reference(REFERENCE_GPU_SO)


@pytest.mark.skipif(gpu_available(), reason="checks the failure without a GPU")
def test_plugin_fails_loudly_without_a_gpu(plugged):
    """No CUDA device: creating the pattern throws (the reference's error style) and the driver reports it;
    nothing falls back to a CPU sweep."""
    P = random_problem(4, 3, 1, 4, seed=1)
    with pytest.raises(RuntimeError):
        plugged.open(to_oracle(P), P.dt, pattern="gpu-wavefront")
    with plugged.open(to_oracle(P), P.dt, pattern="wavefront") as h:   # the CPU patterns still work
        assert np.isfinite(h.sweep(P.source, P.dt)).all()


@pytest.mark.gpu
@pytest.mark.parametrize("p,sn,dt", [(0, 4, 0.5), (1, 8, np.inf), (2, 12, 0.05)])
def test_reference_apply_through_plugin(plugged, p, sn, dt):
    P = random_problem(13, 9, p, sn, seed=50 + p, dt=dt)
    with plugged.open(to_oracle(P), P.dt, pattern="wavefront") as h:
        want = h.sweep(P.source, P.dt)
    with plugged.open(to_oracle(P), P.dt, pattern="gpu-wavefront") as h:
        got = h.sweep(P.source, P.dt)
    assert rel_err(got, want) < 1e-12


@pytest.mark.gpu
def test_reference_source_iteration_through_plugin(plugged):
    """SISolver::Solve (SISolver.cpp:190-254) on the reference's 64x64 lattice case, gpu-wavefront against
    wavefront."""
    P = lattice(64, 1, 8, dt=0.01)
    out = {}
    for pattern in ("wavefront", "gpu-wavefront"):
        with plugged.open(to_oracle(P), P.dt, pattern=pattern, abs_tol=1e-10, max_its=5000) as h:
            psi = h.source_iteration(P.source, P.dt)
            out[pattern] = h.pmv(psi)
    assert rel_err(out["gpu-wavefront"], out["wavefront"]) < 1e-12


@pytest.mark.gpu
def test_reference_idc_integrator_through_plugin(plugged):
    """IDCIntegrator::Step (idc.cpp:521, 846-955) with SISolver substeps, sweeping on the GPU."""
    P = random_problem(12, 10, 1, 8, seed=61, dt=0.05, inflow=False, sigma_range=(0.5, 4.0))
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = 0.05
    out = {}
    for pattern in ("wavefront", "gpu-wavefront"):
        with plugged.open(to_oracle(P), P.dt, pattern=pattern, abs_tol=1e-13, max_its=100000) as h:
            out[pattern] = h.idc_steps(psi0, P.source, P.dt, 2, 4, 3, si_abs_tol=1e-13)
    assert rel_err(out["gpu-wavefront"], out["wavefront"]) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("edges", [1, 2 | 4, 15])
def test_reference_source_iteration_with_reflecting_edges_through_plugin(plugged, edges):
    """The reference's SISolver::Solve with reflecting edges (sequential quadrants, ReflectBoundaries between
    them): gpu-wavefront against wavefront."""
    P = lognormal(20, 1, 8, seed=7, c_range=(0.3, 0.9), dt=0.3)
    out = {}
    for pattern in ("wavefront", "gpu-wavefront"):
        with plugged.open(to_oracle(P), P.dt, pattern=pattern, abs_tol=1e-12, max_its=5000, reflect=edges) as h:
            psi = h.source_iteration(P.source, P.dt)
            out[pattern] = h.pmv(psi)
    assert rel_err(out["gpu-wavefront"], out["wavefront"]) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 2])
def test_reference_source_iteration_with_high_order_cross_sections_through_plugin(plugged, p):
    """The reference's SISolver::Solve with CrossSection objects of DG degree p: gpu-wavefront (which makes its
    context with the cross sections' degree) against wavefront."""
    P = smooth_sigma(12, p, 4, seed=11 + p, dt=0.4)
    out = {}
    for pattern in ("wavefront", "gpu-wavefront"):
        with plugged.open(to_oracle(P), P.dt, pattern=pattern, abs_tol=1e-12, max_its=5000, sigma_degree=p) as h:
            psi = h.source_iteration(P.source, P.dt)
            out[pattern] = h.pmv(psi)
    assert rel_err(out["gpu-wavefront"], out["wavefront"]) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 2])
def test_reference_source_iteration_on_a_periodic_grid_through_plugin(plugged, p):
    """The reference's SISolver::Solve with Global::periodic (halos synchronised between iterations; the plugin
    leaves them dirty after its sweep, as the reference's patterns do): gpu-wavefront against wavefront."""
    P = lognormal(14, p, 4, seed=13 + p, c_range=(0.3, 0.8), dt=0.4)
    out = {}
    for pattern in ("wavefront", "gpu-wavefront"):
        with plugged.open(to_oracle(P), P.dt, pattern=pattern, abs_tol=1e-12, max_its=5000, periodic=True) as h:
            psi = h.source_iteration(P.source, P.dt)
            out[pattern] = h.pmv(psi)
    assert rel_err(out["gpu-wavefront"], out["wavefront"]) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("reflect,periodic", [(15, False), (0, True)])
def test_reference_idc_integrator_with_boundaries_through_plugin(plugged, reflect, periodic):
    """IDCIntegrator::Step with reflecting edges (it reflects each step's initial stage) or on a periodic grid,
    its SISolver substeps sweeping on the GPU: gpu-wavefront against wavefront."""
    P = random_problem(10, 9, 1, 4, seed=62, dt=0.05, inflow=False, sigma_range=(0.5, 4.0))
    psi0 = np.zeros(P.psi_shape())
    psi0[1:-1, 1:-1] = 0.05
    out = {}
    for pattern in ("wavefront", "gpu-wavefront"):
        with plugged.open(to_oracle(P), P.dt, pattern=pattern, abs_tol=1e-13, max_its=100000, reflect=reflect,
                          periodic=periodic) as h:
            out[pattern] = h.idc_steps(psi0, P.source, P.dt, 2, 3, 2, si_abs_tol=1e-13)
    assert rel_err(out["gpu-wavefront"], out["wavefront"]) < 1e-11


@pytest.mark.gpu
def test_reference_source_iteration_at_dg_degree_3_through_plugin(plugged):
    """The reference's SISolver::Solve at DG degree 3 (its sweep on the GPU's elimination kernel)."""
    P = random_problem(9, 8, 3, 4, seed=63, dt=0.3, inflow=True, sigma_range=(0.5, 4.0))
    out = {}
    for pattern in ("wavefront", "gpu-wavefront"):
        with plugged.open(to_oracle(P), P.dt, pattern=pattern, abs_tol=1e-12, max_its=5000) as h:
            psi = h.source_iteration(P.source, P.dt)
            out[pattern] = h.pmv(psi)
    assert rel_err(out["gpu-wavefront"], out["wavefront"]) < 1e-11
