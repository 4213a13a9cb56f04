#!/usr/bin/env python
"""Benchmark: sweep unknowns/s of the B200 transport sweep on the 256x256, Q2 (9 dofs/cell), S16
(144 ordinates) heterogeneous steady problem (log-normal sigma_t, median 1, log-sd 1; scattering
ratio U[0.5, 0.999]; unit isotropic source; seeded synthetic data).

One step = one application of L^{-1} (Omega.grad + sigma_t)^{-1} to the problem's angular source: the
out-of-place sweep source -> psi with the scalar flux phi = P psi fused in, on HBM-resident arrays.
The headline `value` is the fastest sweep that meets the 1e-8 relative accuracy bound in phi: the FP64
sweep (FP32 cell solves with FP64 refinement, timed beside it as `fp32_refined`, is slower on B200:
the refinement lengthens the cell-to-cell chain of a latency-bound wavefront).  Each precision runs
with the tile shape the library's autotuner picks for this problem (idc_autotune), chosen before the
timed region.  `e2e` times K such steps through the C ABI on pinned HOST buffers
(idc_sweep_out_many: every step uploads its source and downloads psi and phi inside the timed region;
the copies of neighbouring steps overlap the sweeps on separate streams).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference solver's own CPU sweep (SweepOperator::Apply, compiled from the
reference's sources into oracle/_ref/libidcref.so) on all host cores, same workload and metric.
Under torchrun (N > 1) the ranks split the one problem by ordinates (each sweeps a slice of every
quadrant's ordinates; one NCCL all-reduce of the moments per step; strong scaling), or with --mode replicas
every rank sweeps its own independent problem (seed = rank; no collective, weak scaling); rank 0 prints the
line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "idc-transport-solver_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

P_DEG, SN = 2, 16
NX = 256
METRIC = "sweep unknowns/s"
UNIT = "unknowns/s"
WORKLOAD = "256x256 Q2 S16 log-normal steady sweep (FP64)"
FALLBACK_HBM_GBS = 6650.0


def problem(seed: int, nx: int | None = None):
    from idcsweep.problems import lognormal
    return lognormal(nx or NX, P_DEG, SN, seed=seed, median=1.0, log_sd=1.0, c_range=(0.5, 0.999), source="uniform")


def algorithmic_bytes(P) -> int:
    """Per launch: read the FP64 angular source and write FP64 psi (16 B per unknown), read sigma_t and
    write the N phi moments once per cell."""
    cells = P.nx * P.ny
    return 16 * P.unknowns_per_sweep + cells * (8 + 8 * P.N)


def hbm_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def measured_traffic(nx):
    """dram read+write bytes per launch of the headline (FP64) sweep kernel from the committed ncu
    summary, for the workload size it was scaled to (None for other sizes)."""
    path = os.path.join(REPO, "profiles", "sweep_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        if int(d.get("workload_nx", NX)) != nx or d.get("precision", "fp64") != "fp64":
            return None
        return float(d["dram_bytes_per_launch"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        if not getattr(self, "lines", None):
            return None
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def emit(d):
    print(json.dumps(d), flush=True)


def bench_config(P, world: int) -> dict:
    """The workload description both arms print (the same keys and values for the same problem)."""
    return {"workload": WORKLOAD if P.nx == NX else WORKLOAD.replace("256x256", f"{P.nx}x{P.nx}"),
            "nx": P.nx, "ny": P.ny, "p": P_DEG, "nq": P.nq, "unknowns_per_step": P.unknowns_per_sweep,
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "l2": "inputs larger than L2 (source 690 MB, psi 690 MB per step); no flush"}


# ----------------------------------------------------------------------------------------------------
# reference arm: the reference's own CPU sweep
# ----------------------------------------------------------------------------------------------------

def time_reference_cpu(P, reps: int, warmup: int = 1):
    """SweepOperator::Apply of the reference (oracle/_ref), OpenMP on all host cores: `warmup` untimed
    sweeps (the first gives the oracle result), then `reps` timed ones.  Returns (seconds per sweep,
    threads, phi of the oracle result)."""
    from oracle.bindings import Problem as OP, Reference
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    ref = Reference()
    o = OP(P.nx, P.ny, P.p, P.xi, P.eta, P.w, P.quad, P.sigma_t, P.sigma_s, P.ax, P.bx, P.ay, P.by)
    with ref.open(o, P.dt) as h:
        psi = h.sweep(P.source, P.dt)
        for _ in range(max(0, warmup - 1)):
            h.sweep(P.source, P.dt)
        sec = h.time_sweeps(P.source, P.dt, reps)
        phi = h.pmv(psi)
    return sec / reps, int(os.environ.get("OMP_NUM_THREADS", threads)), phi


def config0_against_reference(abi, torch, dev):
    """The reference's own CPU-runnable case: 64x64 lattice on [0,7]^2, Q1, S8, one implicit-Euler step of
    dt = 0.01 from zero flux, source iteration to 1e-10 (absolute l2 of phi changes, SISolver's rule).  The
    GPU's idc_source_iteration against the reference's SISolver::Solve (oracle/_ref) on all host cores,
    same inputs; phi compared."""
    from idcsweep.problems import lattice
    from oracle.bindings import Problem as OP, Reference
    P = lattice(64, 1, 8, dt=0.01)
    out = {"workload": "64x64 Q1 S8 lattice, one implicit-Euler step dt 0.01, source iteration to 1e-10"}
    with _ctx_for(abi, P, dev) as c:
        for rep in range(2):   # the first builds the schedule
            psi = torch.from_numpy(P.source).to(f"cuda:{dev}")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            its, change = c.source_iteration(psi.data_ptr(), P.dt, abs_tol=1e-10, max_its=5000, loc=abi.LOC_DEVICE)
            torch.cuda.synchronize()
            sec = time.perf_counter() - t0
        phi = torch.zeros(P.phi_shape(), dtype=torch.float64, device=f"cuda:{dev}")
        c.pmv(1.0, 0.0, psi.data_ptr(), phi.data_ptr(), loc=abi.LOC_DEVICE)
        gphi = phi.cpu().numpy()
    out["gpu"] = {"ms": sec * 1e3, "iterations": its, "last_change": change}
    threads = os.cpu_count() or 1
    o = OP(P.nx, P.ny, P.p, P.xi, P.eta, P.w, P.quad, P.sigma_t, P.sigma_s, P.ax, P.bx, P.ay, P.by)
    with Reference().open(o, P.dt, abs_tol=1e-10, max_its=5000) as h:
        h.source_iteration(P.source, P.dt)   # warm-up
        t0 = time.perf_counter()
        rpsi = h.source_iteration(P.source, P.dt)
        rsec = time.perf_counter() - t0
        rphi = h.pmv(rpsi)
    out["reference_cpu"] = {"ms": rsec * 1e3, "threads": int(os.environ.get("OMP_NUM_THREADS", threads))}
    out["speedup"] = rsec / sec
    out["phi_rel_diff"] = float(np.abs(gphi - rphi).max() / np.abs(rphi).max())
    return out


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        # torchrun sets OMP_NUM_THREADS=1 for every rank; the other ranks exit without work, so rank 0 takes
        # every core this process may run on (set before the reference library, and its OpenMP, is loaded)
        os.environ["OMP_NUM_THREADS"] = str(len(os.sched_getaffinity(0)))
    P = problem(0, args.nx)
    steps = max(1, args.steps)
    warm = max(1, args.warmup)
    t0 = time.time()
    sec, threads, _ = time_reference_cpu(P, steps, warm)
    value = P.unknowns_per_sweep / sec
    # the same config as the GPU arm at this N: one problem split by ordinates (strong) or one per GPU (weak)
    cfg = bench_config(P, args.gpus)
    scaling = "weak"
    if args.gpus > 1 and args.mode == "partitioned":
        cfg["parallelism"] = f"ordinates{args.gpus}"
        scaling = "strong"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": scaling,
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "reference_path": "SweepOperator::Apply (wavefront pattern, Gaussian-elimination cell solves), FP64, "
                          "OpenMP on all host cores",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{steps} full sweeps of the workload after {warm} warm-up sweep(s)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.time() - t0,
    }
    emit(line)
    return 0


# ----------------------------------------------------------------------------------------------------
# the other configurations, measured beside the headline (rank 0, one GPU)
# ----------------------------------------------------------------------------------------------------

def _ctx_for(abi, P, dev):
    c = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by, device=dev)
    c.set_ordinates(P.xi, P.eta, P.w, P.quad)
    c.set_sigma(P.sigma_t, P.sigma_s)
    return c


def extra_gmres_dsa(abi, torch, dev):
    """256x256 Q2 S16 log-normal steady problem, GMRES(30) + DSA to 1e-10: FP64 sweeps, per-cell refined FP32
    sweeps, and FP32 Krylov sweeps inside FP64 iterative refinement of the solve (error against the FP64 solve
    stated); then the Krylov iterations' moments-only sweep alone in FP64 and FP32."""
    P = problem(0)
    out = {"workload": "256x256 Q2 S16 log-normal steady, GMRES(30)+DSA(30 CG steps), abs tol 1e-10"}
    sols = {}
    for name, prec in (("fp64", abi.PREC_FP64), ("fp32_refined", abi.PREC_FP32_REFINED),
                       ("fp32_krylov_fp64_refinement", abi.PREC_FP32_IR)):
        with _ctx_for(abi, P, dev) as c:
            c.set_preconditioner(abi.PRECOND_DSA, 30)
            d = torch.from_numpy(P.source).to(f"cuda:{dev}")
            c.gmres_solve(d.data_ptr(), P.dt, abs_tol=1e-10, restart=30, max_its=3000, precision=prec,
                          loc=abi.LOC_DEVICE)   # warm-up (schedules, buffers)
            d = torch.from_numpy(P.source).to(f"cuda:{dev}")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            its, res = c.gmres_solve(d.data_ptr(), P.dt, abs_tol=1e-10, restart=30, max_its=3000, precision=prec,
                                     loc=abi.LOC_DEVICE)
            torch.cuda.synchronize()
            out[name] = {"iterations": its, "residual": res, "ms": (time.perf_counter() - t0) * 1e3}
            sols[name] = d.cpu().numpy()
    for name in ("fp32_refined", "fp32_krylov_fp64_refinement"):
        out[name]["psi_rel_diff_vs_fp64"] = float(np.abs(sols[name] - sols["fp64"]).max() / np.abs(sols["fp64"]).max())
    out["speedup_fp32_krylov_fp64_refinement_vs_fp64"] = out["fp64"]["ms"] / out["fp32_krylov_fp64_refinement"]["ms"]
    # the Krylov iterations' moments-only sweep alone (no source, psi not stored), FP64 against FP32
    with _ctx_for(abi, P, dev) as c:
        x = torch.from_numpy(np.random.default_rng(1).uniform(0.1, 1.0, P.phi_shape())).to(f"cuda:{dev}")
        ph = torch.zeros_like(x)
        sweeps = {}
        for name, prec in (("fp64", abi.PREC_FP64), ("fp32", abi.PREC_FP32)):
            ms = []
            for rep in range(8):
                c.sweep_fused(None, None, P.dt, x.data_ptr(), 1.0, ph.data_ptr(), prec)
                ms.append(c.last_timing()[0])
            sweeps[name] = {"kernel_ms": min(ms[3:]), "phi": ph.clone()}
        out["moments_only_sweep"] = {
            "fp64_kernel_ms": sweeps["fp64"]["kernel_ms"], "fp32_kernel_ms": sweeps["fp32"]["kernel_ms"],
            "speedup_fp32_vs_fp64": sweeps["fp64"]["kernel_ms"] / sweeps["fp32"]["kernel_ms"],
            "err_phi_fp32_vs_fp64": float(((sweeps["fp32"]["phi"] - sweeps["fp64"]["phi"]).abs().max() /
                                           sweeps["fp64"]["phi"].abs().max()).item())}
    return out


def extra_idc(abi, torch, dev, steps=10):
    """512x512 Q1 S12 lattice, IMEX-IDC (4 Gauss-Lobatto nodes, 3 corrections), dt = 0.005, one CUDA graph
    per step; `steps` of the configuration's 100 steps are timed."""
    from idcsweep.problems import lattice
    P = lattice(512, 1, 12, dt=0.005)
    out = {"workload": f"512x512 Q1 S12 lattice, IMEX-IDC 4 nodes 3 corrections, dt 0.005, {steps} steps timed"}
    with _ctx_for(abi, P, dev) as c:
        psi = torch.zeros(P.psi_shape(), dtype=torch.float64, device=f"cuda:{dev}")
        src = torch.from_numpy(P.source).to(f"cuda:{dev}")
        for name, prec in (("fp64", abi.PREC_FP64), ("fp32_refined", abi.PREC_FP32_REFINED)):
            # the autotuner times plain sweeps; the library's default picks the IMEX sweeps' kernel by grid size
            # (512^2 at Q1: the lane kernel, 8-wide segments), so FP64 keeps it
            if prec == abi.PREC_FP64:
                c.set_tile_shape(0, 0)
                out.setdefault("tile_shape", {})[name] = "default (IMEX at Q1 512^2: lane, seg 8)"
            else:
                out.setdefault("tile_shape", {})[name] = c.autotune(src.data_ptr(), P.dt, prec)
            c.idc_integrate(psi.data_ptr(), src.data_ptr(), P.dt, 2, 4, 3, abi.SCATTER_EXPLICIT, prec, use_graph=True,
                            loc=abi.LOC_DEVICE)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sw = c.idc_integrate(psi.data_ptr(), src.data_ptr(), P.dt, steps, 4, 3, abi.SCATTER_EXPLICIT, prec,
                                 use_graph=True, loc=abi.LOC_DEVICE)
            torch.cuda.synchronize()
            sec = time.perf_counter() - t0
            out[name] = {"ms_per_step": sec * 1e3 / steps, "sweeps": sw,
                         "sweep_unknowns_per_s": sw * P.unknowns_per_sweep / sec}
    return out


def extra_adjoint(abi, torch, dev):
    """128x128 Q1 S8, log-normal sigma_t (median 2, log-sd 0.7), c = 0.9, Gaussian source at the left third,
    detector = scalar flux over a 16x16 window at the right third: gradients of all 3 nx ny per-cell
    parameters (sigma_t, sigma_s, source) from one adjoint solve (GMRES with the transposed DSA)."""
    from idcsweep.problems import detector_window, lognormal
    P = lognormal(128, 1, 8, seed=0, median=2.0, log_sd=0.7, c_fixed=0.9, source="gaussian")
    c_det = torch.from_numpy(detector_window(P, cells=16)).to(f"cuda:{dev}")
    out = {"workload": "128x128 Q1 S8 log-normal (median 2, log-sd 0.7), c = 0.9, Gaussian source, 16x16 detector; "
                       "adjoint GMRES(30) + transposed DSA (20 CG steps), abs tol 1e-12",
           "gradient_entries": 3 * P.nx * P.ny}
    with _ctx_for(abi, P, dev) as c:
        psi = torch.from_numpy(P.source).to(f"cuda:{dev}")
        c.set_preconditioner(abi.PRECOND_DSA, 30)   # forward DSA; the adjoint uses its transpose
        c.gmres_solve(psi.data_ptr(), P.dt, abs_tol=1e-12, restart=30, max_its=3000, loc=abi.LOC_DEVICE)
        c.set_preconditioner(abi.PRECOND_DSA, 20)   # 20 inner CG steps: the fastest adjoint solve here
        g_t = torch.zeros((P.nx + 2) * (P.ny + 2), dtype=torch.float64, device=f"cuda:{dev}")
        g_s = torch.zeros_like(g_t)
        g_q = torch.zeros(P.phi_shape(), dtype=torch.float64, device=f"cuda:{dev}")
        for name, prec in (("fp64", abi.PREC_FP64), ("fp32_refined", abi.PREC_FP32_REFINED)):
            args = (psi.data_ptr(), c_det.data_ptr(), g_t.data_ptr(), g_s.data_ptr(), g_q.data_ptr())
            c.adjoint_grad(*args, dt=P.dt, abs_tol=1e-12, precision=prec, loc=abi.LOC_DEVICE)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            its, res = c.adjoint_grad(*args, dt=P.dt, abs_tol=1e-12, precision=prec, loc=abi.LOC_DEVICE)
            torch.cuda.synchronize()
            sec = time.perf_counter() - t0
            out[name] = {"grads_per_s": 3 * P.nx * P.ny / sec, "ms": sec * 1e3, "adjoint_iterations": its}
    return out


def extra_adjoint_transient(abi, torch, dev, steps=10, dt=0.5, every=0):
    """The same 128x128 Q1 S8 problem, time dependent: gradients of the detector response after 10
    implicit-Euler steps of dt = 0.5 from zero flux with respect to all per-cell sigma_t, sigma_s, source
    moments (and the initial angular flux), by the checkpointed backward adjoint (states every ~sqrt(10)
    steps, recomputed per segment).  grads_per_s counts the 3 nx ny per-cell parameters, as the steady line."""
    from idcsweep.problems import detector_window, lognormal
    P = lognormal(128, 1, 8, seed=0, median=2.0, log_sd=0.7, c_fixed=0.9, source="gaussian")
    d = f"cuda:{dev}"
    c_det = torch.from_numpy(detector_window(P, cells=16)).to(d)
    src = torch.from_numpy(P.source).to(d)
    psi0 = torch.zeros_like(src)
    out = {"workload": f"128x128 Q1 S8 as the adjoint line, {steps} implicit-Euler steps of dt {dt} from zero "
                       "flux; GMRES(30) + DSA (20 CG steps) forward and adjoint, abs tol 1e-12",
           "gradient_entries": 3 * P.nx * P.ny, "initial_flux_entries": int(np.prod(P.psi_shape()))}
    with _ctx_for(abi, P, dev) as c:
        c.set_preconditioner(abi.PRECOND_DSA, 20)
        g_t = torch.zeros((P.nx + 2) * (P.ny + 2), dtype=torch.float64, device=d)
        g_s = torch.zeros_like(g_t)
        g_q = torch.zeros(P.phi_shape(), dtype=torch.float64, device=d)
        g_p = torch.zeros_like(src)
        args = (psi0.data_ptr(), src.data_ptr(), c_det.data_ptr(), dt, steps)
        kw = dict(checkpoint_every=every, dsigma_t=g_t.data_ptr(), dsigma_s=g_s.data_ptr(), dsource=g_q.data_ptr(),
                  dpsi0=g_p.data_ptr(), abs_tol=1e-12, loc=abi.LOC_DEVICE)
        c.adjoint_transient(*args, **kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J, solves = c.adjoint_transient(*args, **kw)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        out["fp64"] = {"grads_per_s": out["gradient_entries"] / sec, "ms": sec * 1e3, "gmres_solves": solves,
                       "J": J}
    return out


def extra_adjoint_idc(abi, torch, dev, steps=4, dt=0.5, nodes=4, corrections=3, every=0):
    """The same 128x128 Q1 S8 problem with IDC time stepping (4 Gauss-Lobatto nodes, 3 corrections, implicit
    scattering: every substep a GMRES + DSA solve): gradients of the detector response after 4 steps of
    dt = 0.5 from zero flux through the correction sweeps (idc_adjoint_idc), checkpointed."""
    from idcsweep.problems import detector_window, lognormal
    P = lognormal(128, 1, 8, seed=0, median=2.0, log_sd=0.7, c_fixed=0.9, source="gaussian")
    d = f"cuda:{dev}"
    c_det = torch.from_numpy(detector_window(P, cells=16)).to(d)
    src = torch.from_numpy(P.source).to(d)
    psi0 = torch.zeros_like(src)
    out = {"workload": f"128x128 Q1 S8 as the adjoint line, {steps} IDC steps ({nodes} Gauss-Lobatto nodes, "
                       f"{corrections} corrections, implicit scattering) of dt {dt} from zero flux; GMRES(30) + DSA "
                       "(20 CG steps) forward and adjoint, abs tol 1e-12",
           "gradient_entries": 3 * P.nx * P.ny}
    with _ctx_for(abi, P, dev) as c:
        c.set_preconditioner(abi.PRECOND_DSA, 20)
        g_t = torch.zeros((P.nx + 2) * (P.ny + 2), dtype=torch.float64, device=d)
        g_s = torch.zeros_like(g_t)
        g_q = torch.zeros(P.phi_shape(), dtype=torch.float64, device=d)
        g_p = torch.zeros_like(src)
        args = (psi0.data_ptr(), src.data_ptr(), c_det.data_ptr(), dt, steps, nodes, corrections)
        kw = dict(checkpoint_every=every, dsigma_t=g_t.data_ptr(), dsigma_s=g_s.data_ptr(), dsource=g_q.data_ptr(),
                  dpsi0=g_p.data_ptr(), abs_tol=1e-12, loc=abi.LOC_DEVICE)
        c.adjoint_idc(*args, **kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J, solves = c.adjoint_idc(*args, **kw)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        out["fp64"] = {"grads_per_s": out["gradient_entries"] / sec, "ms": sec * 1e3, "gmres_solves": solves,
                       "J": J}
    return out


def extra_batched(abi, torch, dev, n_problems=64):
    """64 independent steady problems: side U{32,...,384}, S4/S8/S12/S16, Q1/Q2, log-normal sigma_t (median 1,
    log-sd 1), c U[0.3, 0.99] (seeded); one sweep of every problem, batched (one launch per DG degree,
    autotuned tile shapes) against one problem at a time with the default FP64 sweep."""
    from idcsweep.quadrature import level_symmetric_2d
    rng = np.random.default_rng(2024)
    ctxs, srcs, outs, phis, unknowns = [], [], [], [], 0
    try:
        for _ in range(n_problems):
            n = int(rng.choice(np.arange(32, 385, 32)))
            sn = int(rng.choice([4, 8, 12, 16]))
            p = int(rng.choice([1, 2]))
            st = np.zeros((n + 2, n + 2))
            st[1:-1, 1:-1] = np.exp(rng.standard_normal((n, n)))
            ss = np.zeros_like(st)
            ss[1:-1, 1:-1] = rng.uniform(0.3, 0.99, (n, n)) * st[1:-1, 1:-1]
            xi, eta, w, q = level_symmetric_2d(sn)
            c = abi.SweepContext(n, n, p, 0.0, 7.0, 0.0, 7.0, device=dev)
            c.set_ordinates(xi, eta, w, q)
            c.set_sigma(st.ravel().copy(), ss.ravel().copy())
            s_ = torch.zeros((n + 2, n + 2, xi.size, p + 1, p + 1), dtype=torch.float64, device=f"cuda:{dev}")
            s_[1:-1, 1:-1, :, 0, 0] = 1.0 / (4 * math.pi)
            ctxs.append(c)
            srcs.append(s_)
            outs.append(torch.zeros_like(s_))
            phis.append(torch.zeros((n + 2, n + 2, p + 1, p + 1), dtype=torch.float64, device=f"cuda:{dev}"))
            unknowns += n * n * xi.size * (p + 1) ** 2
        for _ in range(2):
            one = 0.0
            for k, c in enumerate(ctxs):
                c.sweep_out(srcs[k].data_ptr(), outs[k].data_ptr(), math.inf, phis[k].data_ptr(), abi.PREC_FP64,
                            loc=abi.LOC_DEVICE)
                one += c.last_timing()[0]
        with abi.Batch() as b:
            for c in ctxs:
                b.add(c)
            S, O, F = [x.data_ptr() for x in srcs], [x.data_ptr() for x in outs], [x.data_ptr() for x in phis]
            for _ in range(2):
                b.sweep(S, O, F, math.inf, abi.PREC_FP64)
            default_ms = min((b.sweep(S, O, F, math.inf, abi.PREC_FP64), b.last_ms())[1] for _ in range(3))
            default_shapes = {f"dg{p}": list(b.get_shape(p, abi.PREC_FP64)) for p in (1, 2)}
            b.autotune(S, O, math.inf, abi.PREC_FP64)
            res = {"fp64_default_shapes": {"device_ms": default_ms, "shapes_seg_warps": default_shapes},
                   "fp64_shapes_seg_warps": {f"dg{p}": list(b.get_shape(p, abi.PREC_FP64)) for p in (1, 2)}}
            for name, prec in (("fp64", abi.PREC_FP64), ("fp32_refined", abi.PREC_FP32_REFINED)):
                for _ in range(2):
                    b.sweep(S, O, F, math.inf, prec)
                best = min((b.sweep(S, O, F, math.inf, prec), b.last_ms())[1] for _ in range(3))
                res[name] = {"device_ms": best, "unknowns_per_s": unknowns / (best * 1e-3),
                             "hbm_frac_of_measured": 16.0 * unknowns / (best * 1e-3) / 1e9 / hbm_peak()[0]}
            # GMRES + DSA (20 CG steps) to 1e-8 on every problem: one at a time, then batched (one batched sweep per
            # Krylov step for all unconverged problems)
            for c in ctxs:
                c.set_preconditioner(abi.PRECOND_DSA, 20)
            sizes = [int(np.prod(s_.shape)) // (s_.shape[0] * s_.shape[1]) * (s_.shape[0] - 2) * (s_.shape[1] - 2)
                     for s_ in srcs]
            work = [x.clone() for x in srcs]
            for k, c in enumerate(ctxs):   # warm-up (buffers, schedules)
                c.gmres_solve(work[k].data_ptr(), math.inf, abs_tol=1e-8, restart=30, max_its=3000,
                              loc=abi.LOC_DEVICE)
            work = [x.clone() for x in srcs]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            single_its = []
            for k, c in enumerate(ctxs):
                single_its.append(c.gmres_solve(work[k].data_ptr(), math.inf, abs_tol=1e-8, restart=30, max_its=3000,
                                                loc=abi.LOC_DEVICE)[0])
            torch.cuda.synchronize()
            single_s = time.perf_counter() - t0
            single_psi = work
            work = [x.clone() for x in srcs]
            b.gmres_solve([x.data_ptr() for x in work], math.inf, abs_tol=1e-8, restart=30, max_its=3000)   # warm-up
            work = [x.clone() for x in srcs]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            batch_its, batch_res = b.gmres_solve([x.data_ptr() for x in work], math.inf, abs_tol=1e-8, restart=30,
                                                 max_its=3000)
            torch.cuda.synchronize()
            batch_s = time.perf_counter() - t0
            diff = max(float(((work[k] - single_psi[k]).abs().max() / single_psi[k].abs().max()).item())
                       for k in range(len(ctxs)))
            sweeps_single = sum((i + 2) * u for i, u in zip(single_its, sizes))
            sweeps_batch = sum((i + 2) * u for i, u in zip(batch_its, sizes))
            solves = {"workload": "GMRES(30) + DSA (20 CG steps) to 1e-8 on every problem, FP64",
                      "one_at_a_time": {"ms": single_s * 1e3, "krylov_iterations": int(sum(single_its)),
                                        "sweep_unknowns_per_s": sweeps_single / single_s},
                      "batched": {"ms": batch_s * 1e3, "krylov_iterations": int(sum(batch_its)),
                                  "max_iterations": int(max(batch_its)),
                                  "sweep_unknowns_per_s": sweeps_batch / batch_s},
                      "speedup": single_s / batch_s, "psi_rel_diff_batched_vs_single": diff}
        return {"workload": f"{n_problems} independent steady problems, sides 32..384, S4..S16, Q1/Q2",
                "unknowns_per_sweep": unknowns, "one_at_a_time_fp64": {"device_ms": one,
                                                                      "unknowns_per_s": unknowns / (one * 1e-3)},
                "batched_autotuned": res, "speedup_fp64": one / res["fp64"]["device_ms"],
                "gmres_dsa_solves": solves}
    finally:
        for c in ctxs:
            c.close()


# ----------------------------------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------------------------------

def run_partitioned(args):
    """One problem (the workload) split by ordinates over the ranks: every rank sweeps a balanced slice of each
    quadrant's ordinates of the whole grid (its own context, source slice and psi slice resident on its GPU)
    and one all-reduce (sum, NCCL) of the partial moments per step completes phi -- the path's only exchange.
    `value` = the whole problem's unknowns / the slowest rank's time per step (strong scaling).  `e2e` adds,
    on every rank, the upload of its source slice and the download of its psi slice and of phi."""
    import datetime
    import torch
    import torch.distributed as tdist
    from idcsweep import abi
    from idcsweep.distributed import local_quadrature, partition_ordinates

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    P = problem(0, args.nx)
    idx = partition_ordinates(P.quad, world, rank)
    xi, eta, w, q = local_quadrature(P.xi, P.eta, P.w, P.quad, idx)
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by, device=dev)
    ctx.set_ordinates(xi, eta, w, q)
    ctx.set_sigma(P.sigma_t, P.sigma_s)
    h_src = np.ascontiguousarray(P.source[:, :, idx])
    src = torch.from_numpy(h_src).to(f"cuda:{dev}")
    out = torch.empty_like(src)
    phi = torch.zeros(P.phi_shape(), dtype=torch.float64, device=f"cuda:{dev}")
    shape = (0, 0) if args.no_autotune else ctx.autotune(src.data_ptr(), P.dt, abi.PREC_FP64)
    ctx.set_tile_shape(*shape)

    counted = [0]

    def step():
        ctx.sweep_out(src.data_ptr(), out.data_ptr(), P.dt, phi.data_ptr(), abi.PREC_FP64, loc=abi.LOC_DEVICE)
        counted[0] += ctx.last_timing()[1]
        tdist.all_reduce(phi)   # on torch's current stream, after the (synchronous) sweep returned

    def time_steps(fn, steps):
        torch.cuda.synchronize()
        tdist.barrier()
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        tdist.barrier()
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1) / steps], device=f"cuda:{dev}")
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        return float(t.item())

    warm = max(3, args.warmup)
    for _ in range(warm):
        step()
    clocks = ClockSampler(dev) if rank == 0 else None
    if clocks:
        clocks.__enter__()
    counted[0] = 0
    ms = time_steps(step, args.steps)
    launches = counted[0]
    if clocks:
        clocks.__exit__()
    kernel_ms = ctx.last_timing()[0]

    # end to end: this rank's host slice in, its psi slice and phi out, every step
    hs = torch.from_numpy(h_src).pin_memory()
    ho = torch.empty_like(hs).pin_memory()
    hp = torch.zeros(P.phi_shape(), dtype=torch.float64).pin_memory()

    def e2e_step():
        src.copy_(hs, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        step()
        ho.copy_(out, non_blocking=True)
        hp.copy_(phi, non_blocking=True)

    e2e_step()
    e2e_ms = None if args.no_e2e else time_steps(e2e_step, max(2, args.steps))
    phi_host = phi.cpu().numpy()
    tdist.barrier()
    ctx.close()
    if rank == 0:
        unknowns = P.unknowns_per_sweep
        alg = algorithmic_bytes(P)
        peak, peak_kind = hbm_peak()
        cfg = bench_config(P, world)
        cfg["parallelism"] = f"ordinates{world}"
        emit({
            "metric": METRIC, "value": unknowns / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": cfg, "tile_shape": {"fp64": list(shape)},
            "roofline": {"bound": "hbm", "achieved": alg / world / (kernel_ms * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": alg / world / (kernel_ms * 1e-3) / 1e9 / peak, "traffic": None,
                         "algorithmic_bytes_per_rank": alg / world, "kernel_ms": kernel_ms, "peak_kind": peak_kind},
            "e2e": None if e2e_ms is None else {
                "value": unknowns / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h_src.nbytes) * world,
                "d2h_bytes_per_step": int(h_src.nbytes + phi_host.nbytes) * world, "ms_per_step": e2e_ms},
            "gpu_launches": launches, "clocks": clocks.summary() if clocks else None,
            "exchange": "one NCCL all-reduce (sum) of phi per step, %d bytes" % phi_host.nbytes})
    tdist.destroy_process_group()
    return 0


def run_ours(args):
    import torch
    from idcsweep import abi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)

    P = problem(rank, args.nx)
    ctx = abi.SweepContext(P.nx, P.ny, P.p, P.ax, P.bx, P.ay, P.by, device=dev)
    ctx.set_ordinates(P.xi, P.eta, P.w, P.quad)
    ctx.set_sigma(P.sigma_t, P.sigma_s)

    src = torch.from_numpy(P.source).to(f"cuda:{dev}")
    out = torch.empty_like(src)
    phi = torch.zeros(P.phi_shape(), dtype=torch.float64, device=f"cuda:{dev}")

    def barrier():
        if dist is not None:
            dist.barrier()

    shapes = {}

    def timed(prec, steps, warmup, sampler=False):
        if prec not in shapes:   # the library's autotuner: a tile shape per precision, outside the timing
            shapes[prec] = (tuple(args.tile) if args.tile else (0, 0) if args.no_autotune else
                            ctx.autotune(src.data_ptr(), P.dt, prec))
        ctx.set_tile_shape(*shapes[prec])
        for _ in range(warmup):
            ctx.sweep_out(src.data_ptr(), out.data_ptr(), P.dt, phi.data_ptr(), prec, loc=abi.LOC_DEVICE)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        kernel_ms, launches = [], 0
        stream = torch.cuda.current_stream()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks = ClockSampler(dev) if sampler else None
        if clocks:
            clocks.__enter__()
        ev0.record(stream)
        for _ in range(steps):
            # each call is synchronous (it checks the device error word), so host wall time and events
            # on the current stream bracket exactly the K sweeps
            ctx.sweep_out(src.data_ptr(), out.data_ptr(), P.dt, phi.data_ptr(), prec, loc=abi.LOC_DEVICE)
            ms, n = ctx.last_timing()
            kernel_ms.append(ms)
            launches += n
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.__exit__()
        total_ms = ev0.elapsed_time(ev1)
        if dist is not None:
            t = torch.tensor([total_ms], device=f"cuda:{dev}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        return total_ms / steps, statistics.mean(kernel_ms), launches, (clocks.summary() if clocks else None)

    warm = max(3, args.warmup)
    ms32 = k32 = msf = kf = phi32 = phif = None
    if not args.fp64_only:
        ms32, k32, _, _ = timed(abi.PREC_FP32_REFINED, args.steps, warm)
        phi32 = phi.clone()
        msf, kf, _, _ = timed(abi.PREC_FP32, args.steps, warm)   # unrefined FP32 arithmetic (about 1e-7)
        phif = phi.clone()
    ms64, k64, launches, clocks = timed(abi.PREC_FP64, args.steps, warm, sampler=(rank == 0))
    phi64 = phi.clone()

    # end to end through the C ABI with pinned host buffers
    h_src = torch.from_numpy(P.source).pin_memory()
    h_out = torch.empty_like(h_src).pin_memory()
    h_phi = torch.zeros(P.phi_shape(), dtype=torch.float64).pin_memory()
    hs, ho, hp = h_src.numpy(), h_out.numpy(), h_phi.numpy()
    e2e_s, e2e_phi_err = float("nan"), None
    if not args.no_e2e:
        e2e_steps = max(2, args.steps)
        ctx.sweep_out_many([hs] * 2, [ho] * 2, [hp] * 2, P.dt, abi.PREC_FP64)   # buffers and streams
        barrier()
        t0 = time.perf_counter()
        ctx.sweep_out_many([hs] * e2e_steps, [ho] * e2e_steps, [hp] * e2e_steps, P.dt, abi.PREC_FP64)
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        if dist is not None:
            t = torch.tensor([e2e_s], device=f"cuda:{dev}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e_phi_err = float(np.abs(hp - phi64.cpu().numpy()).max() / np.abs(hp).max())

    unknowns = P.unknowns_per_sweep
    alg = algorithmic_bytes(P)
    peak, peak_kind = hbm_peak()
    traffic = measured_traffic(P.nx)
    err_fp32_vs_fp64 = None if phi32 is None else float(((phi32 - phi64).abs().max() / phi64.abs().max()).item())

    if rank != 0:
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    line = {
        "metric": METRIC,
        "value": world * unknowns / (ms64 * 1e-3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": warm,
        "ms_per_step": ms64,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(P, world),
        "tile_shape": {name: list(shapes[p]) for name, p in (("fp64", abi.PREC_FP64),
                                                             ("fp32_refined", abi.PREC_FP32_REFINED),
                                                             ("fp32", abi.PREC_FP32)) if p in shapes},
        "roofline": {"bound": "hbm", "achieved": alg / (k64 * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (k64 * 1e-3) / 1e9 / peak, "traffic": traffic,
                     "algorithmic_bytes": alg, "kernel_ms": k64, "peak_kind": peak_kind},
        "fp32_refined": None if ms32 is None else {
            "value": world * unknowns / (ms32 * 1e-3), "ms_per_step": ms32, "kernel_ms": k32,
            "roofline_frac": alg / (k32 * 1e-3) / 1e9 / peak},
        "speedup_fp32_refined_vs_fp64": None if ms32 is None else ms64 / ms32,
        "err_phi_fp32_refined_vs_fp64_gpu": err_fp32_vs_fp64,
        "fp32": None if msf is None else {
            "value": world * unknowns / (msf * 1e-3), "ms_per_step": msf, "kernel_ms": kf,
            "speedup_vs_fp64": ms64 / msf,
            "err_phi_vs_fp64_gpu": float(((phif - phi64).abs().max() / phi64.abs().max()).item())},
        "e2e": None if args.no_e2e else {
            "value": world * unknowns / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(hs.nbytes),
            "d2h_bytes_per_step": int(P.nx * P.ny * P.nq * P.N * 8 + hp.nbytes), "ms_per_step": e2e_s * 1e3,
            "phi_rel_diff_vs_device_run": e2e_phi_err},
        "gpu_launches": launches,
        "clocks": clocks,
    }

    if not args.no_extras and world == 1:
        for key, fn in EXTRAS.items():
            try:
                line[key] = fn(abi, torch, dev)
            except Exception as e:   # reported, never fatal for the headline line
                line[key] = {"error": str(e)[:200]}

    if not args.no_cpu_baseline and world == 1:
        try:
            sec, threads, phi_ref = time_reference_cpu(P, args.steps, warm)
            line["cpu_baseline"] = {"value": unknowns / sec, "unit": UNIT, "cores": threads, "kind": "reference",
                                    "sample": f"{args.steps} full sweeps of the workload after {warm} warm-up "
                                              "sweep(s)"}
            scale = np.abs(phi_ref).max()
            line["err_phi_vs_oracle"] = {
                name: float(np.abs(f.cpu().numpy() - phi_ref).max() / scale)
                for name, f in (("fp64", phi64), ("fp32_refined", phi32), ("fp32", phif)) if f is not None}
        except Exception as e:  # the reference library may be absent where it was never built
            line["cpu_baseline"] = None
            line["cpu_baseline_error"] = str(e)[:200]
        try:   # the reference's own small case, solved by both sides
            line["config0_source_iteration"] = config0_against_reference(abi, torch, dev)
        except Exception as e:
            line["config0_source_iteration"] = {"error": str(e)[:200]}
    emit(line)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


EXTRAS = {"gmres_dsa": extra_gmres_dsa, "idc": extra_idc, "adjoint": extra_adjoint,
          "adjoint_transient": extra_adjoint_transient, "adjoint_idc": extra_adjoint_idc, "batched": extra_batched}


def run_only_extra(name):
    """One of the other configurations alone (profiling runs: its launch list without the headline's)."""
    import torch
    from idcsweep import abi
    abi.load_library()
    print(json.dumps({name: EXTRAS[name](abi, torch, 0)}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--mode", choices=("partitioned", "replicas"), default="partitioned",
                    help="more than one GPU (torchrun): one problem split by ordinates with an all-reduce of the "
                         "moments per step (strong scaling, the default), or one independent problem per GPU "
                         "(weak scaling)")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg (profiling runs)")
    ap.add_argument("--nx", type=int, default=NX, help="grid side (default: the benchmark's 256; smaller for ncu)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default tile shapes, no tuning launches (profiling runs)")
    ap.add_argument("--tile", type=lambda v: [int(x) for x in v.split(",")], default=None, metavar="SEG,WARPS",
                    help="one fixed tile shape for every precision, no tuning launches (profiling runs; "
                         "WARPS 0 = the lane kernel)")
    ap.add_argument("--fp64-only", action="store_true",
                    help="time the FP64 sweep alone, without the FP32 legs (profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations (GMRES+DSA, IDC, adjoint, batched) measured beside the headline")
    ap.add_argument("--only-extra", choices=tuple(EXTRAS), default=None,
                    help="run one of the other configurations alone and print its JSON (profiling runs)")
    args = ap.parse_args()
    if args.only_extra:
        return run_only_extra(args.only_extra)
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.mode == "partitioned" and "WORLD_SIZE" in os.environ and int(os.environ["WORLD_SIZE"]) > 1:
        return run_partitioned(args)
    if args.mode == "partitioned" and "WORLD_SIZE" in os.environ and args.gpus == 1 and os.environ.get(
            "IDC_BENCH_PARTITIONED_ONE"):   # the partitioned path on one rank (its code path, checked on one GPU)
        return run_partitioned(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
