"""ctypes binding of the C ABI in include/idcsweep.h (libidcsweep.so).

This is the host-side mirror of the reference's sweep/operator interface for Python callers (tests,
bench).  Arrays are numpy float64 host arrays (``loc=HOST``) or raw device pointers (``loc=DEVICE``,
e.g. ``torch.Tensor.data_ptr()``), always in the reference's halo-padded layouts.

The library is loaded from the package's build directory; if it is missing the import fails loudly
(there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "build", "libidcsweep.so")

IDC_OK = 0
PRECOND_NONE, PRECOND_DSA = 0, 1
SCATTER_EXPLICIT, SCATTER_IMPLICIT = 0, 1
EDGE_X_MIN, EDGE_X_MAX, EDGE_Y_MIN, EDGE_Y_MAX = 1, 2, 4, 8
IDC_ERR_ARG = 1
IDC_ERR_UNSUPPORTED = 2
IDC_ERR_CUDA = 3
IDC_ERR_TIMEOUT = 4
IDC_ERR_NOT_CONVERGED = 5
IDC_ERR_STATE = 6
IDC_ERR_NOMEM = 7

LOC_HOST = 0
LOC_DEVICE = 1

PREC_FP64 = 0
PREC_FP32_REFINED = 1
PREC_FP32 = 2
PREC_FP32_IR = 3          # idc_gmres_solve: FP32 Krylov sweeps inside FP64 iterative refinement

IDC_NOALLOC_MAX_ITEMS = 4096        # include/idcsweep.h
IDC_NOALLOC_MAX_ORDINATES = 1024

# Every symbol include/idcsweep.h declares (checked by tests/test_abi_symbols.py).
EXPORTED_SYMBOLS = (
    "idc_ctx_create", "idc_ctx_destroy", "idc_set_ordinates", "idc_set_sigma", "idc_sweep", "idc_pmv",
    "idc_smv", "idc_lmv", "idc_source_iteration", "idc_strerror", "idc_last_error_message", "idc_last_timing",
    "idc_set_tiling", "idc_sweep_out", "idc_sweep_noalloc", "idc_gmres_solve", "idc_sweep_adjoint",
    "idc_adjoint_grad", "idc_set_preconditioner", "idc_idc_integrate", "idc_write_sd2", "idc_read_sd2",
    "idc_write_af2", "idc_read_af2", "idc_sweep_fused", "idc_set_tile_shape", "idc_autotune", "idc_batch_create",
    "idc_batch_add", "idc_batch_sweep", "idc_batch_autotune", "idc_batch_last_timing", "idc_batch_destroy",
    "idc_batch_set_shape", "idc_batch_get_shape", "idc_sweep_out_many", "idc_adjoint_transient",
    "idc_set_spin_limit", "idc_batch_gmres_solve", "idc_set_allreduce", "idc_adjoint_idc", "idc_lmv_transpose",
    "idc_set_reflecting", "idc_set_periodic",
)


class IdcError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: status {code} ({msg})")
        self.code = code


class ProblemDesc(C.Structure):
    _fields_ = [("nx", C.c_int64), ("ny", C.c_int64), ("ax", C.c_double), ("bx", C.c_double),
                ("ay", C.c_double), ("by", C.c_double), ("dg_degree", C.c_int64), ("sigma_degree", C.c_int64),
                ("device", C.c_int32), ("flags", C.c_int32)]


_dp = C.POINTER(C.c_double)
_lib = None


# int (*)(double *data, int64_t n, void *user): the all-reduce hook of idc_set_allreduce
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_void_p)


def load_library(path: str = LIB_PATH):
    """Loads libidcsweep.so (once) and declares the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built: run __graft_entry__.build() or make -C csrc")
    lib = C.CDLL(path)
    vp = C.c_void_p
    lib.idc_ctx_create.argtypes = [C.POINTER(ProblemDesc), C.POINTER(vp)]
    lib.idc_ctx_destroy.argtypes = [vp]
    lib.idc_set_ordinates.argtypes = [vp, C.c_int64, vp, vp, vp, vp]
    lib.idc_set_sigma.argtypes = [vp, vp, vp, C.c_int]
    lib.idc_sweep.argtypes = [vp, vp, C.c_double, vp, C.c_int, C.c_int]
    lib.idc_pmv.argtypes = [vp, C.c_double, C.c_double, vp, vp, C.c_int]
    lib.idc_smv.argtypes = [vp, C.c_double, C.c_double, vp, vp, C.c_int]
    lib.idc_lmv.argtypes = [vp, C.c_double, C.c_double, vp, vp, C.c_int]
    lib.idc_source_iteration.argtypes = [vp, vp, C.c_double, C.c_double, C.c_int64, C.c_int, C.c_int,
                                         C.POINTER(C.c_int64), _dp]
    lib.idc_strerror.argtypes = [C.c_int]
    lib.idc_strerror.restype = C.c_char_p
    lib.idc_last_error_message.argtypes = []
    lib.idc_last_error_message.restype = C.c_char_p
    lib.idc_last_timing.argtypes = [vp, _dp, C.POINTER(C.c_int64)]
    lib.idc_set_tiling.argtypes = [vp, C.c_int32, C.c_int32]
    lib.idc_set_spin_limit.argtypes = [vp, C.c_int64]
    lib.idc_set_allreduce.argtypes = [vp, ALLREDUCE_FN, vp]
    lib.idc_adjoint_idc.argtypes = [vp, vp, vp, C.c_double, C.c_int64, C.c_int32, C.c_int32, vp, C.c_int64, C.c_double,
                                    C.c_int32, C.c_int64, C.c_int, vp, vp, vp, vp, _dp, C.c_int, C.POINTER(C.c_int64)]
    lib.idc_lmv_transpose.argtypes = [vp, C.c_double, C.c_double, vp, vp, C.c_int]
    lib.idc_set_reflecting.argtypes = [vp, C.c_int32]
    lib.idc_set_periodic.argtypes = [vp, C.c_int32]
    lib.idc_sweep_out.argtypes = [vp, vp, vp, C.c_double, vp, C.c_int, C.c_int]
    lib.idc_sweep_out_many.argtypes = [vp, C.c_int64, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.c_double,
                                       C.c_int, C.c_int]
    lib.idc_sweep_adjoint.argtypes = [vp, vp, vp, C.c_double, vp, C.c_int, C.c_int]
    lib.idc_set_preconditioner.argtypes = [vp, C.c_int, C.c_int32]
    lib.idc_sweep_fused.argtypes = [vp, vp, vp, C.c_double, vp, C.c_double, vp, C.c_int, C.c_int]
    lib.idc_set_tile_shape.argtypes = [vp, C.c_int32, C.c_int32]
    lib.idc_autotune.argtypes = [vp, vp, C.c_double, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.idc_batch_create.argtypes = [C.POINTER(vp)]
    lib.idc_batch_add.argtypes = [vp, vp]
    lib.idc_batch_sweep.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.c_double, C.c_int]
    lib.idc_batch_autotune.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.c_double, C.c_int]
    lib.idc_batch_last_timing.argtypes = [vp, _dp]
    lib.idc_batch_destroy.argtypes = [vp]
    lib.idc_batch_gmres_solve.argtypes = [vp, C.POINTER(vp), C.c_double, C.c_double, C.c_int32, C.c_int64, C.c_int,
                                          C.POINTER(C.c_int64), _dp]
    lib.idc_batch_set_shape.argtypes = [vp, C.c_int, C.c_int, C.c_int32, C.c_int32]
    lib.idc_batch_get_shape.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.idc_idc_integrate.argtypes = [vp, vp, vp, C.c_double, C.c_int64, C.c_int32, C.c_int32, C.c_int, C.c_int,
                                      C.c_double, C.c_int32, C.c_int64, C.c_int, C.c_int, C.POINTER(C.c_int64)]
    lib.idc_adjoint_grad.argtypes = [vp, vp, vp, C.c_double, C.c_double, C.c_int32, C.c_int64, C.c_int, vp, vp, vp,
                                     C.c_int, C.POINTER(C.c_int64), _dp]
    lib.idc_adjoint_transient.argtypes = [vp, vp, vp, C.c_double, C.c_int64, vp, C.c_int64, C.c_double, C.c_int32,
                                          C.c_int64, C.c_int, vp, vp, vp, vp, _dp, C.c_int, C.POINTER(C.c_int64)]
    lib.idc_gmres_solve.argtypes = [vp, vp, C.c_double, C.c_double, C.c_int32, C.c_int64, C.c_int, C.c_int,
                                    C.POINTER(C.c_int64), _dp]
    lib.idc_sweep_noalloc.argtypes = [C.POINTER(ProblemDesc), C.c_int64, vp, vp, vp, vp, vp, vp, vp, C.c_double, vp,
                                      C.c_int, vp]
    for name in EXPORTED_SYMBOLS:
        if name not in ("idc_strerror", "idc_last_error_message"):
            getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def _check(rc: int, where: str):
    if rc != IDC_OK:
        lib = load_library()
        msg = lib.idc_last_error_message().decode(errors="replace")
        raise IdcError(rc, where, msg or lib.idc_strerror(rc).decode())


def _host_ptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("arrays must be C-contiguous float64")
    return C.c_void_p(a.ctypes.data)


def _ptr(a, loc: int):
    if a is None:
        return None
    if loc == LOC_DEVICE:
        return C.c_void_p(int(a))
    return _host_ptr(a)


class SweepContext:
    """One grid on one GPU: the device-side counterpart of SweepOperator<RKDG::OrdinateFlux> plus the
    TransportOperator and SISolver routines that operate on its arrays."""

    def __init__(self, nx: int, ny: int, p: int, ax=0.0, bx=1.0, ay=0.0, by=1.0, device: int = 0,
                 sigma_degree: int = 0):
        """sigma_degree: 0 for one cross-section value per cell, p for (p+1)^2 Legendre moments per cell."""
        lib = load_library()
        self._lib = lib
        self.nx, self.ny, self.p = int(nx), int(ny), int(p)
        self.N = (self.p + 1) ** 2
        desc = ProblemDesc(self.nx, self.ny, ax, bx, ay, by, self.p, int(sigma_degree), device, 0)
        h = C.c_void_p()
        _check(lib.idc_ctx_create(C.byref(desc), C.byref(h)), "idc_ctx_create")
        self._h = h
        self.nq = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.idc_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- configuration --
    def set_ordinates(self, xi, eta, w, quad_bounds):
        self._ord = [np.ascontiguousarray(a, np.float64) for a in (xi, eta, w)]
        self._qb = np.ascontiguousarray(quad_bounds, np.int64)
        _check(self._lib.idc_set_ordinates(self._h, int(self._ord[0].size), *[_host_ptr(a) for a in self._ord],
                                           C.c_void_p(self._qb.ctypes.data)), "idc_set_ordinates")
        self.nq = int(self._ord[0].size)

    def set_sigma(self, sigma_t, sigma_s=None, loc: int = LOC_HOST):
        if loc == LOC_HOST:
            sigma_t = np.ascontiguousarray(sigma_t, np.float64)
            sigma_s = None if sigma_s is None else np.ascontiguousarray(sigma_s, np.float64)
        _check(self._lib.idc_set_sigma(self._h, _ptr(sigma_t, loc), _ptr(sigma_s, loc), loc), "idc_set_sigma")

    def set_tiling(self, ordinates_per_block: int = 0, rows_per_block: int = 0):
        _check(self._lib.idc_set_tiling(self._h, int(ordinates_per_block), int(rows_per_block)), "idc_set_tiling")

    # -- operators --
    def psi_shape(self):
        return (self.nx + 2, self.ny + 2, self.nq, self.p + 1, self.p + 1)

    def phi_shape(self):
        return (self.nx + 2, self.ny + 2, self.p + 1, self.p + 1)

    def sweep(self, psi, dt=np.inf, phi=None, precision=PREC_FP64, loc=LOC_HOST):
        """In place: psi <- L^{-1} psi; phi (if given) <- P psi."""
        _check(self._lib.idc_sweep(self._h, _ptr(psi, loc), float(dt), _ptr(phi, loc), int(precision), loc),
               "idc_sweep")

    def sweep_out(self, source, result, dt=np.inf, phi=None, precision=PREC_FP64, loc=LOC_HOST):
        """result <- L^{-1} source (interior cells); phi (if given) <- P result."""
        _check(self._lib.idc_sweep_out(self._h, _ptr(source, loc), _ptr(result, loc), float(dt), _ptr(phi, loc),
                                       int(precision), loc), "idc_sweep_out")

    def sweep_out_many(self, sources, results, phis=None, dt=np.inf, precision=PREC_FP64, loc=LOC_HOST):
        """results[k] <- L^{-1} sources[k] (interior cells), phis[k] <- P results[k]; on host arrays the
        copies of neighbouring steps overlap the sweeps."""
        n = len(sources)
        arr = lambda xs: (C.c_void_p * n)(*[_ptr(x, loc) for x in xs])
        _check(self._lib.idc_sweep_out_many(self._h, n, arr(sources), arr(results),
                                            None if phis is None else arr(phis), float(dt), int(precision), loc),
               "idc_sweep_out_many")

    def pmv(self, alpha, beta, psi, phi, loc=LOC_HOST):
        _check(self._lib.idc_pmv(self._h, alpha, beta, _ptr(psi, loc), _ptr(phi, loc), loc), "idc_pmv")

    def smv(self, alpha, beta, phi, psi, loc=LOC_HOST):
        _check(self._lib.idc_smv(self._h, alpha, beta, _ptr(phi, loc), _ptr(psi, loc), loc), "idc_smv")

    def lmv(self, alpha, beta, x, y, loc=LOC_HOST):
        _check(self._lib.idc_lmv(self._h, alpha, beta, _ptr(x, loc), _ptr(y, loc), loc), "idc_lmv")

    def source_iteration(self, source, dt=np.inf, abs_tol=1e-10, max_its=500, precision=PREC_FP64, loc=LOC_HOST):
        """In place: source <- psi of the converged source iteration.  Returns (iterations, last change)."""
        its = C.c_int64()
        err = C.c_double()
        _check(self._lib.idc_source_iteration(self._h, _ptr(source, loc), float(dt), float(abs_tol), int(max_its),
                                              int(precision), loc, C.byref(its), C.byref(err)),
               "idc_source_iteration")
        return int(its.value), float(err.value)

    def gmres_solve(self, source, dt=np.inf, abs_tol=1e-8, restart=30, max_its=3000, precision=PREC_FP64,
                    loc=LOC_HOST):
        """In place: source <- psi of the Peierls-form GMRES solve.  Returns (iterations, final residual)."""
        its = C.c_int64()
        res = C.c_double()
        _check(self._lib.idc_gmres_solve(self._h, _ptr(source, loc), float(dt), float(abs_tol), int(restart),
                                         int(max_its), int(precision), loc, C.byref(its), C.byref(res)),
               "idc_gmres_solve")
        return int(its.value), float(res.value)

    def idc_integrate(self, psi, source, dt, steps, num_nodes=4, num_corrections=3, scattering=SCATTER_EXPLICIT,
                      precision=PREC_FP64, abs_tol=1e-12, restart=30, max_its=2000, use_graph=True, loc=LOC_HOST):
        """In place: psi <- psi after `steps` IDC steps of size dt with the constant source.  Returns sweeps."""
        sw = C.c_int64()
        _check(self._lib.idc_idc_integrate(self._h, _ptr(psi, loc), _ptr(source, loc), float(dt), int(steps),
                                           int(num_nodes), int(num_corrections), int(scattering), int(precision),
                                           float(abs_tol), int(restart), int(max_its), int(bool(use_graph)), loc,
                                           C.byref(sw)), "idc_idc_integrate")
        return int(sw.value)

    def sweep_fused(self, source_ptr, result_ptr, dt, phi_scatter_ptr, scatter_scale, phi_ptr, precision=PREC_FP64):
        """Device pointers (int or None): result <- L^{-1}(source + scale S phi_scatter), phi <- P result."""
        v = lambda x: None if x is None else C.c_void_p(int(x))
        _check(self._lib.idc_sweep_fused(self._h, v(source_ptr), v(result_ptr), float(dt), v(phi_scatter_ptr),
                                         float(scatter_scale), v(phi_ptr), int(precision), LOC_DEVICE),
               "idc_sweep_fused")

    def set_tile_shape(self, seg: int, warps: int):
        _check(self._lib.idc_set_tile_shape(self._h, int(seg), int(warps)), "idc_set_tile_shape")

    def autotune(self, source_ptr, dt=np.inf, precision=PREC_FP64):
        """Times every tile shape on this problem (device source pointer); keeps and returns (seg, warps)."""
        sg, wp = C.c_int32(), C.c_int32()
        _check(self._lib.idc_autotune(self._h, C.c_void_p(int(source_ptr)), float(dt), int(precision), C.byref(sg),
                                      C.byref(wp)), "idc_autotune")
        return int(sg.value), int(wp.value)

    def set_preconditioner(self, kind: int, inner_steps: int = 30):
        """Right preconditioner of gmres_solve (and, transposed, of adjoint_grad): PRECOND_NONE or PRECOND_DSA
        (inner_steps CG steps)."""
        _check(self._lib.idc_set_preconditioner(self._h, int(kind), int(inner_steps)), "idc_set_preconditioner")

    def sweep_adjoint(self, source, result, dt=np.inf, moments=None, precision=PREC_FP64, loc=LOC_HOST):
        """result <- L^{-T} source (interior cells, transposed sweep); moments (if given) <- sum_q result_q."""
        _check(self._lib.idc_sweep_adjoint(self._h, _ptr(source, loc), _ptr(result, loc), float(dt),
                                           _ptr(moments, loc), int(precision), loc), "idc_sweep_adjoint")

    def adjoint_grad(self, psi, detector, dsigma_t=None, dsigma_s=None, dsource=None, dt=np.inf, abs_tol=1e-12,
                     restart=30, max_its=3000, precision=PREC_FP64, loc=LOC_HOST):
        """Gradients of J = detector . phi(psi) w.r.t. sigma_t, sigma_s (halo cell layout) and the isotropic
        source moments (phi layout), written into the given arrays.  Returns (iterations, final residual)."""
        its = C.c_int64()
        res = C.c_double()
        _check(self._lib.idc_adjoint_grad(self._h, _ptr(psi, loc), _ptr(detector, loc), float(dt), float(abs_tol),
                                          int(restart), int(max_its), int(precision), _ptr(dsigma_t, loc),
                                          _ptr(dsigma_s, loc), _ptr(dsource, loc), loc, C.byref(its), C.byref(res)),
               "idc_adjoint_grad")
        return int(its.value), float(res.value)

    def adjoint_transient(self, psi0, source, detector, dt, steps, checkpoint_every=0, dsigma_t=None, dsigma_s=None,
                          dsource=None, dpsi0=None, abs_tol=1e-12, restart=30, max_its=3000, precision=PREC_FP64,
                          loc=LOC_HOST):
        """Gradients of J = detector . phi(psi^steps) after `steps` implicit-Euler steps from psi0 with the
        constant source, written into the given arrays (sigma_t, sigma_s: halo cell layout; dsource: phi
        layout; dpsi0: psi layout).  Returns (J, number of forward and adjoint GMRES solves)."""
        jv = C.c_double()
        ns = C.c_int64()
        _check(self._lib.idc_adjoint_transient(self._h, _ptr(psi0, loc), _ptr(source, loc), float(dt), int(steps),
                                               _ptr(detector, loc), int(checkpoint_every), float(abs_tol),
                                               int(restart), int(max_its), int(precision), _ptr(dsigma_t, loc),
                                               _ptr(dsigma_s, loc), _ptr(dsource, loc), _ptr(dpsi0, loc),
                                               C.byref(jv), loc, C.byref(ns)), "idc_adjoint_transient")
        return float(jv.value), int(ns.value)

    def adjoint_idc(self, psi0, source, detector, dt, steps, num_nodes=4, num_corrections=3, checkpoint_every=0,
                    dsigma_t=None, dsigma_s=None, dsource=None, dpsi0=None, abs_tol=1e-12, restart=30, max_its=3000,
                    precision=PREC_FP64, loc=LOC_HOST):
        """Gradients of J = detector . phi(psi^steps) after `steps` implicit-scattering IDC steps (num_nodes
        Gauss-Lobatto nodes, num_corrections corrections) from psi0 with the constant source, written into the
        given arrays.  Returns (J, number of forward and adjoint GMRES solves)."""
        jv = C.c_double()
        ns = C.c_int64()
        _check(self._lib.idc_adjoint_idc(self._h, _ptr(psi0, loc), _ptr(source, loc), float(dt), int(steps),
                                         int(num_nodes), int(num_corrections), _ptr(detector, loc),
                                         int(checkpoint_every), float(abs_tol), int(restart), int(max_its),
                                         int(precision), _ptr(dsigma_t, loc), _ptr(dsigma_s, loc),
                                         _ptr(dsource, loc), _ptr(dpsi0, loc), C.byref(jv), loc, C.byref(ns)),
               "idc_adjoint_idc")
        return float(jv.value), int(ns.value)

    def lmv_transpose(self, alpha, beta, x_ptr, y_ptr):
        """Device pointers: y <- beta y + alpha L^T x (interior cells)."""
        _check(self._lib.idc_lmv_transpose(self._h, float(alpha), float(beta), C.c_void_p(int(x_ptr)),
                                           C.c_void_p(int(y_ptr)), LOC_DEVICE), "idc_lmv_transpose")

    def set_periodic(self, on: bool = True):
        """Periodic boundaries on all four edges (the reference's `periodic` key)."""
        _check(self._lib.idc_set_periodic(self._h, 1 if on else 0), "idc_set_periodic")

    def set_reflecting(self, edges: int = 0):
        """Reflecting edges: EDGE_X_MIN | EDGE_X_MAX | EDGE_Y_MIN | EDGE_Y_MAX (0: none)."""
        _check(self._lib.idc_set_reflecting(self._h, int(edges)), "idc_set_reflecting")

    def set_spin_limit(self, polls: int = 0):
        """Polls before a device-side wait gives up (0: the default)."""
        _check(self._lib.idc_set_spin_limit(self._h, int(polls)), "idc_set_spin_limit")

    def set_allreduce(self, fn=None):
        """fn(ptr, n) -> int sums the n doubles at device address ptr over the ranks in place (0 on success);
        None turns the hook off.  The wrapper is kept alive with the context."""
        if fn is None:
            self._allreduce = None
            _check(self._lib.idc_set_allreduce(self._h, ALLREDUCE_FN(), None), "idc_set_allreduce")
            return

        def tramp(ptr, n, user):
            try:
                return int(fn(int(ptr), int(n)))
            except Exception:   # never let an exception cross the C boundary
                return 1

        self._allreduce = ALLREDUCE_FN(tramp)
        _check(self._lib.idc_set_allreduce(self._h, self._allreduce, None), "idc_set_allreduce")

    def last_timing(self):
        ms = C.c_double()
        n = C.c_int64()
        _check(self._lib.idc_last_timing(self._h, C.byref(ms), C.byref(n)), "idc_last_timing")
        return float(ms.value), int(n.value)


class Batch:
    """Independent problems (SweepContexts on one GPU) swept in one persistent launch per DG degree."""

    def __init__(self):
        self._lib = load_library()
        h = C.c_void_p()
        _check(self._lib.idc_batch_create(C.byref(h)), "idc_batch_create")
        self._h = h
        self._members = []

    def add(self, ctx: "SweepContext"):
        _check(self._lib.idc_batch_add(self._h, ctx._h), "idc_batch_add")
        self._members.append(ctx)

    def _arr(self, ptrs):
        n = len(self._members)
        if ptrs is None:
            return None
        assert len(ptrs) == n
        return (C.c_void_p * n)(*[None if p is None else C.c_void_p(int(p)) for p in ptrs])

    def sweep(self, src_ptrs, out_ptrs, phi_ptrs=None, dt=np.inf, precision=PREC_FP64):
        _check(self._lib.idc_batch_sweep(self._h, self._arr(src_ptrs), self._arr(out_ptrs), self._arr(phi_ptrs),
                                         float(dt), int(precision)), "idc_batch_sweep")

    def gmres_solve(self, psi_ptrs, dt=np.inf, abs_tol=1e-8, restart=30, max_its=3000, precision=PREC_FP64):
        """In place on every member (device pointers, Q in, psi out).  Returns (iterations, residuals) lists."""
        n = len(psi_ptrs)
        its = (C.c_int64 * n)()
        res = (C.c_double * n)()
        _check(self._lib.idc_batch_gmres_solve(self._h, self._arr(psi_ptrs), float(dt), float(abs_tol), int(restart),
                                               int(max_its), int(precision), its, res), "idc_batch_gmres_solve")
        return list(its), list(res)

    def autotune(self, src_ptrs, out_ptrs, dt=np.inf, precision=PREC_FP64):
        _check(self._lib.idc_batch_autotune(self._h, self._arr(src_ptrs), self._arr(out_ptrs), float(dt),
                                            int(precision)), "idc_batch_autotune")

    def set_shape(self, dg_degree: int, precision: int, seg: int, warps: int):
        _check(self._lib.idc_batch_set_shape(self._h, int(dg_degree), int(precision), int(seg), int(warps)),
               "idc_batch_set_shape")

    def get_shape(self, dg_degree: int, precision: int):
        sg, wp = C.c_int32(), C.c_int32()
        _check(self._lib.idc_batch_get_shape(self._h, int(dg_degree), int(precision), C.byref(sg), C.byref(wp)),
               "idc_batch_get_shape")
        return int(sg.value), int(wp.value)

    def last_ms(self) -> float:
        ms = C.c_double()
        _check(self._lib.idc_batch_last_timing(self._h, C.byref(ms)), "idc_batch_last_timing")
        return float(ms.value)

    def close(self):
        if self._h:
            self._lib.idc_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def sweep_noalloc(nx, ny, p, ax, bx, ay, by, xi_ptr, eta_ptr, w_ptr, nq, quad_bounds, sigma_t_ptr, source_ptr,
                  result_ptr, dt=np.inf, phi_ptr=None, precision=PREC_FP64, device=0, stream=None):
    """idc_sweep_noalloc: the allocation-free out-of-place sweep.  Every array argument is a device
    pointer (int) the caller owns; quad_bounds is host data.  Returns the status code."""
    lib = load_library()
    desc = ProblemDesc(int(nx), int(ny), ax, bx, ay, by, int(p), 0, int(device), 0)
    qb = np.ascontiguousarray(quad_bounds, np.int64)
    v = lambda x: None if x is None else C.c_void_p(int(x))
    return lib.idc_sweep_noalloc(C.byref(desc), int(nq), v(xi_ptr), v(eta_ptr), v(w_ptr), C.c_void_p(qb.ctypes.data),
                                 v(sigma_t_ptr), v(source_ptr), v(result_ptr), float(dt), v(phi_ptr), int(precision),
                                 v(stream))
