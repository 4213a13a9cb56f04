"""ctypes bindings to the two CPU oracles.  TEST INFRASTRUCTURE ONLY.

* ``Restatement`` -> oracle/_build/liboracle.so, the plain-C restatement (sweep_oracle.c).
* ``Reference``   -> oracle/_ref/libidcref.so, the reference solver compiled from its own sources
  by oracle/Makefile.ref with the driver oracle/ref_driver.cpp.  Present only where the reference
  tree was available at build time (it travels with the repository snapshot once built).
  ``Reference(REFERENCE_GPU_SO)`` is the same reference with the GPU sweep pattern plugged in
  (oracle/sweep_pattern_gpu.cpp, pattern "gpu-wavefront"), linked against libidcsweep.so.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "liboracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libidcref.so")
REFERENCE_GPU_SO = os.path.join(HERE, "_ref", "libidcref_gpu.so")

_dp = C.POINTER(C.c_double)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


@dataclass
class Problem:
    """A 2-D problem on the reference's halo-padded layouts (see sweep_oracle.h)."""

    nx: int
    ny: int
    p: int
    xi: np.ndarray
    eta: np.ndarray
    w: np.ndarray
    quad: np.ndarray           # int64[5]
    sigma_t: np.ndarray        # (nx+2)*(ny+2)
    sigma_s: np.ndarray        # (nx+2)*(ny+2)
    ax: float = 0.0
    bx: float = 1.0
    ay: float = 0.0
    by: float = 1.0

    @property
    def nq(self) -> int:
        return int(self.xi.size)

    @property
    def N(self) -> int:
        return (self.p + 1) ** 2

    @property
    def dx(self) -> float:
        return (self.bx - self.ax) / self.nx

    @property
    def dy(self) -> float:
        return (self.by - self.ay) / self.ny

    def psi_shape(self):
        return (self.nx + 2, self.ny + 2, self.nq, self.p + 1, self.p + 1)

    def phi_shape(self):
        return (self.nx + 2, self.ny + 2, self.p + 1, self.p + 1)


class _Grid(C.Structure):
    _fields_ = [("nx", C.c_int64), ("ny", C.c_int64), ("dx", C.c_double), ("dy", C.c_double),
                ("p", C.c_int64), ("nq", C.c_int64), ("xi", _dp), ("eta", _dp), ("w", _dp),
                ("quad", C.c_int64 * 5)]


class Restatement:
    """The plain-C restatement of the reference's sweep and operators."""

    def __init__(self, so_path: str = RESTATEMENT_SO):
        if not os.path.exists(so_path):
            raise FileNotFoundError(f"{so_path} missing: run `make -C oracle`")
        lib = C.CDLL(so_path)
        g = C.POINTER(_Grid)
        lib.oracle_sweep.argtypes = [g, _dp, C.c_double, _dp]
        lib.oracle_sweep_adjoint.argtypes = [g, _dp, C.c_double, _dp]
        lib.oracle_pmv.argtypes = [g, C.c_double, C.c_double, _dp, _dp]
        lib.oracle_smv.argtypes = [g, C.c_double, C.c_double, _dp, _dp, _dp]
        lib.oracle_lmv.argtypes = [g, C.c_double, C.c_double, _dp, _dp, _dp]
        lib.oracle_si.argtypes = [g, _dp, _dp, C.c_double, C.c_double, C.c_int64, _dp, _dp]
        lib.oracle_si.restype = C.c_int64
        self.lib = lib

    def _grid(self, P: Problem):
        self._keep = (np.ascontiguousarray(P.xi, np.float64), np.ascontiguousarray(P.eta, np.float64),
                      np.ascontiguousarray(P.w, np.float64))
        gr = _Grid(P.nx, P.ny, P.dx, P.dy, P.p, P.nq, _p(self._keep[0]), _p(self._keep[1]),
                   _p(self._keep[2]), (C.c_int64 * 5)(*[int(v) for v in P.quad]))
        return C.byref(gr), gr

    def sweep(self, P: Problem, source: np.ndarray, dt: float = np.inf) -> np.ndarray:
        psi = np.ascontiguousarray(source, np.float64).copy()
        g, _k = self._grid(P)
        rc = self.lib.oracle_sweep(g, _p(P.sigma_t), dt, _p(psi))
        assert rc == 0
        return psi

    def sweep_adjoint(self, P: Problem, source: np.ndarray, dt: float = np.inf) -> np.ndarray:
        psi = np.ascontiguousarray(source, np.float64).copy()
        g, _k = self._grid(P)
        rc = self.lib.oracle_sweep_adjoint(g, _p(P.sigma_t), dt, _p(psi))
        assert rc == 0
        return psi

    def pmv(self, P: Problem, psi: np.ndarray, phi: np.ndarray | None = None, alpha=1.0, beta=0.0):
        phi = np.zeros(P.phi_shape()) if phi is None else np.ascontiguousarray(phi, np.float64).copy()
        g, _k = self._grid(P)
        self.lib.oracle_pmv(g, alpha, beta, _p(np.ascontiguousarray(psi, np.float64)), _p(phi))
        return phi

    def smv(self, P: Problem, phi: np.ndarray, psi: np.ndarray, alpha=1.0, beta=1.0):
        out = np.ascontiguousarray(psi, np.float64).copy()
        g, _k = self._grid(P)
        self.lib.oracle_smv(g, alpha, beta, _p(P.sigma_s), _p(np.ascontiguousarray(phi, np.float64)), _p(out))
        return out

    def lmv(self, P: Problem, x: np.ndarray, y: np.ndarray | None = None, alpha=1.0, beta=0.0):
        out = np.zeros(P.psi_shape()) if y is None else np.ascontiguousarray(y, np.float64).copy()
        g, _k = self._grid(P)
        self.lib.oracle_lmv(g, alpha, beta, _p(P.sigma_t), _p(np.ascontiguousarray(x, np.float64)), _p(out))
        return out

    def source_iteration(self, P: Problem, source: np.ndarray, dt=np.inf, abs_tol=1e-10, max_its=500):
        psi = np.ascontiguousarray(source, np.float64).copy()
        err = C.c_double()
        g, _k = self._grid(P)
        its = self.lib.oracle_si(g, _p(P.sigma_t), _p(P.sigma_s), dt, abs_tol, max_its, _p(psi), C.byref(err))
        return psi, int(its), float(err.value)


class Reference:
    """The reference solver's own routines, compiled from its sources (oracle/Makefile.ref)."""

    def __init__(self, so_path: str = REFERENCE_SO):
        if not os.path.exists(so_path):
            raise FileNotFoundError(f"{so_path} missing: run `make -f oracle/Makefile.ref`")
        lib = C.CDLL(so_path)
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_int64, C.c_int64, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_char_p,
                                   C.c_double, C.c_int64]
        lib.ref_create_reflecting.restype = C.c_void_p
        lib.ref_create_reflecting.argtypes = lib.ref_create.argtypes + [C.c_int]
        lib.ref_create_ex.restype = C.c_void_p
        lib.ref_create_ex.argtypes = lib.ref_create.argtypes + [C.c_int, C.c_int, C.c_int]
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_apply.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
        lib.ref_apply_timed.argtypes = [C.c_void_p, _dp, C.c_double, C.c_int64, _dp]
        lib.ref_pmv.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp]
        lib.ref_smv.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp]
        lib.ref_lmv.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp]
        lib.ref_si_solve.argtypes = [C.c_void_p, _dp, C.c_double, C.POINTER(C.c_int64), _dp]
        lib.ref_write_sd.argtypes = [C.c_void_p, _dp, C.c_char_p]
        lib.ref_write_af.argtypes = [C.c_void_p, _dp, C.c_char_p]
        lib.ref_idc_steps.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_int64, C.c_int64, C.c_int64, C.c_double,
                                      C.c_int64]
        for f in ("ref_apply", "ref_apply_timed", "ref_pmv", "ref_smv", "ref_lmv", "ref_si_solve", "ref_write_sd",
                  "ref_write_af", "ref_idc_steps"):
            getattr(lib, f).restype = C.c_int
        self.lib = lib

    def open(self, P: Problem, dt: float = np.inf, pattern: str = "wavefront", abs_tol=1e-10, max_its=500,
             reflect: int = 0, sigma_degree: int = 0, periodic: bool = False):
        """reflect: the reflecting edges as the reference's BoundaryEdge bits (X_Min 1, X_Max 2, Y_Min 4,
        Y_Max 8); with any, the reference sweeps the quadrants in sequence and reflects between them.
        sigma_degree: 0, or p when P.sigma_t / P.sigma_s hold (p+1)^2 Legendre moments per cell.
        periodic: the reference's Global::periodic (halos synchronised from the opposite edges)."""
        keep = [np.ascontiguousarray(a, np.float64) for a in (P.xi, P.eta, P.w, P.sigma_t, P.sigma_s)]
        h = self.lib.ref_create_ex(P.nx, P.ny, P.ax, P.bx, P.ay, P.by, P.p, P.nq, *[_p(a) for a in keep],
                                   dt, pattern.encode(), abs_tol, max_its, int(reflect), int(sigma_degree),
                                   1 if periodic else 0)
        if not h:
            raise RuntimeError("ref_create failed")
        return _RefHandle(self.lib, h, P, keep)


class _RefHandle:
    def __init__(self, lib, h, P, keep):
        self.lib, self.h, self.P, self._keep = lib, h, P, keep

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def sweep(self, source: np.ndarray, dt: float = np.inf) -> np.ndarray:
        psi = np.ascontiguousarray(source, np.float64).copy()
        sec = C.c_double()
        assert self.lib.ref_apply(self.h, _p(psi), dt, C.byref(sec)) == 0
        return psi

    def time_sweeps(self, source: np.ndarray, dt: float, reps: int) -> float:
        src = np.ascontiguousarray(source, np.float64)
        sec = C.c_double()
        assert self.lib.ref_apply_timed(self.h, _p(src), dt, reps, C.byref(sec)) == 0
        return float(sec.value)

    def pmv(self, psi, phi=None, alpha=1.0, beta=0.0):
        phi = np.zeros(self.P.phi_shape()) if phi is None else np.ascontiguousarray(phi, np.float64).copy()
        assert self.lib.ref_pmv(self.h, alpha, beta, _p(np.ascontiguousarray(psi, np.float64)), _p(phi)) == 0
        return phi

    def smv(self, phi, psi, alpha=1.0, beta=1.0):
        out = np.ascontiguousarray(psi, np.float64).copy()
        assert self.lib.ref_smv(self.h, alpha, beta, _p(np.ascontiguousarray(phi, np.float64)), _p(out)) == 0
        return out

    def lmv(self, x, y=None, alpha=1.0, beta=0.0):
        out = np.zeros(self.P.psi_shape()) if y is None else np.ascontiguousarray(y, np.float64).copy()
        assert self.lib.ref_lmv(self.h, alpha, beta, _p(np.ascontiguousarray(x, np.float64)), _p(out)) == 0
        return out

    def write_sd(self, phi, path: str):
        """The reference's DensityFunction::WriteToDisk of phi (halo layout)."""
        assert self.lib.ref_write_sd(self.h, _p(np.ascontiguousarray(phi, np.float64)), path.encode()) == 0

    def write_af(self, psi, path: str):
        """The reference's OrdinateFlux::WriteToDisk of psi (halo layout)."""
        assert self.lib.ref_write_af(self.h, _p(np.ascontiguousarray(psi, np.float64)), path.encode()) == 0

    def idc_steps(self, psi0, source, dt, steps, num_nodes=4, num_corrections=3, si_abs_tol=1e-14,
                  si_max_its=100000):
        """psi after `steps` steps of the reference's IDCIntegrator (non-hybrid update form, Gauss-Lobatto
        nodes, source-iteration substeps to si_abs_tol); ghost cells of the result are zero."""
        psi = np.ascontiguousarray(psi0, np.float64).copy()
        src = np.ascontiguousarray(source, np.float64)
        assert self.lib.ref_idc_steps(self.h, _p(psi), _p(src), float(dt), int(steps), int(num_nodes),
                                      int(num_corrections), float(si_abs_tol), int(si_max_its)) == 0
        return psi

    def source_iteration(self, source, dt=np.inf):
        psi = np.ascontiguousarray(source, np.float64).copy()
        its = C.c_int64()
        sec = C.c_double()
        assert self.lib.ref_si_solve(self.h, _p(psi), dt, C.byref(its), C.byref(sec)) == 0
        return psi


def reference_available() -> bool:
    return os.path.exists(REFERENCE_SO)
