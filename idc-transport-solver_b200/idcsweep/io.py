"""The reference's .sd2 (scalar flux) and .af2 (angular flux) binary files, through libidcsweep's C ABI
(idc_read_sd2 / idc_write_sd2 / idc_read_af2 / idc_write_af2; host only, no GPU needed).  Arrays are on
the halo layouts: phi (nx+2, ny+2, P, P), psi (nx+2, ny+2, nq, P, P)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .abi import load_library

_i64p = C.POINTER(C.c_int64)
_dp = C.POINTER(C.c_double)


def _lib():
    lib = load_library()
    if not getattr(lib, "_io_bound", False):
        lib.idc_write_sd2.argtypes = [C.c_char_p, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_int64, _dp]
        lib.idc_read_sd2.argtypes = [C.c_char_p, _i64p, _i64p, _dp, _dp, _dp, _dp, _i64p, _dp, C.c_int64, _i64p]
        lib.idc_write_af2.argtypes = [C.c_char_p, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_char_p, C.c_int64, C.c_int64, C.c_int64, _dp]
        lib.idc_read_af2.argtypes = [C.c_char_p, _i64p, _i64p, _dp, _dp, _dp, _dp, C.c_char_p, C.c_int64, _i64p, _i64p,
                                     _dp, C.c_int64, _i64p]
        lib._io_bound = True
    return lib


@dataclass
class Header:
    nx: int
    ny: int
    ax: float
    bx: float
    ay: float
    by: float
    dg_degree: int
    count: int
    ordinate_type: str = ""
    ang_order: int = 0


def _ptr(a):
    return a.ctypes.data_as(_dp)


def write_sd2(path: str, phi: np.ndarray, ax: float, bx: float, ay: float, by: float) -> None:
    phi = np.ascontiguousarray(phi, np.float64)
    nx, ny, P = phi.shape[0] - 2, phi.shape[1] - 2, phi.shape[2]
    rc = _lib().idc_write_sd2(path.encode(), nx, ny, ax, bx, ay, by, P - 1, _ptr(phi))
    if rc != 0:
        raise OSError(f"idc_write_sd2 failed for {path}")


def read_sd2(path: str):
    """Returns (Header, phi)."""
    v = [C.c_int64() for _ in range(4)]
    d = [C.c_double() for _ in range(4)]
    lib = _lib()
    args = (path.encode(), C.byref(v[0]), C.byref(v[1]), C.byref(d[0]), C.byref(d[1]), C.byref(d[2]), C.byref(d[3]),
            C.byref(v[2]))
    if lib.idc_read_sd2(*args, None, 0, C.byref(v[3])) != 0:
        raise OSError(f"not a readable .sd2 file: {path}")
    h = Header(v[0].value, v[1].value, d[0].value, d[1].value, d[2].value, d[3].value, v[2].value, v[3].value)
    P = h.dg_degree + 1
    phi = np.empty((h.nx + 2, h.ny + 2, P, P))
    if lib.idc_read_sd2(*args, _ptr(phi), phi.size, C.byref(v[3])) != 0:
        raise OSError(f"truncated .sd2 file: {path}")
    return h, phi


def write_af2(path: str, psi: np.ndarray, ax: float, bx: float, ay: float, by: float, ordinate_type: str,
              ang_order: int) -> None:
    psi = np.ascontiguousarray(psi, np.float64)
    nx, ny, nq, P = psi.shape[0] - 2, psi.shape[1] - 2, psi.shape[2], psi.shape[3]
    rc = _lib().idc_write_af2(path.encode(), nx, ny, ax, bx, ay, by, ordinate_type.encode(), int(ang_order), P - 1,
                              nq, _ptr(psi))
    if rc != 0:
        raise OSError(f"idc_write_af2 failed for {path}")


def read_af2(path: str):
    """Returns (Header, psi)."""
    v = [C.c_int64() for _ in range(5)]
    d = [C.c_double() for _ in range(4)]
    name = C.create_string_buffer(4096)
    lib = _lib()
    args = (path.encode(), C.byref(v[0]), C.byref(v[1]), C.byref(d[0]), C.byref(d[1]), C.byref(d[2]), C.byref(d[3]),
            name, 4096, C.byref(v[2]), C.byref(v[3]))
    if lib.idc_read_af2(*args, None, 0, C.byref(v[4])) != 0:
        raise OSError(f"not a readable .af2 file: {path}")
    h = Header(v[0].value, v[1].value, d[0].value, d[1].value, d[2].value, d[3].value, v[3].value, v[4].value,
               name.value.decode(), v[2].value)
    P = h.dg_degree + 1
    nq = h.count // ((h.nx + 2) * (h.ny + 2) * P * P)
    psi = np.empty((h.nx + 2, h.ny + 2, nq, P, P))
    if lib.idc_read_af2(*args, _ptr(psi), psi.size, C.byref(v[4])) != 0:
        raise OSError(f"truncated .af2 file: {path}")
    return h, psi
