"""The C-ABI library loads and exports every entry point include/idcsweep.h declares; argument checks
that need no GPU behave like the reference's (errors are status codes, never aborts)."""
import ctypes as C
import os
import re

import pytest

from conftest import REPO, gpu_available
from idcsweep import abi

HEADER = os.path.join(REPO, "include", "idcsweep.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(idc_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_what_the_binding_lists():
    assert declared_functions() == sorted(abi.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = abi.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_strerror_and_null_arguments():
    lib = abi.load_library()
    assert lib.idc_strerror(abi.IDC_OK) == b"ok"
    assert lib.idc_strerror(abi.IDC_ERR_TIMEOUT) == b"device-side wait timed out"
    assert lib.idc_strerror(12345) == b"unknown status"
    assert lib.idc_ctx_create(None, None) == abi.IDC_ERR_ARG
    assert lib.idc_sweep(None, None, 1.0, None, 0, 0) == abi.IDC_ERR_ARG
    assert lib.idc_pmv(None, 1.0, 0.0, None, None, 0) == abi.IDC_ERR_ARG
    assert lib.idc_ctx_destroy(None) == abi.IDC_OK
    assert b"null" in lib.idc_last_error_message()


def test_descriptor_validation_before_device():
    lib = abi.load_library()
    h = C.c_void_p()
    bad = abi.ProblemDesc(0, 4, 0.0, 1.0, 0.0, 1.0, 1, 0, 0, 0)
    assert lib.idc_ctx_create(C.byref(bad), C.byref(h)) == abi.IDC_ERR_ARG
    p4 = abi.ProblemDesc(4, 4, 0.0, 1.0, 0.0, 1.0, 4, 0, 0, 0)   # DG degree <= 3
    assert lib.idc_ctx_create(C.byref(p4), C.byref(h)) == abi.IDC_ERR_UNSUPPORTED
    hi = abi.ProblemDesc(4, 4, 0.0, 1.0, 0.0, 1.0, 1, 2, 0, 0)   # cross sections: degree 0 or the DG degree
    assert lib.idc_ctx_create(C.byref(hi), C.byref(h)) == abi.IDC_ERR_ARG
    empty = abi.ProblemDesc(4, 4, 1.0, 1.0, 0.0, 1.0, 1, 0, 0, 0)
    assert lib.idc_ctx_create(C.byref(empty), C.byref(h)) == abi.IDC_ERR_ARG


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU path")
def test_no_device_is_a_status_not_a_crash():
    lib = abi.load_library()
    h = C.c_void_p()
    ok = abi.ProblemDesc(4, 4, 0.0, 1.0, 0.0, 1.0, 1, 0, 0, 0)
    assert lib.idc_ctx_create(C.byref(ok), C.byref(h)) == abi.IDC_ERR_CUDA
    assert not h.value


def test_solver_entry_points_reject_null_arguments():
    """The solver and adjoint entry points answer a null context or array with IDC_ERR_ARG before they touch
    a device, like the reference's argument checks (no GPU needed)."""
    lib = abi.load_library()
    its, res, jv, ns = C.c_int64(), C.c_double(), C.c_double(), C.c_int64()
    assert lib.idc_gmres_solve(None, None, 1.0, 1e-8, 30, 10, 0, 0, C.byref(its), C.byref(res)) == abi.IDC_ERR_ARG
    assert lib.idc_adjoint_grad(None, None, None, 1.0, 1e-8, 30, 10, 0, None, None, None, 0, C.byref(its),
                                C.byref(res)) == abi.IDC_ERR_ARG
    assert lib.idc_adjoint_transient(None, None, None, 0.1, 3, None, 0, 1e-8, 30, 10, 0, None, None, None, None,
                                     C.byref(jv), 0, C.byref(ns)) == abi.IDC_ERR_ARG
    assert b"null" in lib.idc_last_error_message()


def test_batch_tile_shapes_validated_without_a_device():
    """idc_batch_set_shape: the modal kernel's shapes (seg 4..32, warps 1..7) at any precision, the lane
    kernel's (seg 4, 8 or 16, warps 0) in FP64 only; anything else is IDC_ERR_ARG; 0, 0 restores the default
    (none for a degree without members)."""
    with abi.Batch() as b:
        b.set_shape(1, abi.PREC_FP64, 8, 0)
        assert b.get_shape(1, abi.PREC_FP64) == (8, 0)
        b.set_shape(2, abi.PREC_FP32_REFINED, 32, 5)
        assert b.get_shape(2, abi.PREC_FP32_REFINED) == (32, 5)
        for args in ((1, abi.PREC_FP32_REFINED, 8, 0), (1, abi.PREC_FP64, 32, 0), (1, abi.PREC_FP64, 12, 3),
                     (1, abi.PREC_FP64, 8, 8), (2, abi.PREC_FP64, 16, -1)):
            with pytest.raises(abi.IdcError) as e:
                b.set_shape(*args)
            assert e.value.code == abi.IDC_ERR_ARG
        assert b.get_shape(1, abi.PREC_FP64) == (8, 0)   # a rejected shape leaves the set one
        b.set_shape(1, abi.PREC_FP64, 0, 0)
        assert b.get_shape(1, abi.PREC_FP64) == (0, 0)
