"""The C ABI library loads on a CPU-only machine and exports include/mfp_spmv.h."""
import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from matrix_format_performance_b200 import _capi
from matrix_format_performance_b200._capi import MfpError, call


def header_functions():
    src = (ROOT / "include" / "mfp_spmv.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"^\s*(?:int|uint32_t|const char \*)\s*(mfp_\w+)\s*\(", src, flags=re.M))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = _capi.load()
    names = header_functions()
    assert len(names) > 50
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(_capi.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mfp_\w+)", out))
    assert set(names) <= exported


def test_python_binding_declares_every_header_function():
    assert set(header_functions()) == set(_capi.declared_symbols())


def test_library_is_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", str(_capi.LIB_PATH)], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_version_and_status_strings():
    lib = _capi.load()
    assert lib.mfp_version() == 100
    assert lib.mfp_status_string(0) == b"success"
    assert lib.mfp_status_string(6) == b"device wait gave up"


def test_invalid_arguments_are_reported_without_gpu():
    with pytest.raises(MfpError, match="plan output is NULL"):
        call("mfp_csr_plan_create", 1, 1, 0, None, 0, None, None)
    rp = np.array([0, 2, 1], np.uint32)
    h = C.c_void_p()
    with pytest.raises(MfpError, match="decreases"):
        call("mfp_csr_plan_create", 2, 2, 1, C.c_void_p(rp.ctypes.data), 0, None, C.byref(h))
    with pytest.raises(MfpError, match="unknown CSR algorithm"):
        call("mfp_csr_plan_create", 2, 2, 1, C.c_void_p(rp.ctypes.data), 7, None, C.byref(h))
    n = C.c_size_t()
    call("mfp_coo_workspace_bytes", 10, 5000, C.byref(n))
    assert n.value == 16 + 20 * 24  # a header, then 24 bytes per 256-element warp tile


def test_device_converters_check_arguments_without_gpu():
    """The on-device converters reject bad arguments before any CUDA call."""
    with pytest.raises(MfpError, match="bad value type"):
        call("mfp_dev_ell_from_csr", 7, 1, None, None, None, 1, None, None, None)
    with pytest.raises(MfpError, match="bad value type"):
        call("mfp_dev_csr_from_coo", 9, 1, 1, 0, None, None, None, None, None, None, None)
    with pytest.raises(MfpError, match="bad value type"):
        call("mfp_dev_scoo_sort_cols", 4, 1, 1, 1, 0, None, None, None, None)
    with pytest.raises(MfpError, match="null"):
        call("mfp_dev_rows_statistics", 4, None, None, None)
    with pytest.raises(MfpError, match="bad format or value type"):
        call("mfp_matrix_create_device", 11, 0, 1, 1, 0, None, None, None, None, C.byref(C.c_void_p()))
    rp = np.array([0, 1], np.uint32)
    with pytest.raises(MfpError, match="slice_size 0"):
        call("mfp_dev_scoo_from_csr", 0, 1, 1, C.c_void_p(rp.ctypes.data), None, None,
             C.byref(_capi.ScooParams(4, 0, 1)), None, None, None, C.c_void_p(rp.ctypes.data), None)


def test_host_scoo_sort_cols_checks_arguments():
    with pytest.raises(MfpError, match="null slices_ptr"):
        call("mfp_scoo_sort_cols_f32", 1, None, None, None, None)
