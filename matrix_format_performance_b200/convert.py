"""On-device format conversion over torch CUDA tensors (mfp_dev_* in the C ABI).

The same layouts as the host converters in formats.py (the reference's
common/matrix_converter.cpp and common/scoo_matrix_class.cpp), built by the
engine's CUDA kernels from device arrays, so a matrix uploaded once as CSR (or
as COO triplets) becomes every other format without a host round trip.
Index arrays are int32 tensors holding the reference's unsigned ids.
"""
from __future__ import annotations

import ctypes as C

from . import _capi
from ._capi import call
from .device import _dptr, _stream

_VT_TORCH = {"torch.float32": 0, "torch.float64": 1}


def _vt(t) -> int:
    return _VT_TORCH[str(t.dtype)]


def _p(t):
    return _dptr(t) if t is not None and t.numel() else C.c_void_p(None)


def rows_statistics(row_ptr, stream=None) -> _capi.RowsStatistic:
    """get_rows_statistics (matrix_converter.cpp:95-127) of a device row_ptr."""
    s = _capi.RowsStatistic()
    call("mfp_dev_rows_statistics", row_ptr.numel() - 1, _dptr(row_ptr), C.byref(s), _stream(stream))
    return s


def check_csr(row_ptr, columns, cols: int, stream=None) -> None:
    call("mfp_dev_check_csr", row_ptr.numel() - 1, cols, columns.numel(), _dptr(row_ptr), _p(columns), _stream(stream))


def coo_count(row_ptr, element_start: int = 0, stream=None) -> int:
    n = C.c_uint32()
    call("mfp_dev_coo_count", row_ptr.numel() - 1, _dptr(row_ptr), element_start, C.byref(n), _stream(stream))
    return n.value


def coo_from_csr(row_ptr, columns, data, element_start: int = 0, stream=None):
    """coo_matrix_class (matrix_converter.cpp:211-280) -> (data, cols, rows)."""
    import torch
    n = coo_count(row_ptr, element_start, stream)
    od = torch.empty(n, dtype=data.dtype, device=data.device)
    oc = torch.empty(n, dtype=torch.int32, device=data.device)
    orow = torch.empty(n, dtype=torch.int32, device=data.device)
    call("mfp_dev_coo_from_csr", _vt(data), row_ptr.numel() - 1, _dptr(row_ptr), _p(columns), _p(data), element_start,
         _p(od), _p(oc), _p(orow), _stream(stream))
    return od, oc, orow


def ell_from_csr(row_ptr, columns, data, width: int | None = None, stream=None):
    """ell_matrix_class (matrix_converter.cpp:139-203) -> (data, columns, width),
    column-major [slot * rows + row]; width None = the longest row."""
    import torch
    rows = row_ptr.numel() - 1
    if width is None:
        width = rows_statistics(row_ptr, stream).max_elements_in_rows if rows else 0
    ed = torch.empty(rows * width, dtype=data.dtype, device=data.device)
    ec = torch.empty(rows * width, dtype=torch.int32, device=data.device)
    call("mfp_dev_ell_from_csr", _vt(data), rows, _dptr(row_ptr), _p(columns), _p(data), width, _p(ed), _p(ec),
         _stream(stream))
    return ed, ec, width


def scoo_from_csr(row_ptr, columns, data, params: _capi.ScooParams, stream=None):
    """scoo_matrix_class (scoo_matrix_class.cpp:58-139) -> (values, c_index, r_index, slices_ptr)."""
    import torch
    nnz = columns.numel()
    ov = torch.empty(nnz, dtype=data.dtype, device=data.device)
    oc = torch.empty(nnz, dtype=torch.int32, device=data.device)
    orow = torch.empty(nnz, dtype=torch.int32, device=data.device)
    sp = torch.empty(params.slices_count + 1, dtype=torch.int32, device=data.device)
    call("mfp_dev_scoo_from_csr", _vt(data), row_ptr.numel() - 1, nnz, _dptr(row_ptr), _p(columns), _p(data),
         C.byref(params), _p(ov), _p(oc), _p(orow), _dptr(sp), _stream(stream))
    return ov, oc, orow, sp


def scoo_sort_cols(values, c_index, r_index, rows: int, cols: int, slice_size: int, stream=None) -> None:
    """The sort_cols layout (scoo_matrix_class.cpp:102-138, stable) of device SCOO arrays, in place."""
    call("mfp_dev_scoo_sort_cols", _vt(values), rows, cols, slice_size, values.numel(), _p(values), _p(c_index),
         _p(r_index), _stream(stream))


def hybrid_from_csr(row_ptr, columns, data, width: int, stream=None):
    """hybrid_matrix_class::allocate (matrix_converter.cpp:296-310) at a given
    ELL width -> ((ell_data, ell_columns), (coo_data, coo_cols, coo_rows))."""
    ed, ec, _ = ell_from_csr(row_ptr, columns, data, width, stream)
    return (ed, ec), coo_from_csr(row_ptr, columns, data, width, stream)


def hybrid_width(row_ptr, percent: float, stream=None) -> int:
    """ELL width of hybrid_matrix_class::allocate: avg + (max - avg) * percent."""
    s = rows_statistics(row_ptr, stream)
    return int(s.avg_elements_in_rows + (s.max_elements_in_rows - s.avg_elements_in_rows) * percent)


def csr_from_coo(rows: int, cols: int, row_ids, col_ids, values, dtype=None, stream=None):
    """csr_matrix_class from COO triplets (matrix_converter.cpp:15-87) -> (row_ptr, columns, data).
    values are FP64 like the reference's get_dbl_data(); dtype float32 / float64."""
    import torch
    dtype = dtype or torch.float32
    nnz = row_ids.numel()
    rp = torch.empty(rows + 1, dtype=torch.int32, device=row_ids.device)
    co = torch.empty(nnz, dtype=torch.int32, device=row_ids.device)
    d = torch.empty(nnz, dtype=dtype, device=row_ids.device)
    call("mfp_dev_csr_from_coo", _VT_TORCH[str(dtype)], rows, cols, nnz, _p(row_ids), _p(col_ids), _p(values),
         _dptr(rp), _p(co), _p(d), _stream(stream))
    return rp, co, d


def scratch_bytes() -> int:
    """Bytes the converters' scratch pool holds on the current device."""
    n = C.c_uint64()
    call("mfp_dev_scratch_bytes", C.byref(n))
    return n.value


def release_scratch() -> None:
    """Waits for the device and returns the converters' unused scratch to the driver."""
    call("mfp_dev_scratch_release")
