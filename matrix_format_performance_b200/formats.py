"""Host-side layouts with the reference's names, built by the C ABI.

Each class mirrors the reference class of the same name
(common/matrix_converter.h:24-96, common/scoo_matrix_class.h:14-39) and is
filled by the library's bit-exact converters (include/mfp_spmv.h).  Arrays
are numpy; value arrays are float32 or float64 like the reference's two
template instantiations.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import call

_VT = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}
_SFX = {np.dtype(np.float32): "f32", np.dtype(np.float64): "f64"}


def ptr(a: np.ndarray | None):
    """ctypes void* to a contiguous numpy array (None for empty/None)."""
    if a is None or a.size == 0:
        return None
    assert a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


@dataclass
class matrix_class:
    """COO triplets with double values: the reader's matrix_market::matrix_class."""
    rows: int
    cols: int
    row_ids: np.ndarray
    col_ids: np.ndarray
    data: np.ndarray
    storage_scheme: int = 0  # 0 = general

    def __post_init__(self):
        self.row_ids = _u32(self.row_ids)
        self.col_ids = _u32(self.col_ids)
        self.data = np.ascontiguousarray(self.data, dtype=np.float64)

    @property
    def nnz(self) -> int:
        return int(self.data.size)


class csr_matrix_class:
    """csr_matrix_class<T> (matrix_converter.cpp:15-87)."""

    def __init__(self, matrix: matrix_class | None = None, dtype=np.float32):
        self.dtype = np.dtype(dtype)
        if matrix is None:
            return
        self.rows, self.cols, self.nnz = matrix.rows, matrix.cols, matrix.nnz
        self.row_ptr = np.empty(self.rows + 1, np.uint32)
        self.columns = np.empty(self.nnz, np.uint32)
        self.data = np.empty(self.nnz, self.dtype)
        call(f"mfp_csr_from_coo_{_SFX[self.dtype]}", self.rows, self.cols, self.nnz, matrix.storage_scheme,
             ptr(matrix.row_ids), ptr(matrix.col_ids), ptr(matrix.data), ptr(self.row_ptr),
             ptr(self.columns), ptr(self.data))

    @classmethod
    def from_arrays(cls, rows, cols, row_ptr, columns, data, dtype=None):
        m = cls(None, dtype if dtype is not None else np.asarray(data).dtype)
        m.rows, m.cols = int(rows), int(cols)
        m.row_ptr = _u32(row_ptr)
        m.columns = _u32(columns)
        m.data = np.ascontiguousarray(data, dtype=m.dtype)
        m.nnz = int(m.data.size)
        return m

    def astype(self, dtype) -> "csr_matrix_class":
        return csr_matrix_class.from_arrays(self.rows, self.cols, self.row_ptr, self.columns,
                                            self.data.astype(dtype), dtype)

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.row_ptr.astype(np.int64))

    def get_matrix_size(self) -> int:
        return self.nnz


def get_rows_statistics(m: csr_matrix_class) -> _capi.RowsStatistic:
    s = _capi.RowsStatistic()
    call("mfp_get_rows_statistics", m.rows, ptr(m.row_ptr), C.byref(s))
    return s


class ell_matrix_class:
    """ell_matrix_class<T> (matrix_converter.cpp:129-203): column-major, padded."""

    def __init__(self, m: csr_matrix_class, elements_in_rows: int | None = None):
        self.rows, self.cols, self.dtype = m.rows, m.cols, m.dtype
        if elements_in_rows is None:
            w = C.c_uint32()
            call("mfp_ell_width", m.rows, ptr(m.row_ptr), C.byref(w))
            elements_in_rows = w.value
        self.elements_in_rows = int(elements_in_rows)
        n = self.rows * self.elements_in_rows
        self.data = np.empty(n, self.dtype)
        self.columns = np.empty(n, np.uint32)
        call(f"mfp_ell_from_csr_{_SFX[self.dtype]}", m.rows, ptr(m.row_ptr), ptr(m.columns), ptr(m.data),
             self.elements_in_rows, ptr(self.data), ptr(self.columns))

    @staticmethod
    def estimate_size(m: csr_matrix_class) -> int:
        w = C.c_uint32()
        call("mfp_ell_width", m.rows, ptr(m.row_ptr), C.byref(w))
        return int(w.value) * m.rows

    def get_matrix_size(self) -> int:
        return self.rows * self.elements_in_rows


class coo_matrix_class:
    """coo_matrix_class<T> (matrix_converter.cpp:211-280)."""

    def __init__(self, m: csr_matrix_class, element_start: int = 0):
        self.rows, self.cols, self.dtype = m.rows, m.cols, m.dtype
        n = C.c_uint32()
        call("mfp_coo_count", m.rows, ptr(m.row_ptr), element_start, C.byref(n))
        self.elements_count = int(n.value)
        self.data = np.empty(self.elements_count, self.dtype)
        self.cols_ = np.empty(self.elements_count, np.uint32)
        self.rows_ = np.empty(self.elements_count, np.uint32)
        call(f"mfp_coo_from_csr_{_SFX[self.dtype]}", m.rows, ptr(m.row_ptr), ptr(m.columns), ptr(m.data),
             element_start, ptr(self.data), ptr(self.cols_), ptr(self.rows_))

    def get_matrix_size(self) -> int:
        return self.elements_count


class hybrid_matrix_class:
    """hybrid_matrix_class<T> (matrix_converter.cpp:288-310)."""

    def __init__(self, m: csr_matrix_class):
        self.rows, self.cols, self.dtype = m.rows, m.cols, m.dtype
        self.ell_matrix = None
        self.coo_matrix = None

    def allocate(self, m: csr_matrix_class, percent: float) -> None:
        self.allocate_width(m, hybrid_width(m, percent))

    def allocate_width(self, m: csr_matrix_class, width: int) -> None:
        self.ell_matrix = ell_matrix_class(m, int(width))
        self.coo_matrix = coo_matrix_class(m, int(width))


def hybrid_width(m: csr_matrix_class, percent: float) -> int:
    """ELL width of hybrid_matrix_class::allocate: avg + (max - avg) * percent."""
    w = C.c_uint32()
    call("mfp_hybrid_width", m.rows, ptr(m.row_ptr), float(percent), C.byref(w))
    return int(w.value)


def row_length_quantile(m: csr_matrix_class, q: float) -> int:
    w = C.c_uint32()
    call("mfp_row_length_quantile", m.rows, ptr(m.row_ptr), float(q), C.byref(w))
    return int(w.value)


class scoo_matrix_class:
    """scoo_matrix_class<T> (scoo_matrix_class.cpp:58-139).  sort_cols=True applies
    the reference's disabled sort_cols block (:102-138) with a stable sort."""

    def __init__(self, sm_count: int, shared_mem_size: int, m: csr_matrix_class, sort_cols: bool = False):
        self.rows, self.cols, self.dtype, self.nnz = m.rows, m.cols, m.dtype, m.nnz
        p = _capi.ScooParams()
        call("mfp_scoo_params_compute", m.rows, sm_count, shared_mem_size, _VT[self.dtype], C.byref(p))
        self.params = p
        self.slices_count, self.slice_size, self.lane_size = p.slices_count, p.slice_size, p.lane_size
        self.values = np.empty(m.nnz, self.dtype)
        self.c_index = np.empty(m.nnz, np.uint32)
        self.r_index = np.empty(m.nnz, np.uint32)
        self.slices_ptr = np.empty(p.slices_count + 1, np.uint32)
        call(f"mfp_scoo_from_csr_{_SFX[self.dtype]}", m.rows, ptr(m.row_ptr), ptr(m.columns), ptr(m.data),
             C.byref(p), ptr(self.values), ptr(self.c_index), ptr(self.r_index), ptr(self.slices_ptr))
        self.sort_cols = bool(sort_cols)
        if sort_cols:
            call(f"mfp_scoo_sort_cols_{_SFX[self.dtype]}", p.slices_count, ptr(self.slices_ptr), ptr(self.values),
                 ptr(self.c_index), ptr(self.r_index))


def fill_row_blocks(m: csr_matrix_class, nnz_per_wg: int = 64) -> np.ndarray:
    """fill_row_blocks (csr_adaptive_spmv.cu:180-240) with its bin size as a parameter."""
    n = C.c_uint32()
    call("mfp_csr_adaptive_row_blocks", m.rows, ptr(m.row_ptr), nnz_per_wg, None, C.byref(n))
    out = np.empty(n.value + 1, np.uint32)
    call("mfp_csr_adaptive_row_blocks", m.rows, ptr(m.row_ptr), nnz_per_wg, ptr(out), C.byref(n))
    return out


class measurement_class:
    """measurement_class (common/measurement_class.h:11-58)."""

    def __init__(self, format: str = "", elapsed: float = 0.0, load_store_bytes: float = 0.0,
                 operations_count: float = 0.0):
        self.count = 0
        if format == "" and elapsed == 0.0:
            self.format, self.elapsed, self.effective_bandwidth, self.computational_throughput = "", 0.0, 0.0, 0.0
            return
        r = _capi.Measurement()
        call("mfp_measurement_make", format.encode(), float(elapsed), float(load_store_bytes),
             float(operations_count), C.byref(r))
        self.format = r.format.decode()
        self.elapsed, self.effective_bandwidth = r.elapsed, r.effective_bandwidth
        self.computational_throughput = r.computational_throughput

    def __iadd__(self, rhs: "measurement_class"):
        self.elapsed += rhs.elapsed
        self.effective_bandwidth += rhs.effective_bandwidth
        self.computational_throughput += rhs.computational_throughput
        self.format = rhs.format
        self.count += 1
        return self

    def finalize(self) -> None:
        if self.count:
            self.elapsed /= self.count
            self.effective_bandwidth /= self.count
            self.computational_throughput /= self.count


def compare_results(a: np.ndarray, b: np.ndarray) -> tuple[float, int | None]:
    """compare_results (measurement_class.h:60-89): (relative squared error, first bad index)."""
    assert a.dtype == b.dtype and a.size == b.size
    err = C.c_double()
    bad = C.c_uint32()
    aa, bb = np.ascontiguousarray(a), np.ascontiguousarray(b)  # alive across the call
    call(f"mfp_compare_results_{_SFX[a.dtype]}", a.size, ptr(aa), ptr(bb), C.byref(err), C.byref(bad))
    return err.value, (None if bad.value == 0xFFFFFFFF else int(bad.value))


def lowp_quantize(m: csr_matrix_class, value_type: int):
    """16-bit value bit patterns and per-row scales (mfp_lowp_quantize)."""
    v = np.ascontiguousarray(m.data, np.float64)
    q = np.empty(m.nnz, np.uint16)
    sc = np.empty(m.rows, np.float32)
    call("mfp_lowp_quantize", value_type, m.rows, ptr(m.row_ptr), ptr(v), ptr(q), ptr(sc))
    return q, sc


def lowp_dequantize(q: np.ndarray, scale: np.ndarray, row_ptr: np.ndarray, value_type: int) -> np.ndarray:
    """Exact float64 values scale_i * float(q_ij) of a reduced-precision CSR."""
    if value_type == 2:
        f = (q.astype(np.uint32) << 16).view(np.float32)
    else:
        f = q.view(np.float16).astype(np.float32)
    rows = np.repeat(np.arange(row_ptr.size - 1), np.diff(row_ptr.astype(np.int64)))
    return f.astype(np.float64) * scale.astype(np.float64)[rows]
