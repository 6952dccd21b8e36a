"""Device-resident matrices: the reference-facing SpMV call per format.

A DeviceMatrix uploads one layout once (mfp_matrix_create_*) and runs
y = A*x through mfp_matrix_spmv (device x, y) or mfp_matrix_spmv_host (host
x, y with the copies inside).  Device memory for x and y comes from torch
tensors; only raw pointers and the CUDA stream handle cross into the
library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import call
from .formats import (coo_matrix_class, csr_matrix_class, ell_matrix_class, hybrid_matrix_class, ptr,
                      scoo_matrix_class)

CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE, ELL, COO, SCOO, HYBRID, CSR_LOWP, ELL_LOWP = range(9)
BF16, F16 = 2, 3
FORMAT_NAMES = {"csr": CSR_SCALAR, "csr_vector": CSR_VECTOR, "csr_adaptive": CSR_ADAPTIVE, "ell": ELL,
                "coo": COO, "scoo": SCOO, "hybrid": HYBRID}
# JSON labels of the reference (gpu_matrix_multiplier.cu:129, :443, :546, :712, :1092;
# csr_adaptive_spmv.cu:320; scoo_spmv.cu:221)
LABELS = {CSR_SCALAR: "GPU CSR", CSR_VECTOR: "GPU CSR (vector)", CSR_ADAPTIVE: "GPU CSR-Adaptive", ELL: "GPU ELL",
          COO: "GPU COO", SCOO: "GPU SCOO", HYBRID: "GPU Hybrid (atomic)",
          CSR_LOWP: "GPU CSR (16-bit values)", ELL_LOWP: "GPU ELL (16-bit values)"}
_VT = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}


def _cfg(config: dict | None):
    if not config:
        return None
    c = _capi.CsrConfig()
    for k, v in config.items():
        setattr(c, k, int(v))
    return C.byref(c)


def _dptr(t) -> C.c_void_p:
    """Device pointer of a torch tensor (or an int address)."""
    if isinstance(t, int):
        return C.c_void_p(t)
    assert t.is_cuda and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


def _stream(stream) -> C.c_void_p:
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


class DeviceMatrix:
    def __init__(self, handle: C.c_void_p, fmt: int, dtype):
        self._h = handle
        self.format = fmt
        self.dtype = np.dtype(dtype)
        self.label = LABELS[fmt]

    # -- construction -------------------------------------------------------
    @classmethod
    def from_csr(cls, m: csr_matrix_class, fmt: int = CSR_SCALAR, config: dict | None = None) -> "DeviceMatrix":
        h = C.c_void_p()
        call("mfp_matrix_create_csr", fmt, _VT[m.dtype], m.rows, m.cols, m.nnz, ptr(m.row_ptr), ptr(m.columns),
             ptr(m.data), _cfg(config), C.byref(h))
        return cls(h, fmt, m.dtype)

    @classmethod
    def from_ell(cls, e: ell_matrix_class) -> "DeviceMatrix":
        h = C.c_void_p()
        call("mfp_matrix_create_ell", _VT[e.dtype], e.rows, e.cols, e.elements_in_rows, ptr(e.columns),
             ptr(e.data), C.byref(h))
        return cls(h, ELL, e.dtype)

    @classmethod
    def from_coo(cls, c: coo_matrix_class) -> "DeviceMatrix":
        h = C.c_void_p()
        call("mfp_matrix_create_coo", _VT[c.dtype], c.rows, c.cols, c.elements_count, ptr(c.rows_), ptr(c.cols_),
             ptr(c.data), C.byref(h))
        return cls(h, COO, c.dtype)

    @classmethod
    def from_scoo(cls, s: scoo_matrix_class) -> "DeviceMatrix":
        h = C.c_void_p()
        call("mfp_matrix_create_scoo", _VT[s.dtype], s.rows, s.cols, s.nnz, C.byref(s.params), ptr(s.c_index),
             ptr(s.r_index), ptr(s.slices_ptr), ptr(s.values), C.byref(h))
        return cls(h, SCOO, s.dtype)

    @classmethod
    def from_hybrid(cls, hm: hybrid_matrix_class) -> "DeviceMatrix":
        e, c = hm.ell_matrix, hm.coo_matrix
        h = C.c_void_p()
        call("mfp_matrix_create_hybrid", _VT[e.dtype], e.rows, e.cols, e.elements_in_rows, ptr(e.columns),
             ptr(e.data), c.elements_count, ptr(c.rows_), ptr(c.cols_), ptr(c.data), C.byref(h))
        return cls(h, HYBRID, e.dtype)

    @classmethod
    def from_csr_lowp(cls, m: csr_matrix_class, value_type: int = BF16, index16: bool = False) -> "DeviceMatrix":
        """16-bit values (BF16/FP16) with per-row FP32 scales; x and y float32."""
        v = np.ascontiguousarray(m.data, np.float64)
        h = C.c_void_p()
        call("mfp_matrix_create_lowp", value_type, int(index16), m.rows, m.cols, m.nnz, ptr(m.row_ptr),
             ptr(m.columns), ptr(v), C.byref(h))
        dm = cls(h, CSR_LOWP, np.float32)
        dm.label = f"GPU CSR ({'BF16' if value_type == BF16 else 'FP16'}{', 16-bit deltas' if index16 else ''})"
        return dm

    @classmethod
    def from_ell_lowp(cls, m: csr_matrix_class, value_type: int = BF16, index16: bool = False) -> "DeviceMatrix":
        """ELL with 16-bit values and per-row FP32 scales (width = longest row);
        index16: 16-bit column offsets from the row."""
        v = np.ascontiguousarray(m.data, np.float64)
        h = C.c_void_p()
        call("mfp_matrix_create_lowp_ell", value_type, int(index16), m.rows, m.cols, m.nnz, ptr(m.row_ptr),
             ptr(m.columns), ptr(v), C.byref(h))
        dm = cls(h, ELL_LOWP, np.float32)
        dm.label = f"GPU ELL ({'BF16' if value_type == BF16 else 'FP16'}{', 16-bit offsets' if index16 else ''})"
        return dm

    @classmethod
    def build(cls, m: csr_matrix_class, fmt: int, *, sm_count: int = 148, shared_mem: int = 49152,
              hybrid_width: int | None = None, config: dict | None = None) -> "DeviceMatrix":
        """Builds format `fmt` from CSR with the reference converters."""
        if fmt in (CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE):
            return cls.from_csr(m, fmt, config)
        if fmt == ELL:
            return cls.from_ell(ell_matrix_class(m))
        if fmt == COO:
            return cls.from_coo(coo_matrix_class(m))
        if fmt == SCOO:
            return cls.from_scoo(scoo_matrix_class(sm_count, shared_mem, m))
        if fmt == HYBRID:
            hm = hybrid_matrix_class(m)
            if hybrid_width is None:
                hm.allocate(m, 0.2)
            else:
                hm.allocate_width(m, hybrid_width)
            return cls.from_hybrid(hm)
        raise ValueError(f"unknown format {fmt}")

    @classmethod
    def from_device_csr(cls, row_ptr, columns, data, cols: int, fmt: int, *, config: dict | None = None,
                        ell_width: int | None = None, scoo: "_capi.ScooParams | None" = None,
                        scoo_sort_cols: bool = False) -> "DeviceMatrix":
        """Builds format `fmt` from a CSR already on the GPU (torch tensors):
        the layout is converted by the engine's kernels (mfp_matrix_create_device).
        ell_width: ELL / hybrid ELL part (None = longest row); scoo_sort_cols: the
        SCOO slices in column order."""
        o = _capi.DeviceBuildOptions()
        o.ell_width = _capi.ELL_WIDTH_LONGEST if ell_width is None else int(ell_width)
        o.scoo_sort_cols = int(bool(scoo_sort_cols))
        cfg = _capi.CsrConfig()
        if config:
            for k, v in config.items():
                setattr(cfg, k, int(v))
            o.csr = C.pointer(cfg)
        if scoo is not None:
            o.scoo = C.pointer(scoo)
        dt = np.dtype(str(data.dtype).replace("torch.", ""))
        nnz = columns.numel()
        h = C.c_void_p()
        call("mfp_matrix_create_device", fmt, _VT[dt], row_ptr.numel() - 1, cols, nnz, _dptr(row_ptr),
             _dptr(columns) if nnz else None, _dptr(data) if nnz else None, C.byref(o), C.byref(h))
        return cls(h, fmt, dt)

    # -- use ------------------------------------------------------------------
    def info(self) -> _capi.MatrixInfo:
        i = _capi.MatrixInfo()
        call("mfp_matrix_get_info", self._h, C.byref(i))
        return i

    def spmv(self, x, y, stream=None) -> None:
        call("mfp_matrix_spmv", self._h, _dptr(x), _dptr(y), _stream(stream))

    def spmv_host(self, x: np.ndarray, y: np.ndarray, stream=None) -> None:
        assert x.dtype == self.dtype and y.dtype == self.dtype
        call("mfp_matrix_spmv_host", self._h, ptr(x), ptr(y), _stream(stream))

    def spmv_host_batch(self, xs: list, ys: list, stream=None) -> None:
        """ys[i] = A @ xs[i] for host vectors, copies overlapped with the
        kernels (mfp_matrix_spmv_host_batch); page-locked vectors overlap."""
        assert len(xs) == len(ys)
        for x, y in zip(xs, ys):
            assert x.dtype == self.dtype and y.dtype == self.dtype
        n = len(xs)
        px = (C.c_void_p * max(1, n))(*[x.ctypes.data for x in xs])
        py = (C.c_void_p * max(1, n))(*[y.ctypes.data for y in ys])
        call("mfp_matrix_spmv_host_batch", self._h, n, px, py, _stream(stream))

    def time(self, x, y, reps: int = 20, flush_l2: bool = True, stream=None) -> tuple[float, float]:
        mean, med = C.c_double(), C.c_double()
        call("mfp_matrix_time", self._h, _dptr(x), _dptr(y), reps, int(flush_l2), _stream(stream),
             C.byref(mean), C.byref(med))
        return mean.value, med.value

    def close(self) -> None:
        if self._h:
            _capi.load().mfp_matrix_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_info(device: int = 0) -> _capi.DeviceInfo:
    d = _capi.DeviceInfo()
    call("mfp_get_device_info", device, C.byref(d))
    return d
