"""Batched SpMV: hundreds of CSR matrices of uneven sizes in one launch.

The matrices become one block-diagonal CSR on the device (mfp_batch_create):
x and y are single concatenated device vectors and matrix k owns the slices
[x_offsets[k], x_offsets[k+1]) and [y_offsets[k], y_offsets[k+1]).  The plan
starts as the CSR scalar default; `autotune` times the candidate plans (CSR
scalar thresholds, the persistent streaming kernel, CSR vector lanes,
CSR-Adaptive bins) on the batch itself and keeps the fastest; `graph_launch`
replays a CUDA graph of the launch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import call
from .device import _dptr, _stream
from .formats import csr_matrix_class

ALGO_NAMES = {0: "csr_scalar", 1: "csr_vector", 2: "csr_adaptive"}


class Batch:
    def __init__(self, mats: list[csr_matrix_class]):
        if not mats:
            raise ValueError("empty batch")
        dt = np.dtype(mats[0].dtype)
        if any(np.dtype(m.dtype) != dt for m in mats):
            raise ValueError("all matrices of a batch share one value type")
        self.dtype = dt
        n = len(mats)
        self._keep = [(np.ascontiguousarray(m.row_ptr, np.uint32), np.ascontiguousarray(m.columns, np.uint32),
                       np.ascontiguousarray(m.data, dt)) for m in mats]
        rows = np.array([m.rows for m in mats], np.uint32)
        cols = np.array([m.cols for m in mats], np.uint32)
        P = C.c_void_p * n
        rp = P(*[a[0].ctypes.data for a in self._keep])
        ci = P(*[a[1].ctypes.data if a[1].size else 0 for a in self._keep])
        va = P(*[a[2].ctypes.data if a[2].size else 0 for a in self._keep])
        self._h = C.c_void_p()
        call("mfp_batch_create", 0 if dt == np.float32 else 1, n, C.c_void_p(rows.ctypes.data),
             C.c_void_p(cols.ctypes.data), rp, ci, va, C.byref(self._h))
        self._keep = None
        self.x_offsets = np.empty(n + 1, np.uint64)
        self.y_offsets = np.empty(n + 1, np.uint64)
        call("mfp_batch_offsets", self._h, C.c_void_p(self.x_offsets.ctypes.data),
             C.c_void_p(self.y_offsets.ctypes.data))

    def info(self) -> _capi.BatchInfo:
        i = _capi.BatchInfo()
        call("mfp_batch_get_info", self._h, C.byref(i))
        return i

    def set_config(self, algo: int = 0, **csr) -> None:
        c = _capi.BatchConfig()
        c.algo = algo
        for k, v in csr.items():
            setattr(c.csr, k, int(v))
        call("mfp_batch_set_config", self._h, C.byref(c))

    def autotune(self, x, y, reps: int = 5, stream=None) -> tuple[dict, float]:
        c = _capi.BatchConfig()
        best = C.c_double()
        call("mfp_batch_autotune", self._h, _dptr(x), _dptr(y), reps, _stream(stream), C.byref(c), C.byref(best))
        return config_dict(c), best.value

    def spmv(self, x, y, stream=None) -> None:
        call("mfp_batch_spmv", self._h, _dptr(x), _dptr(y), _stream(stream))

    def graph_launch(self, x, y, stream=None) -> None:
        call("mfp_batch_graph_launch", self._h, _dptr(x), _dptr(y), _stream(stream))

    def close(self) -> None:
        if self._h:
            _capi.load().mfp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def config_dict(c: _capi.BatchConfig) -> dict:
    return {"algo": ALGO_NAMES.get(c.algo, c.algo), "vector_lanes": c.csr.vector_lanes, "bin_nnz": c.csr.bin_nnz,
            "assist_threshold": c.csr.assist_threshold, "long_row_threshold": c.csr.long_row_threshold,
            "kernel": c.csr.kernel}


def uneven_set(count: int = 512, lo: int = 1_000, hi: int = 200_000, seed0: int = 0, dtype=np.float32):
    """The batched configuration's matrices: seeds seed0.., rows log-uniform in
    [lo, hi], structure drawn from {uniform 4-64 nnz/row, Zipf(1.8) rows,
    tridiagonal, block-diagonal 32x32 dense blocks}, values U[-1, 1]."""
    from . import synth
    out, kinds = [], []
    for k in range(count):
        rng = np.random.default_rng(1_000_003 * (seed0 + k) + 17)
        rows = int(np.exp(rng.uniform(np.log(lo), np.log(hi + 1))))
        rows = min(max(rows, lo), hi)
        fam = int(rng.integers(0, 4))
        s = seed0 + k
        if fam == 0:
            m = synth.uniform(rows, 4, 64, seed=s)
        elif fam == 1:
            m = synth.power_law(rows=rows, alpha=1.8, k_lo=1, k_hi=rows, seed=s)
        elif fam == 2:
            m = synth.tridiagonal(rows, seed=s)
        else:
            m = synth.block_diagonal(rows, block=32, seed=s)
        out.append(m.astype(dtype))
        kinds.append(("uniform_4_64", "zipf_1.8", "tridiagonal", "block_diag_32")[fam])
    return out, kinds
