"""Seeded synthetic matrices for the five benchmark configurations.

They stand in for the SuiteSparse matrices the reference was measured on
(those files are not shipped).  Generation runs in the C library
(csrc/synth.cpp); matrices are pure functions of their parameters.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import call
from .formats import csr_matrix_class, ptr

LAPLACIAN_2D, POWER_LAW, STENCIL_27, BANDED, UNIFORM, TRIDIAGONAL, BLOCK_DIAGONAL = range(7)


def synth_csr(kind: int, seed: int = 0, n: int = 0, cols: int = 0, alpha: float = 0.0, k_lo: int = 0,
              k_hi: int = 0, band: int = 0) -> csr_matrix_class:
    """CSR with float64 values (cast with .astype for float32 kernels)."""
    p = _capi.SynthParams(kind, seed, n, cols, alpha, k_lo, k_hi, band)
    rows, ncols, nnz = C.c_uint32(), C.c_uint32(), C.c_uint64()
    call("mfp_synth_csr", C.byref(p), C.byref(rows), C.byref(ncols), C.byref(nnz), None, None, None)
    rp = np.empty(rows.value + 1, np.uint32)
    ci = np.empty(nnz.value, np.uint32)
    va = np.empty(nnz.value, np.float64)
    call("mfp_synth_csr", C.byref(p), C.byref(rows), C.byref(ncols), C.byref(nnz), ptr(rp),
         ptr(ci) if nnz.value else C.c_void_p(1), ptr(va) if nnz.value else C.c_void_p(1))
    return csr_matrix_class.from_arrays(rows.value, ncols.value, rp, ci, va, np.float64)


def vector(seed: int, n: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    out = np.empty(n, np.float64)
    call("mfp_synth_vector_f64", seed, n, lo, hi, ptr(out))
    return out


def laplacian_2d(n: int = 512) -> csr_matrix_class:
    """5-point Laplacian on an n x n grid: 4 on the diagonal, -1 off it."""
    return synth_csr(LAPLACIAN_2D, n=n)


def power_law(rows: int = 4_194_304, alpha: float = 2.0, k_lo: int = 1, k_hi: int = 50_000,
              seed: int = 0, cols: int = 0) -> csr_matrix_class:
    """Row lengths Zipf(alpha) on k >= 1 clipped to [k_lo, k_hi]; distinct uniform columns; U[-1,1]."""
    return synth_csr(POWER_LAW, seed=seed, n=rows, cols=cols or rows, alpha=alpha, k_lo=k_lo, k_hi=k_hi)


def stencil_27(n: int = 128, seed: int = 0) -> csr_matrix_class:
    """27-point stencil on an n^3 grid, values U[-1,1]."""
    return synth_csr(STENCIL_27, seed=seed, n=n)


def banded(n: int = 8_388_608, half_band: int = 64, per_row: int = 32, seed: int = 0) -> csr_matrix_class:
    """per_row distinct columns uniform in [r - half_band, r + half_band]; values U[-1,1]."""
    return synth_csr(BANDED, seed=seed, n=n, band=half_band, k_lo=per_row)


def uniform(rows: int, k_lo: int, k_hi: int, seed: int = 0, cols: int = 0) -> csr_matrix_class:
    return synth_csr(UNIFORM, seed=seed, n=rows, cols=cols or rows, k_lo=k_lo, k_hi=k_hi)


def tridiagonal(rows: int, seed: int = 0) -> csr_matrix_class:
    return synth_csr(TRIDIAGONAL, seed=seed, n=rows)


def block_diagonal(rows: int, block: int = 32, seed: int = 0) -> csr_matrix_class:
    return synth_csr(BLOCK_DIAGONAL, seed=seed, n=rows, band=block)


@dataclass(frozen=True)
class Workload:
    name: str
    description: str


WORKLOADS = {
    "laplacian": Workload("laplacian_512", "2D 5-point Laplacian on a 512x512 grid (262,144 rows, 1,308,672 nnz)"),
    "power_law": Workload("power_law_4M", "4,194,304 x 4,194,304, row lengths Zipf(2.0) clipped to [1, 50000], "
                                          "distinct uniform columns, values U[-1,1], seed 0"),
    "stencil": Workload("stencil27_128", "27-point stencil on a 128^3 grid (2,097,152 rows, 55,742,968 nnz)"),
    "banded": Workload("banded_8M", "n = 8,388,608, half band 64, 32 distinct columns per row (268,435,456 nnz)"),
}
