"""Batched SpMV: many CSR matrices of uneven sizes as one block-diagonal CSR.

CPU: invalid input is rejected before any device work.
GPU: every matrix's slice of y is within 1e-5 (per row, of sum_j |a_ij x_j|)
of the FP64 oracle for the default plan, for each family of candidate plans,
and after autotuning; the CUDA-graph replay gives the same bits as the direct
launch; empty matrices and empty rows are handled.
"""
import ctypes as C

import numpy as np
import pytest

from matrix_format_performance_b200 import synth
from matrix_format_performance_b200._capi import MfpError, call
from matrix_format_performance_b200.formats import csr_matrix_class


def _small_set():
    mats = [synth.uniform(3_000, 4, 64, seed=1), synth.power_law(rows=20_000, alpha=1.8, k_hi=20_000, seed=2),
            synth.tridiagonal(5_000, seed=3), synth.block_diagonal(4_096, block=32, seed=4),
            synth.uniform(1_000, 0, 2, seed=5), synth.laplacian_2d(40)]
    # an all-empty matrix and a one-row matrix
    mats.append(csr_matrix_class.from_arrays(7, 9, np.zeros(8, np.uint32), np.zeros(0, np.uint32), np.zeros(0)))
    mats.append(synth.uniform(1, 3, 3, seed=6, cols=50))
    return [m.astype(np.float32) for m in mats]


def test_batch_rejects_bad_row_ptr():
    rp = np.array([0, 2, 1], np.uint32)
    ci = np.array([0, 1], np.uint32)
    v = np.ones(2, np.float32)
    rows = np.array([2], np.uint32)
    cols = np.array([2], np.uint32)
    P = C.c_void_p * 1
    h = C.c_void_p()
    with pytest.raises(MfpError, match="matrix 0"):
        call("mfp_batch_create", 0, 1, C.c_void_p(rows.ctypes.data), C.c_void_p(cols.ctypes.data),
             P(rp.ctypes.data), P(ci.ctypes.data), P(v.ctypes.data), C.byref(h))


def _check(oracle_lib, mats, b, y, x):
    for k, m in enumerate(mats):
        xs = x[b.x_offsets[k]:b.x_offsets[k + 1]].astype(np.float64)
        ys, ab = oracle_lib.csr_spmv_exact(m.rows, m.row_ptr, m.columns, m.data.astype(np.float64), xs)
        got = y[b.y_offsets[k]:b.y_offsets[k + 1]].astype(np.float64)
        assert np.all(np.abs(got - ys) <= 1e-5 * ab), k


@pytest.mark.gpu
def test_batch_parity_plans_autotune_and_graph(oracle_lib):
    import torch
    from matrix_format_performance_b200.batch import Batch
    mats = _small_set()
    b = Batch(mats)
    info = b.info()
    assert info.matrices == len(mats) and info.rows == sum(m.rows for m in mats)
    assert info.nnz == sum(m.nnz for m in mats)
    x = synth.vector(3, int(b.x_offsets[-1])).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    yt = torch.full((int(b.y_offsets[-1]),), float("nan"), device="cuda")
    b.spmv(xt, yt)
    torch.cuda.synchronize()
    _check(oracle_lib, mats, b, yt.cpu().numpy(), x)
    for algo, kw in ((0, {"assist_threshold": 32, "long_row_threshold": 2048}), (0, {"kernel": 2}),
                     (1, {"vector_lanes": 8}), (1, {"vector_lanes": 32}), (2, {"bin_nnz": 508})):
        b.set_config(algo, **kw)
        yt.fill_(float("nan"))
        b.spmv(xt, yt)
        torch.cuda.synchronize()
        _check(oracle_lib, mats, b, yt.cpu().numpy(), x)
    cfg, best = b.autotune(xt, yt, reps=3)
    assert best > 0 and cfg["algo"] in ("csr_scalar", "csr_vector", "csr_adaptive")
    yt.fill_(float("nan"))
    b.spmv(xt, yt)
    torch.cuda.synchronize()
    direct = yt.cpu().numpy().copy()
    _check(oracle_lib, mats, b, direct, x)
    for _ in range(2):
        yt.fill_(float("nan"))
        b.graph_launch(xt, yt)
        torch.cuda.synchronize()
        assert np.array_equal(direct.view(np.uint32), yt.cpu().numpy().view(np.uint32))
    # a new (x, y) pair is captured again
    y2 = torch.full_like(yt, float("nan"))
    b.graph_launch(xt, y2)
    torch.cuda.synchronize()
    assert np.array_equal(direct.view(np.uint32), y2.cpu().numpy().view(np.uint32))
    b.close()


@pytest.mark.gpu
def test_batch_default_plan_matches_per_matrix_handles():
    """The default plan (CSR scalar) sums each row in CSR order, as the
    per-matrix CSR handles do: identical bits for rows below the long-row
    threshold."""
    import torch
    from matrix_format_performance_b200.batch import Batch
    from matrix_format_performance_b200.device import CSR_SCALAR, DeviceMatrix
    mats = [synth.uniform(2_000, 1, 40, seed=s).astype(np.float32) for s in range(12)]
    b = Batch(mats)
    x = synth.vector(4, int(b.x_offsets[-1])).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    yb = torch.empty(int(b.y_offsets[-1]), device="cuda")
    b.spmv(xt, yb)
    for k, m in enumerate(mats):
        h = DeviceMatrix.from_csr(m, CSR_SCALAR)
        yk = torch.empty(m.rows, device="cuda")
        h.spmv(xt[int(b.x_offsets[k]):int(b.x_offsets[k + 1])], yk)
        torch.cuda.synchronize()
        assert torch.equal(yk, yb[int(b.y_offsets[k]):int(b.y_offsets[k + 1])])
        h.close()
    b.close()
