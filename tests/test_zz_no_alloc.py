"""The allocation-free COO entry point (mfp_coo_spmv_f32_noalloc).

It exists for callers that may not allocate device memory (hosts that hand out
every byte through their own pool, loops that cannot take cudaMalloc's cost),
so its workspace is a fixed array inside the library.  It runs the same
two-pass COO as the regular entry point, which takes a caller's workspace, so
the two must agree bit for bit; both are also checked against the oracle's
extended-precision product.  Two calls run in a row: the second finds the
first call's contents in the shared array.  This file sorts last, so a run
that stops at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from matrix_format_performance_b200 import formats as F
from matrix_format_performance_b200 import synth
from matrix_format_performance_b200._capi import MfpError, call

TOL = 1e-5  # per row, relative to sum |a_ij x_j| (the tolerance of the other float32 tests)
MAX_NNZ = 44_739_072  # what the fixed 4 MiB array covers


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.gpu
def test_noalloc_coo_matches_oracle_and_workspace_coo_on_consecutive_calls():
    from oracle import load_oracle
    m = synth.power_law(rows=400_000, seed=21).astype(np.float32)
    coo = F.coo_matrix_class(m)
    x = synth.vector(9, m.cols).astype(np.float32)
    d_v = torch.from_numpy(coo.data).cuda()
    d_c = torch.from_numpy(coo.cols_.view(np.int32)).cuda()
    d_r = torch.from_numpy(coo.rows_.view(np.int32)).cuda()
    d_x = torch.from_numpy(x).cuda()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    nbytes = C.c_size_t()
    call("mfp_coo_workspace_bytes", m.rows, m.nnz, C.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    y_ws = torch.full((m.rows,), float("nan"), device="cuda")
    call("mfp_coo_spmv_f32", m.rows, m.cols, m.nnz, _ptr(d_v), _ptr(d_c), _ptr(d_r), _ptr(d_x), _ptr(y_ws),
         _ptr(ws), nbytes.value, stream)
    torch.cuda.synchronize()
    y_ws = y_ws.cpu().numpy()
    ys, ab = load_oracle().csr_spmv_exact(m.rows, m.row_ptr, m.columns, m.data, x)
    for _ in range(2):
        y = torch.full((m.rows,), float("nan"), device="cuda")
        call("mfp_coo_spmv_f32_noalloc", m.rows, m.cols, m.nnz, _ptr(d_v), _ptr(d_c), _ptr(d_r), _ptr(d_x),
             _ptr(y), stream)
        torch.cuda.synchronize()
        got = y.cpu().numpy()
        err = np.abs(got.astype(np.float64) - ys)
        assert np.all(err <= TOL * ab), f"{np.count_nonzero(~(err <= TOL * ab))} rows out of tolerance"
        assert np.array_equal(got, y_ws)


@pytest.mark.gpu
def test_noalloc_coo_empty_rows_before_and_after():
    """Rows before the first and after the last element come back as 0."""
    from oracle import load_oracle
    rows, cols = 300_000, 1000
    rng = np.random.default_rng(4)
    r = np.sort(rng.integers(120_000, 130_000, size=50_000)).astype(np.uint32)
    c = rng.integers(0, cols, size=r.size).astype(np.uint32)
    v = rng.uniform(-1, 1, size=r.size).astype(np.float32)
    x = rng.uniform(-1, 1, size=cols).astype(np.float32)
    rp = np.zeros(rows + 1, np.int64)
    np.add.at(rp, r.astype(np.int64) + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    d = [torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda() for a in (v, c, r, x)]
    ys, ab = load_oracle().csr_spmv_exact(rows, rp, c, v, x)
    for _ in range(2):
        y = torch.full((rows,), float("nan"), device="cuda")
        call("mfp_coo_spmv_f32_noalloc", rows, cols, r.size, *[_ptr(t) for t in d], _ptr(y), stream)
        torch.cuda.synchronize()
        got = y.cpu().numpy().astype(np.float64)
        assert np.all(np.abs(got - ys) <= TOL * ab)
        assert not np.any(got[:120_000]) and not np.any(got[130_000:])


@pytest.mark.gpu
def test_noalloc_coo_rejects_sizes_beyond_its_scratch():
    with pytest.raises(MfpError, match="fixed scratch holds 4194304 bytes"):
        call("mfp_coo_spmv_f32_noalloc", 10, 10, MAX_NNZ + 1, None, None, None, None, None, None)
