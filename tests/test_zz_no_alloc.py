"""The allocation-free COO entry point (mfp_coo_spmv_f32_noalloc).

It exists for callers that may not allocate device memory (hosts that hand out
every byte through their own pool, loops that cannot take cudaMalloc's cost),
so its scratch is a fixed array inside the library.  Checked against the
regular COO entry point, which gets a workspace from the caller, on two calls
in a row (the second call finds the first call's scratch contents).  This
file sorts last so a run that stops at the first failure has run the rest.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from matrix_format_performance_b200 import formats as F
from matrix_format_performance_b200 import synth
from matrix_format_performance_b200._capi import MfpError, call

TOL = 1e-5  # per row, relative to sum |a_ij x_j| (the tolerance of the other float32 tests)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.gpu
def test_noalloc_coo_matches_workspace_coo_on_consecutive_calls():
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
    ws = torch.zeros(nbytes.value, dtype=torch.uint8, device="cuda")
    y_ref = torch.full((m.rows,), float("nan"), device="cuda")
    call("mfp_coo_spmv_f32", m.rows, m.cols, m.nnz, _ptr(d_v), _ptr(d_c), _ptr(d_r), _ptr(d_x), _ptr(y_ref),
         _ptr(ws), nbytes.value, stream)
    torch.cuda.synchronize()
    ref = y_ref.cpu().numpy().astype(np.float64)
    _, ab = load_oracle().csr_spmv_exact(m.rows, m.row_ptr, m.columns, m.data, x)
    for _ in range(2):
        y = torch.full((m.rows,), float("nan"), device="cuda")
        call("mfp_coo_spmv_f32_noalloc", m.rows, m.cols, m.nnz, _ptr(d_v), _ptr(d_c), _ptr(d_r), _ptr(d_x),
             _ptr(y), stream)
        torch.cuda.synchronize()
        got = y.cpu().numpy().astype(np.float64)
        assert np.all(np.abs(got - ref) <= TOL * ab)


@pytest.mark.gpu
def test_noalloc_coo_rejects_sizes_beyond_its_scratch():
    with pytest.raises(MfpError, match="fixed scratch holds 1048576 bytes"):
        call("mfp_coo_spmv_f32_noalloc", 10, 10, 200_000_000, None, None, None, None, None, None)
