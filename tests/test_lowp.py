"""Reduced-precision CSR: 16-bit values with per-row FP32 scales.

CPU: the quantizer rounds like numpy (FP16) / like the round-to-nearest-even
rule (BF16), and the 16-bit column deltas decode to the original columns.
GPU: both kernels (pipelined, for 16-byte-aligned arrays; row-block, for any
alignment) equal the dequantized matrix times x within 1e-5 (FP32
accumulation) and the format stays within 1e-2 of the FP64 product, both per
row relative to sum_j |a_ij x_j|.
"""
import ctypes as C

import numpy as np
import pytest

from matrix_format_performance_b200 import formats as F
from matrix_format_performance_b200 import synth
from matrix_format_performance_b200._capi import MfpError, call

BF16, F16 = 2, 3


def bf16_rne(f32: np.ndarray) -> np.ndarray:
    u = f32.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


@pytest.mark.parametrize("vt", [BF16, F16])
def test_quantizer_rounding_and_scales(vt):
    m = synth.stencil_27(12, seed=3)
    q, sc = F.lowp_quantize(m, vt)
    rows = np.repeat(np.arange(m.rows), np.diff(m.row_ptr.astype(np.int64)))
    mx = np.maximum.reduceat(np.abs(m.data), m.row_ptr[:-1].astype(np.int64))
    assert np.array_equal(sc, mx.astype(np.float32))
    f = (m.data / sc.astype(np.float64)[rows]).astype(np.float32)
    want = bf16_rne(f) if vt == BF16 else f.astype(np.float16).view(np.uint16)
    assert np.array_equal(q, want)
    deq = F.lowp_dequantize(q, sc, m.row_ptr, vt)
    rel = np.abs(deq - m.data) / np.abs(sc.astype(np.float64)[rows])
    assert rel.max() <= (2.0 ** -8 if vt == BF16 else 2.0 ** -11)


def test_quantizer_empty_and_zero_rows():
    rp = np.array([0, 0, 2, 2], np.uint32)
    v = np.array([0.0, 0.0])
    q = np.empty(2, np.uint16)
    sc = np.empty(3, np.float32)
    call("mfp_lowp_quantize", BF16, 3, F.ptr(rp), F.ptr(v), F.ptr(q), F.ptr(sc))
    assert np.array_equal(sc, np.ones(3, np.float32)) and np.array_equal(q, np.zeros(2, np.uint16))


def test_delta_encoding_round_trip_and_limit():
    m = synth.banded(n=20_000, seed=1)
    n = m.nnz
    d = np.empty(n, np.uint16)
    b = np.empty((n + 2047) // 2048, np.uint32)
    call("mfp_lowp_deltas", n, F.ptr(m.columns), F.ptr(d), F.ptr(b))
    assert np.array_equal(b[np.arange(n) // 2048] + d.astype(np.uint32), m.columns)
    spread = np.array([0, 70_000] * 4, np.uint32)
    d2 = np.empty(spread.size, np.uint16)
    b2 = np.empty(1, np.uint32)
    with pytest.raises(MfpError, match="16-bit deltas"):
        call("mfp_lowp_deltas", spread.size, F.ptr(spread), F.ptr(d2), F.ptr(b2))


_CASES = {
    "stencil_32": lambda: synth.stencil_27(32, seed=5),
    "banded_100k": lambda: synth.banded(n=100_000, seed=6),
    "power_law_100k": lambda: synth.power_law(rows=100_000, seed=7),
    # rows longer than a pipeline stage (split into sub-chunks), rotated rows of 32
    "long_rows": lambda: synth.uniform(300, 0, 30_000, seed=11, cols=60_000),
    # empty rows, a partial last row block, < 8-element tails
    "sparse_ragged": lambda: synth.uniform(5_003, 0, 3, seed=12),
    "tiny": lambda: synth.uniform(3, 1, 5, seed=13),
    "equal_rows_16": lambda: synth.uniform(20_000, 16, 16, seed=14),
}
_CACHE = {}


def case(name):
    if name not in _CACHE:
        _CACHE[name] = _CASES[name]()
    return _CACHE[name]


def _check(oracle_lib, m, vt, y, x):
    y = y.astype(np.float64)
    q, sc = F.lowp_quantize(m, vt)
    deq = F.lowp_dequantize(q, sc, m.row_ptr, vt)
    yq, abq = oracle_lib.csr_spmv_exact(m.rows, m.row_ptr, m.columns, deq, x.astype(np.float64))
    assert np.all(np.abs(y - yq) <= 1e-5 * abq)              # kernel arithmetic
    y64, ab = oracle_lib.csr_spmv_exact(m.rows, m.row_ptr, m.columns, m.data, x.astype(np.float64))
    rel = np.abs(y - y64) / np.maximum(ab, 1e-300)
    assert rel.max() <= 1e-2                                  # format accuracy vs FP64


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["stencil_32", "banded_100k", "power_law_100k", "long_rows"])
@pytest.mark.parametrize("vt", [BF16, F16])
@pytest.mark.parametrize("index16", [False, True])
def test_lowp_handle_accuracy(oracle_lib, name, vt, index16):
    """Handles; matrices with rows longer than 1,024 elements (power_law_100k,
    long_rows) run the row-block kernel, whose warps share the long rows."""
    import torch
    from matrix_format_performance_b200.device import DeviceMatrix
    m = case(name)
    if index16 and name == "power_law_100k":
        with pytest.raises(MfpError, match="16-bit deltas"):
            DeviceMatrix.from_csr_lowp(m, vt, True)
        return
    x = synth.vector(0, m.cols).astype(np.float32)
    dm = DeviceMatrix.from_csr_lowp(m, vt, index16)
    xt = torch.from_numpy(x).cuda()
    yt = torch.full((m.rows,), float("nan"), device="cuda")
    dm.spmv(xt, yt)
    torch.cuda.synchronize()
    _check(oracle_lib, m, vt, yt.cpu().numpy(), x)
    info = dm.info()
    assert info.value_type == vt
    assert info.algorithmic_bytes == m.nnz * 6 + m.rows * 4 + (m.rows + 1) * 4 + m.cols * 4 + m.rows * 4


def _dev_copy(a: np.ndarray, offset: int = 0):
    """Device copy of `a` starting `offset` bytes past a 256-byte-aligned allocation."""
    import torch
    raw = torch.zeros(a.nbytes + offset + 16, dtype=torch.uint8, device="cuda")
    if a.nbytes:
        raw[offset:offset + a.nbytes].copy_(torch.from_numpy(a.view(np.uint8).ravel()))
    return raw, raw.data_ptr() + offset


def _raw_lowp(m, vt, index16, x, misalign: bool):
    """y from mfp_lowp_spmv with 16-byte-aligned arrays (pipelined kernel) or
    arrays shifted off 16-byte alignment (row-block kernel)."""
    import torch
    q, sc = F.lowp_quantize(m, vt)
    off16, off32 = (2, 4) if misalign else (0, 0)
    keep = []

    def dev(a, off):
        t, p = _dev_copy(np.ascontiguousarray(a), off)
        keep.append(t)
        return C.c_void_p(p) if a.size else None
    rp = dev(m.row_ptr, off32)
    qd = dev(q, off16)
    scd = dev(sc, 0)
    xd = dev(x, 0)
    yt = torch.full((m.rows,), float("nan"), device="cuda")
    cols = delta = base = None
    if index16:
        d = np.empty(m.nnz, np.uint16)
        b = np.empty(max(1, (m.nnz + 2047) // 2048), np.uint32)
        call("mfp_lowp_deltas", m.nnz, F.ptr(m.columns), F.ptr(d), F.ptr(b))
        delta, base = dev(d, off16), dev(b, 0)
    else:
        cols = dev(m.columns, off32)
    call("mfp_lowp_spmv", vt, m.rows, m.cols, m.nnz, rp, qd, scd, cols, delta, base, xd,
         C.c_void_p(yt.data_ptr()), None)
    torch.cuda.synchronize()
    return yt.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["long_rows", "sparse_ragged", "tiny", "equal_rows_16", "stencil_32"])
@pytest.mark.parametrize("vt", [BF16, F16])
@pytest.mark.parametrize("index16", [False, True])
def test_lowp_pipelined_and_row_block(oracle_lib, name, vt, index16):
    """Both kernels within 1e-5 of the dequantized product; the pipelined
    kernel gives the same bits on a second run; its error word stays clear."""
    m = case(name)
    x = synth.vector(1, m.cols).astype(np.float32)
    y_tma = _raw_lowp(m, vt, index16, x, misalign=False)
    y_rb = _raw_lowp(m, vt, index16, x, misalign=True)
    again = _raw_lowp(m, vt, index16, x, misalign=False)
    assert np.array_equal(y_tma.view(np.uint32), again.view(np.uint32))
    _check(oracle_lib, m, vt, y_tma, x)
    _check(oracle_lib, m, vt, y_rb, x)
    err = C.c_uint32(1)
    call("mfp_lowp_error", 0, 1, C.byref(err))
    assert err.value == 0


# ---- reduced-precision ELL --------------------------------------------------
def _lowp_ell_host(m, vt, index16):
    w = int(np.diff(m.row_ptr.astype(np.int64)).max()) if m.rows else 0
    q = np.empty(w * m.rows, np.uint16)
    idx = np.empty(w * m.rows, np.uint16 if index16 else np.uint32)
    sc = np.empty(m.rows, np.float32)
    v = np.ascontiguousarray(m.data, np.float64)
    call("mfp_lowp_ell_from_csr", vt, int(index16), m.rows, m.cols, F.ptr(m.row_ptr), F.ptr(m.columns), F.ptr(v), w,
         F.ptr(q), F.ptr(idx), F.ptr(sc))
    return w, q, idx, sc


@pytest.mark.parametrize("index16", [False, True])
def test_lowp_ell_layout_decodes_to_the_quantized_csr(index16):
    m = synth.uniform(3_001, 0, 9, seed=21)  # empty rows, rows % 8 != 0
    w, q, idx, sc = _lowp_ell_host(m, BF16, index16)
    qc, scc = F.lowp_quantize(m, BF16)
    assert np.array_equal(sc, scc)
    lens = np.diff(m.row_ptr.astype(np.int64))
    for r in range(0, m.rows, 97):
        for k in range(w):
            o = k * m.rows + r
            col = (r + int(idx[o]) - 32768) if index16 else int(idx[o])
            if k < lens[r]:
                e = m.row_ptr[r] + k
                assert q[o] == qc[e] and col == m.columns[e]
            else:
                assert q[o] == 0 and 0 <= col < m.cols


def test_lowp_ell_offset_limit():
    m = synth.uniform(40_000, 1, 3, seed=22)  # columns anywhere: offsets beyond 16 bits
    with pytest.raises(MfpError, match="16-bit column offsets"):
        _lowp_ell_host(m, BF16, True)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["stencil_32", "banded_100k", "sparse_ragged", "tiny"])
@pytest.mark.parametrize("vt", [BF16, F16])
@pytest.mark.parametrize("index16", [False, True])
def test_lowp_ell_accuracy(oracle_lib, name, vt, index16):
    import torch
    from matrix_format_performance_b200.device import DeviceMatrix
    m = case(name)
    x = synth.vector(0, m.cols).astype(np.float32)
    try:
        dm = DeviceMatrix.from_ell_lowp(m, vt, index16)
    except MfpError as e:  # offsets only for local columns
        assert index16 and "16-bit column offsets" in str(e)
        return
    xt = torch.from_numpy(x).cuda()
    yt = torch.full((m.rows,), float("nan"), device="cuda")
    dm.spmv(xt, yt)
    torch.cuda.synchronize()
    _check(oracle_lib, m, vt, yt.cpu().numpy(), x)
    assert dm.info().value_type == vt


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["stencil_32", "banded_100k"])
@pytest.mark.parametrize("vt", [BF16, F16])
def test_lowp_ell_kernel_variants_agree(oracle_lib, name, vt):
    """The 16-bit-offset ELL kernel's variants give the same bits: x, y and
    scales 32- or 16-byte aligned (runs of x; 32- or 16-byte y stores), y and
    scales shifted by 4 bytes (8 rows per thread, scalar stores), and q
    shifted off 16-byte alignment (lane-interleaved rows)."""
    import torch
    m = case(name)
    assert m.rows % 8 == 0
    w, q, idx, sc = _lowp_ell_host(m, vt, True)
    x = synth.vector(2, m.cols).astype(np.float32)
    keep = []

    def dev(a, off):
        t, p = _dev_copy(np.ascontiguousarray(a), off)
        keep.append(t)
        return C.c_void_p(p)

    outs = []
    for q_off, ys_off in ((0, 0), (0, 16), (0, 4), (2, 4)):
        qd, od = dev(q, q_off), dev(idx, q_off)
        scd, xd = dev(sc, ys_off), dev(x, 0)
        yraw, yp = _dev_copy(np.full(m.rows, np.nan, np.float32), ys_off)
        call("mfp_lowp_ell_spmv", vt, m.rows, m.cols, w, qd, scd, None, od, xd, C.c_void_p(yp), None)
        torch.cuda.synchronize()
        outs.append(yraw[ys_off:ys_off + 4 * m.rows].cpu().numpy().view(np.float32).copy())
    for y in outs[1:]:
        assert np.array_equal(outs[0].view(np.uint32), y.view(np.uint32))
    _check(oracle_lib, m, vt, outs[0], x)
