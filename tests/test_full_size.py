"""Parity at the benchmark configurations' full sizes (needs a B200).

Every plain format on
  power_law_4M   4,194,304 rows, Zipf(2.0) row lengths clipped to [1, 50000]
                 (31,314,811 nnz), FP64 (FP32 runs in test_spmv_gpu.py);
  stencil27_128  27-point stencil on 128^3 (2,097,152 rows, 55,742,968 nnz),
                 FP32 and FP64;
  banded_8M      8,388,608 rows, 32 columns per row in a half band of 64
                 (268,435,456 nnz), FP32 and FP64;
and the reduced-precision layouts (BF16 / FP16 values with per-row FP32
scales, CSR with 16-bit column deltas and ELL with 16-bit offsets) on the
stencil and banded matrices.

Criteria (per row, relative to sum_j |a_ij x_j|, against the oracle's
extended-precision product of the same rounded inputs): 1e-5 for FP32,
1e-12 for FP64; reduced precision within 1e-5 of the dequantized matrix's
product (the kernel's FP32 arithmetic) and within 1e-2 of the FP64 product
(the format).  Every run also checks sum_i y_i against (column sums of A) . x,
a property that does not depend on how the rows were split.

The device layouts are built by the engine's converters from a device CSR
(bit-identical to the host converters, tests/test_convert_gpu.py); the
matrices are the seeded generators' (synth.py).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from matrix_format_performance_b200 import formats as F
from matrix_format_performance_b200 import synth
from matrix_format_performance_b200.device import (COO, CSR_ADAPTIVE, CSR_SCALAR, CSR_VECTOR, ELL, HYBRID, SCOO,
                                                   DeviceMatrix)

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.float32): 1e-5, np.dtype(np.float64): 1e-12}
GEN = {
    "power_law_4M": lambda: synth.power_law(seed=0),
    "stencil27_128": lambda: synth.stencil_27(128, seed=0),
    "banded_8M": lambda: synth.banded(seed=0),
}
PLAIN = [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE, ELL, COO, SCOO, HYBRID]
BF16, F16 = 2, 3
# grouped by matrix, so each matrix is generated once
CASES = ([("power_law_4M", "plain", np.float64, f) for f in PLAIN if f != ELL] +
         [(c, kind, a, b) for c in ("stencil27_128", "banded_8M")
          for kind, a, b in ([("plain", dt, f) for dt in (np.float32, np.float64) for f in PLAIN] +
                             [("lowp", vt, layout) for vt in (BF16, F16) for layout in ("csr", "ell")])])


def _id(c):
    name, kind, a, b = c
    if kind == "plain":
        return f"{name}-{np.dtype(a).name}-fmt{b}"
    return f"{name}-{'bf16' if a == BF16 else 'fp16'}-{b}"


# One configuration at a time is kept (the banded matrix alone is 3.2 GB in FP64).
_STATE = {}


def _matrix(name):
    if _STATE.get("name") != name:
        _STATE.clear()
        _STATE["name"] = name
        _STATE["m64"] = GEN[name]()
    return _STATE["m64"]


def _typed(name, dt):
    """The matrix in dtype dt, x, the oracle's product and device CSR arrays."""
    key = ("typed", np.dtype(dt).str)
    m64 = _matrix(name)
    if key not in _STATE:
        from oracle import load_oracle
        for k in [k for k in _STATE if isinstance(k, tuple) and k[0] == "typed"]:
            del _STATE[k]  # one dtype's device arrays at a time
        m = m64 if np.dtype(dt) == np.float64 else m64.astype(dt)
        x = synth.vector(0, m.cols).astype(dt)
        ys, ab = load_oracle().csr_spmv_exact(m.rows, m.row_ptr, m.columns, m.data, x)
        colsum = np.bincount(m.columns, weights=m.data.astype(np.float64), minlength=m.cols)
        dev = (torch.from_numpy(m.row_ptr.view(np.int32)).cuda(), torch.from_numpy(m.columns.view(np.int32)).cuda(),
               torch.from_numpy(m.data).cuda(), torch.from_numpy(x).cuda())
        _STATE[key] = (m, x, ys, ab, colsum @ x.astype(np.float64), dev)
    return _STATE[key]


def _check(m, y, ys, ab, checksum, tol, what):
    y = y.astype(np.float64)
    err = np.abs(y - ys)
    bad = np.nonzero(~(err <= tol * ab))[0]
    assert bad.size == 0, (f"{what}: {bad.size} rows out of tolerance, first {bad[:5]}, err {err[bad[:5]]}, "
                           f"bound {(tol * ab)[bad[:5]]}")
    # sum_i y_i equals (column sums of A) . x; each row's error is bounded by
    # tol * ab_i, so the sums differ by at most tol * sum_i ab_i (+ FP64 rounding)
    assert abs(y.sum() - checksum) <= (tol + 1e-12) * ab.sum(), what


@pytest.mark.parametrize("case", CASES, ids=[_id(c) for c in CASES])
def test_full_size(case):
    name, kind, a, b = case
    if kind == "plain":
        _plain(name, a, b)
    else:
        _reduced(name, a, b)


def _plain(name, dt, fmt):
    m, x, ys, ab, checksum, (rp, ci, va, xt) = _typed(name, dt)
    hw = F.row_length_quantile(m, 2 / 3) if fmt == HYBRID else None
    dm = DeviceMatrix.from_device_csr(rp, ci, va, m.cols, fmt, ell_width=hw)
    try:
        ys_runs = []
        for _ in range(2):
            yt = torch.full((m.rows,), float("nan"), dtype=xt.dtype, device="cuda")
            dm.spmv(xt, yt)
            torch.cuda.synchronize()
            ys_runs.append(yt.cpu().numpy())
    finally:
        dm.close()
    _check(m, ys_runs[0], ys, ab, checksum, TOL[np.dtype(dt)], f"{name}/{np.dtype(dt).name}/fmt{fmt}")
    # the same launch twice gives the same bits (no atomics in these kernels)
    assert np.array_equal(ys_runs[0].view(np.uint8), ys_runs[1].view(np.uint8))


def _lowp_reference(name, vt):
    """The dequantized matrix's product (kernel arithmetic) and the FP64 product (format accuracy)."""
    key = ("lowp", vt)
    if key not in _STATE:
        from oracle import load_oracle
        orc = load_oracle()
        m = _matrix(name)
        x = synth.vector(0, m.cols).astype(np.float32)
        if "lowp64" not in _STATE:
            _STATE["lowp64"] = orc.csr_spmv_exact(m.rows, m.row_ptr, m.columns, m.data, x.astype(np.float64))
        q, sc = F.lowp_quantize(m, vt)
        deq = F.lowp_dequantize(q, sc, m.row_ptr, vt)
        yq, abq = orc.csr_spmv_exact(m.rows, m.row_ptr, m.columns, deq, x.astype(np.float64))
        del q, deq
        _STATE[key] = (x, yq, abq)
    return _STATE[key] + _STATE["lowp64"]


def _reduced(name, vt, layout):
    m = _matrix(name)
    x, yq, abq, y64, ab64 = _lowp_reference(name, vt)
    build = DeviceMatrix.from_csr_lowp if layout == "csr" else DeviceMatrix.from_ell_lowp
    dm = build(m, vt, True)  # 16-bit column deltas / offsets: the layouts these matrices admit
    try:
        xt = torch.from_numpy(x).cuda()
        yt = torch.full((m.rows,), float("nan"), device="cuda")
        dm.spmv(xt, yt)
        torch.cuda.synchronize()
        y = yt.cpu().numpy().astype(np.float64)
    finally:
        dm.close()
    assert np.all(np.abs(y - yq) <= 1e-5 * abq), f"{name}/{layout}: kernel arithmetic off the dequantized product"
    rel = np.abs(y - y64) / np.maximum(ab64, 1e-300)
    assert rel.max() <= 1e-2, f"{name}/{layout}: max relative error {rel.max():.3g} vs FP64"
    err = C.c_uint32(1)
    from matrix_format_performance_b200._capi import call
    call("mfp_lowp_error", 0, 1, C.byref(err))
    assert err.value == 0
