"""One SpMV per named format on one seeded matrix: the program to run under a
profiler (ncu captures one launch per kernel with -k / -c).

    python -m matrix_format_performance_b200.profile_case --matrix power_law --rows 2097152 \\
        --formats csr,csr_vector,coo [--dtype f32|f64] [--reps 1]
    python -m matrix_format_performance_b200.profile_case --matrix stencil --n 128 --formats ell_bf16

Matrices: power_law (Zipf(2.0) row lengths, --rows rows), stencil (27-point,
--n^3 rows), banded (--rows rows, 32 per row in a half band of 64).  Formats:
csr, csr_vector, csr_adaptive, ell, coo, scoo, hybrid (ELL width at the
2/3-quantile, or --hybrid-width), ell_bf16 / csr_bf16 (16-bit values, 16-bit indices), probe
(mfp_probe_spmv_loads mode 2).  Every layout is converted on the GPU from one
device CSR.  Prints one line with the matrix size when done.
"""
from __future__ import annotations

import argparse
import ctypes as C

import numpy as np


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--matrix", choices=["power_law", "stencil", "banded"], default="power_law")
    ap.add_argument("--rows", type=int, default=2_097_152)
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--formats", default="csr,csr_vector,coo")
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--hybrid-width", type=int, default=None, help="hybrid ELL width (default: 2/3-quantile)")
    a = ap.parse_args()
    import torch

    from . import formats as F
    from . import synth
    from ._capi import call
    from .device import BF16, FORMAT_NAMES, HYBRID, DeviceMatrix
    torch.cuda.set_device(0)
    if a.matrix == "power_law":
        m64 = synth.power_law(rows=a.rows, seed=0)
    elif a.matrix == "stencil":
        m64 = synth.stencil_27(a.n, seed=0)
    else:
        m64 = synth.banded(n=a.rows, seed=0)
    dt = np.float32 if a.dtype == "f32" else np.float64
    m = m64.astype(dt) if dt == np.float32 else m64
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).cuda()
    ci = torch.from_numpy(m.columns.view(np.int32)).cuda()
    va = torch.from_numpy(m.data).cuda()
    x = torch.from_numpy(synth.vector(0, m.cols).astype(dt)).cuda()
    y = torch.empty(m.rows, dtype=x.dtype, device="cuda")
    x32 = torch.from_numpy(synth.vector(0, m.cols).astype(np.float32)).cuda()
    y32 = torch.empty(m.rows, device="cuda")
    for name in a.formats.split(","):
        if name in ("ell_bf16", "csr_bf16"):
            dm = (DeviceMatrix.from_ell_lowp if name == "ell_bf16" else DeviceMatrix.from_csr_lowp)(m64, BF16, True)
            for _ in range(a.reps):
                dm.spmv(x32, y32)
        elif name == "probe":
            out = torch.empty(1 << 16, device="cuda")
            for _ in range(a.reps):
                call("mfp_probe_spmv_loads", 2, 0, m.nnz, C.c_void_p(va.data_ptr()), C.c_void_p(ci.data_ptr()),
                     C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), out.numel(),
                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
            torch.cuda.synchronize()
            continue
        else:
            fmt = FORMAT_NAMES[name]
            hw = (a.hybrid_width if a.hybrid_width is not None else F.row_length_quantile(m, 2 / 3)) \
                if fmt == HYBRID else None
            dm = DeviceMatrix.from_device_csr(rp, ci, va, m.cols, fmt, ell_width=hw)
            for _ in range(a.reps):
                dm.spmv(x, y)
        torch.cuda.synchronize()
        dm.close()
    print(f"profile_case: {a.matrix} {m.rows} rows, {m.nnz} nnz, {a.dtype}: {a.formats}")


if __name__ == "__main__":
    main()
