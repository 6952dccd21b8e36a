"""Reduced-precision SpMV measurement (stencil and banded configurations).

    python -m matrix_format_performance_b200.bench_lowp [--stencil 128] [--banded 8388608] [--reps 20]

For each matrix: device time of every FP32 plain kernel (CSR row-block
scalar, vector, adaptive, the streaming CSR kernel at two chunk sizes, and
ELL; the fastest is "the FP32 plain kernel") and of the 16-bit-value layouts
(CSR and ELL, BF16 and FP16, with uint32 column ids and with 16-bit column
deltas / offsets), CUDA events around each
launch with L2 flushed before it; max and mean per-row relative error against
the FP64 product (|y - y*| / sum_j |a_ij x_j|).  One JSON line per matrix.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def _time(dm, xt, yt, reps, flush, stream):
    import torch
    ts = []
    for i in range(reps + 3):
        flush.fill_(float(i))
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        dm.spmv(xt, yt, stream)
        b.record(stream)
        if i >= 3:
            ts.append((a, b))
    torch.cuda.synchronize()
    ms = sorted(a.elapsed_time(b) for a, b in ts)
    return ms[len(ms) // 2]


def fp64_product(m, x: np.ndarray, rows_per_chunk: int = 1 << 20) -> tuple[np.ndarray, np.ndarray]:
    """(A x, sum_j |a_ij x_j|) in float64 with numpy, chunked over rows."""
    y = np.zeros(m.rows)
    ab = np.zeros(m.rows)
    rp = m.row_ptr.astype(np.int64)
    for r0 in range(0, m.rows, rows_per_chunk):
        r1 = min(m.rows, r0 + rows_per_chunk)
        e0, e1 = rp[r0], rp[r1]
        if e1 == e0:
            continue
        p = m.data[e0:e1].astype(np.float64) * x[m.columns[e0:e1]]
        nonempty = rp[r0 + 1:r1 + 1] > rp[r0:r1]
        idx = (rp[r0:r1] - e0)[nonempty]
        y[r0:r1][nonempty] = np.add.reduceat(p, idx)
        ab[r0:r1][nonempty] = np.add.reduceat(np.abs(p), idx)
    return y, ab


def measure(name: str, m64, reps: int) -> dict:
    import torch
    from . import synth
    from .device import BF16, CSR_ADAPTIVE, CSR_SCALAR, CSR_VECTOR, ELL, F16, DeviceMatrix, device_info
    dev = device_info(0)
    stream = torch.cuda.current_stream()
    flush = torch.empty(int(2 * dev.l2_bytes) // 4 + 1, device="cuda")
    x32 = synth.vector(0, m64.cols).astype(np.float32)
    xt = torch.from_numpy(x32).cuda()
    yt = torch.empty(m64.rows, device="cuda")
    y64, ab = fp64_product(m64, x32.astype(np.float64))
    ab = np.maximum(ab, 1e-300)
    out = {"matrix": name, "rows": m64.rows, "nnz": int(m64.nnz), "fp32": {}, "reduced": {}}
    m32 = m64.astype(np.float32)
    for fmt, label, cfg in ((CSR_SCALAR, "GPU CSR", None), (CSR_VECTOR, "GPU CSR (vector)", None),
                            (CSR_ADAPTIVE, "GPU CSR-Adaptive", None),
                            (CSR_SCALAR, "GPU CSR (streaming, 2048)", {"kernel": 2}),
                            (CSR_SCALAR, "GPU CSR (streaming, 1024)", {"kernel": 3}), (ELL, "GPU ELL", None)):
        if fmt == ELL:
            from .formats import ell_matrix_class
            if ell_matrix_class.estimate_size(m32) * 8 > (1 << 31):
                continue
            dm = DeviceMatrix.from_ell(ell_matrix_class(m32))
        else:
            dm = DeviceMatrix.from_csr(m32, fmt, cfg)
        ms = _time(dm, xt, yt, reps, flush, stream)
        info = dm.info()
        rel = np.abs(yt.cpu().numpy().astype(np.float64) - y64) / ab
        out["fp32"][label] = {"ms": ms, "gbs": info.algorithmic_bytes / (ms * 1e-3) / 1e9,
                              "max_rel_err": float(rel.max()), "mean_rel_err": float(rel.mean())}
        dm.close()
    del m32
    base = min(v["ms"] for v in out["fp32"].values())
    out["fp32_plain_ms"] = base
    for layout, vt, vname, idx16 in [(lay, vt, vn, i) for lay in ("CSR", "ELL") for vt, vn in ((BF16, "BF16"), (F16, "FP16"))
                                     for i in (False, True)]:
        if True:
            key = f"{layout} {vname}{('+delta16' if layout == 'CSR' else '+offset16') if idx16 else ''}"
            try:
                dm = (DeviceMatrix.from_csr_lowp(m64, vt, idx16) if layout == "CSR"
                      else DeviceMatrix.from_ell_lowp(m64, vt, idx16))
            except Exception as e:  # 16-bit deltas need local columns
                out["reduced"][key] = {"skipped": str(e)}
                continue
            ms = _time(dm, xt, yt, reps, flush, stream)
            info = dm.info()
            rel = np.abs(yt.cpu().numpy().astype(np.float64) - y64) / ab
            out["reduced"][key] = {"ms": ms, "speedup_vs_fp32_plain": base / ms,
                                   "gbs_algorithmic": info.algorithmic_bytes / (ms * 1e-3) / 1e9,
                                   "gbs_format": info.format_bytes / (ms * 1e-3) / 1e9,
                                   "format_bytes": int(info.format_bytes),
                                   "max_rel_err": float(rel.max()), "mean_rel_err": float(rel.mean())}
            dm.close()
    return out


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--stencil", type=int, default=128)
    ap.add_argument("--banded", type=int, default=8_388_608)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    import torch
    from . import synth
    torch.cuda.set_device(0)
    for name, gen in ((f"stencil27_{a.stencil}", lambda: synth.stencil_27(a.stencil)),
                      (f"banded_{a.banded}", lambda: synth.banded(n=a.banded))):
        t = time.time()
        m = gen()
        print(f"[bench_lowp] {name}: {m.rows} rows {m.nnz} nnz generated in {time.time() - t:.1f}s",
              file=sys.stderr, flush=True)
        print(json.dumps(measure(name, m, a.reps)), flush=True)
        del m


if __name__ == "__main__":
    main()
