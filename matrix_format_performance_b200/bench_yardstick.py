"""The engine's formats beside cuSPARSE's generic SpMV (the vendor yardstick).

    python -m matrix_format_performance_b200.bench_yardstick [--rows 4194304] [--stencil 128] [--banded 8388608]
        [--which power_law,stencil,banded] [--dtype f32|f64]

For the power-law, stencil and banded matrices (FP32, or FP64 with --dtype
f64): median device time of
the engine's CSR scalar / vector / adaptive, COO, SCOO (also with each slice in
column order, the reference's disabled sort_cols option) and hybrid kernels and
of cusparseSpMV on CSR (default, ALG1, ALG2) and COO (default), 20 launches
each with L2 flushed before every launch.  One JSON line per matrix with ms and
algorithmic GB/s.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def measure(name, m, reps=20):
    import torch

    from . import formats as F
    from . import synth
    from . import yardstick as Y
    from .device import FORMAT_NAMES, LABELS, DeviceMatrix, device_info
    dev = device_info(0)
    vs = m.data.dtype.itemsize
    nbytes = m.nnz * (vs + 4) + (m.rows + 1) * 4 + m.cols * vs + m.rows * vs
    x = torch.from_numpy(synth.vector(5, m.cols).astype(m.data.dtype)).cuda()
    y = torch.empty(m.rows, dtype=x.dtype, device="cuda")
    out = {"matrix": name, "dtype": str(m.data.dtype), "rows": m.rows, "nnz": int(m.nnz), "engine": {},
           "cusparse": {}}
    for key in ("csr", "csr_vector", "csr_adaptive", "coo", "scoo", "hybrid"):
        fmt = FORMAT_NAMES[key]
        dm = DeviceMatrix.build(m, fmt, sm_count=dev.sm_count, shared_mem=int(dev.shared_mem_per_block),
                                hybrid_width=F.row_length_quantile(m, 2 / 3))
        _, med = dm.time(x, y, reps=reps, flush_l2=True)
        out["engine"][LABELS[fmt]] = {"ms": med * 1e3, "gbs": nbytes / med / 1e9}
        dm.close()
    # SCOO with each slice in column order (the reference's disabled sort_cols option)
    dm = DeviceMatrix.from_scoo(F.scoo_matrix_class(dev.sm_count, int(dev.shared_mem_per_block), m, sort_cols=True))
    _, med = dm.time(x, y, reps=reps, flush_l2=True)
    out["engine"]["GPU SCOO (sorted columns)"] = {"ms": med * 1e3, "gbs": nbytes / med / 1e9}
    dm.close()
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).cuda()
    ci = torch.from_numpy(m.columns.view(np.int32)).cuda()
    va = torch.from_numpy(m.data).cuda()
    ri = torch.from_numpy(np.repeat(np.arange(m.rows, dtype=np.int32), np.diff(m.row_ptr.astype(np.int64)))).cuda()
    for label, fmt, alg, idx in (("CSR default", Y.CSR, Y.ALG_DEFAULT, rp), ("CSR ALG1", Y.CSR, Y.ALG1, rp),
                                 ("CSR ALG2", Y.CSR, Y.ALG2, rp), ("COO default", Y.COO, Y.ALG_DEFAULT, ri)):
        med = Y.spmv(fmt, alg, m.rows, m.cols, m.nnz, idx, ci, va, x, y, reps=reps)
        out["cusparse"][label] = {"ms": med * 1e3, "gbs": nbytes / med / 1e9}
    best_e = min(v["ms"] for v in out["engine"].values())
    best_c = min(v["ms"] for v in out["cusparse"].values())
    out["best_engine_vs_best_cusparse"] = best_c / best_e
    return out


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--rows", type=int, default=4_194_304)
    ap.add_argument("--stencil", type=int, default=128)
    ap.add_argument("--banded", type=int, default=8_388_608)
    ap.add_argument("--which", default="power_law,stencil,banded")
    ap.add_argument("--dtype", default="f32", choices=["f32", "f64"])
    a = ap.parse_args()
    import torch

    from . import synth
    torch.cuda.set_device(0)
    which = set(a.which.split(","))
    for key, name, gen in (("power_law", f"power_law_{a.rows}", lambda: synth.power_law(rows=a.rows, seed=0, cols=a.rows)),
                           ("stencil", f"stencil27_{a.stencil}", lambda: synth.stencil_27(a.stencil)),
                           ("banded", f"banded_{a.banded}", lambda: synth.banded(n=a.banded))):
        if key in which:
            print(json.dumps(measure(name, gen().astype(np.float64 if a.dtype == "f64" else np.float32))),
                  flush=True)


if __name__ == "__main__":
    main()
