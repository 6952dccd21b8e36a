"""Batched uneven SpMV measurement (the batched configuration).

    python -m matrix_format_performance_b200.bench_batched [--count 512] [--reps 10]

512 seeded FP32 matrices (rows log-uniform in [1,000, 200,000]; uniform 4-64
nnz/row, Zipf(1.8) rows, tridiagonal, or block-diagonal 32x32 dense blocks)
with one concatenated x and y on the device:
  per_matrix  512 launches, one CSR handle per matrix (default CSR scalar
              plan), issued back to back on one stream (and the same 512
              launches captured in one CUDA graph, without host issue cost)
  batched     one launch of the block-diagonal batch, default plan
  autotuned   the plan mfp_batch_autotune picked, replayed as a CUDA graph
Times: CUDA events around one whole pass (all 512 products), median of
--reps passes, L2 flushed before each pass.  GB/s = the sum over the
matrices of the algorithmic bytes / time.  Parity: every matrix's y of the
graph replay against an FP64 product, per row |y - y*| <= 1e-5 sum_j |a_ij x_j|.
Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--lo", type=int, default=1_000)
    ap.add_argument("--hi", type=int, default=200_000)
    a = ap.parse_args()
    import torch

    from . import synth
    from .batch import Batch, uneven_set
    from .bench_lowp import fp64_product
    from .device import CSR_SCALAR, DeviceMatrix, device_info

    torch.cuda.set_device(0)
    t = time.time()
    mats, kinds = uneven_set(a.count, a.lo, a.hi)
    rows = sum(m.rows for m in mats)
    nnz = sum(m.nnz for m in mats)
    print(f"[bench_batched] {len(mats)} matrices, {rows} rows, {nnz} nnz generated in {time.time() - t:.1f}s",
          file=sys.stderr, flush=True)
    b = Batch(mats)
    info = b.info()
    xo, yo = b.x_offsets.astype(np.int64), b.y_offsets.astype(np.int64)
    x = synth.vector(7, int(xo[-1])).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    yt = torch.zeros(int(yo[-1]), device="cuda")
    handles = [DeviceMatrix.from_csr(m, CSR_SCALAR) for m in mats]
    xs = [xt[xo[k]:xo[k + 1]] for k in range(len(mats))]
    ys = [yt[yo[k]:yo[k + 1]] for k in range(len(mats))]
    dev = device_info(0)
    flush = torch.empty(int(2 * dev.l2_bytes) // 4 + 1, device="cuda")
    stream = torch.cuda.current_stream()

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        ts = []
        for i in range(reps):
            flush.fill_(float(i))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return sorted(ts)[len(ts) // 2]

    def per_matrix():
        for h, xv, yv in zip(handles, xs, ys):
            h.spmv(xv, yv, stream)
    ms_per = timed(per_matrix, a.reps)
    y_per = yt.cpu().numpy().copy()
    # the same 512 launches captured in one CUDA graph: no host issue cost
    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        per_matrix_on = lambda s: [h.spmv(xv, yv, s) for h, xv, yv in zip(handles, xs, ys)]  # noqa: E731
        per_matrix_on(side)
    stream.wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        per_matrix_on(torch.cuda.current_stream())
    ms_per_graph = timed(g.replay, a.reps)
    ms_batch = timed(lambda: b.spmv(xt, yt, stream), a.reps)
    cfg, best_s = b.autotune(xt, yt, reps=5, stream=stream)
    ms_graph = timed(lambda: b.graph_launch(xt, yt, stream), a.reps)
    y = yt.cpu().numpy()

    worst = 0.0
    for k, m in enumerate(mats):
        y64, ab = fp64_product(m, x[xo[k]:xo[k + 1]].astype(np.float64))
        rel = np.abs(y[yo[k]:yo[k + 1]] - y64) / np.maximum(ab, 1e-300)
        worst = max(worst, float(rel.max()) if rel.size else 0.0)
    per_vs_batch = float(np.max(np.abs(y_per - y))) if y.size else 0.0
    gb = info.algorithmic_bytes / 1e9
    out = {"config": "batched_uneven_512", "matrices": len(mats), "rows": rows, "nnz": nnz,
           "families": {k: kinds.count(k) for k in sorted(set(kinds))},
           "algorithmic_bytes": int(info.algorithmic_bytes),
           "per_matrix": {"ms": ms_per, "gbs": gb / (ms_per * 1e-3), "launches": len(mats),
                          "issue": "one C-ABI call per matrix from Python"},
           "per_matrix_graph": {"ms": ms_per_graph, "gbs": gb / (ms_per_graph * 1e-3), "launches": len(mats),
                                "issue": "the 512 launches captured in one CUDA graph"},
           "batched_default": {"ms": ms_batch, "gbs": gb / (ms_batch * 1e-3), "launches": 1},
           "autotuned_graph": {"ms": ms_graph, "gbs": gb / (ms_graph * 1e-3), "launches": 1, "plan": cfg,
                               "autotune_best_ms": best_s * 1e3},
           "speedup_graph_vs_per_matrix": ms_per / ms_graph,
           "speedup_graph_vs_per_matrix_graph": ms_per_graph / ms_graph,
           "max_rel_err_vs_fp64": worst, "max_abs_diff_per_matrix_vs_batched": per_vs_batch,
           "timing": f"CUDA events around one pass, median of {a.reps}, L2 flushed before each pass"}
    print(json.dumps(out), flush=True)
    b.close()
    for h in handles:
        h.close()


if __name__ == "__main__":
    main()
