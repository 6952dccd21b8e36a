"""On-device format conversion beside the host converters.

    python -m matrix_format_performance_b200.bench_convert [--which power_law,stencil,banded] [--reps 5]

For each matrix (FP32): the device converters (mfp_dev_*: COO, SCOO, ELL where
its padding fits, hybrid at the 2/3-quantile width, row statistics, and CSR
from shuffled COO triplets) timed with CUDA events (median of --reps after one
warm-up; each call includes its own scratch allocation and the waits it needs
to size its outputs), and the host converters of formats.cpp (one thread, the
reference's algorithms) timed once.  Bytes per conversion = the arrays it
reads plus the arrays it writes; GB/s against the measured HBM peak.  One JSON
line per matrix.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np


def _peak():
    p = Path(__file__).resolve().parent.parent / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _time_dev(fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        out = fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b) * 1e-3)
        del out
    return float(np.median(ts))


def _time_host(fn):
    t = time.perf_counter()
    fn()
    return time.perf_counter() - t


def measure(name, m, reps, host_limit_nnz=100_000_000):
    import torch

    from . import _capi, convert
    from . import formats as F
    from ._capi import call
    peak, kind = _peak()
    rp, ci, v = (torch.from_numpy(m.row_ptr.view(np.int32)).cuda(), torch.from_numpy(m.columns.view(np.int32)).cuda(),
                 torch.from_numpy(m.data).cuda())
    R, N = m.rows, m.nnz
    res = {"matrix": name, "rows": R, "nnz": N, "peak_gbs": peak, "peak_kind": kind, "conversions": {}}

    def add(key, dev_s, nbytes, host_s=None):
        e = {"device_ms": dev_s * 1e3, "bytes": int(nbytes), "gbs": nbytes / dev_s / 1e9,
             "frac_of_hbm": nbytes / dev_s / 1e9 / peak}
        if host_s is not None:
            e["host_ms"] = host_s * 1e3
            e["speedup_vs_host"] = host_s / dev_s
        res["conversions"][key] = e

    big = N > host_limit_nnz
    add("rows_statistics", _time_dev(lambda: convert.rows_statistics(rp), reps), 2 * (R + 1) * 4,
        _time_host(lambda: F.get_rows_statistics(m)))
    add("coo", _time_dev(lambda: convert.coo_from_csr(rp, ci, v), reps), (R + 1) * 4 + N * 8 + N * 12,
        _time_host(lambda: F.coo_matrix_class(m)))
    p = _capi.ScooParams()
    call("mfp_scoo_params_compute", R, 148, 49152, 0, C.byref(p))
    add("scoo", _time_dev(lambda: convert.scoo_from_csr(rp, ci, v, p), reps),
        (R + 1) * 4 + N * 8 + N * 12 + (p.slices_count + 1) * 4,
        _time_host(lambda: F.scoo_matrix_class(148, 49152, m)))
    if F.ell_matrix_class.estimate_size(m) <= 2_000_000_000:
        w = F.get_rows_statistics(m).max_elements_in_rows
        add("ell", _time_dev(lambda: convert.ell_from_csr(rp, ci, v, w), reps), (R + 1) * 4 + N * 8 + R * w * 8,
            _time_host(lambda: F.ell_matrix_class(m)))
    hw = F.row_length_quantile(m, 2 / 3)
    tail = convert.coo_count(rp, hw)
    add("hybrid", _time_dev(lambda: convert.hybrid_from_csr(rp, ci, v, hw), reps),
        2 * (R + 1) * 4 + (N - tail) * 8 + R * hw * 8 + tail * 8 + tail * 12,
        _time_host(lambda: (F.ell_matrix_class(m, hw), F.coo_matrix_class(m, hw))))
    res["hybrid_width"] = hw
    # CSR from shuffled triplets (the Matrix Market reader's output order is arbitrary)
    rng = np.random.default_rng(0)
    r = np.repeat(np.arange(R, dtype=np.uint32), np.diff(m.row_ptr.astype(np.int64)))
    perm = rng.permutation(N)
    t = F.matrix_class(R, m.cols, r[perm], m.columns[perm], m.data[perm].astype(np.float64))
    del r, perm
    dr, dc, dv = (torch.from_numpy(t.row_ids.view(np.int32)).cuda(), torch.from_numpy(t.col_ids.view(np.int32)).cuda(),
                  torch.from_numpy(t.data).cuda())
    host_s = None if big else _time_host(lambda: F.csr_matrix_class(t, np.float32))
    add("csr_from_shuffled_coo", _time_dev(lambda: convert.csr_from_coo(R, m.cols, dr, dc, dv), reps),
        N * 16 + (R + 1) * 4 + N * 8, host_s)
    del dr, dc, dv
    torch.cuda.empty_cache()
    return res


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--which", default="power_law,stencil,banded")
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    import torch

    from . import synth
    torch.cuda.set_device(0)
    makers = {"power_law": lambda: ("power_law_4M", synth.power_law(rows=4_194_304, seed=0)),
              "stencil": lambda: ("stencil_27pt_128", synth.stencil_27(128, seed=0)),
              "banded": lambda: ("banded_8M", synth.banded(n=8_388_608, seed=0))}
    for k in a.which.split(","):
        name, m = makers[k]()
        print(json.dumps(measure(name, m, a.reps)), flush=True)


if __name__ == "__main__":
    main()
