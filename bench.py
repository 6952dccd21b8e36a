#!/usr/bin/env python
"""SpMV benchmark: GB/s and fraction of HBM peak per format.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--scaling strong|weak] [--no-extras]

Headline workload (one "step"): y = A*x once through each plain format the
layout admits -- CSR scalar, CSR vector, CSR-Adaptive, COO, SCOO, hybrid
ELL+COO -- on power_law_4M: a 4,194,304 x 4,194,304 matrix whose row lengths
are Zipf(2.0) clipped to [1, 50000] (distinct uniform columns, values and x
uniform[-1, 1], FP32).  ELL is skipped on it: its padding (width 50,000 x
4,194,304 rows) does not fit, which is also why the reference's driver drops
such matrices.

value    algorithmic bytes of all SpMVs / max-over-ranks device time of the
         kernels (CUDA events on the launching stream; L2 flushed before every
         launch).  Bytes per SpMV: nnz*(4+4) + (rows+1)*4 + cols*4 + rows*4.
e2e      the same bytes / time through the host-buffer API: every step copies
         its x in from page-locked host memory and its y out, inside the
         timed region.  value: mfp_matrix_spmv_host_batch over the steps of
         a format (step i+1's copy-in and step i-1's copy-out overlap step
         i's kernel); single_call_value: one mfp_matrix_spmv_host per step
         (copy in, kernel, copy out, wait).
Multi-GPU (one rank per GPU): --scaling strong (default) splits the one
power-law matrix into contiguous row blocks balanced by nonzeros
(partition.rank_shard), x replicated, each rank's y slice its own; value
counts the global matrix's bytes once.  --scaling weak gives every rank its
own 4,194,304-row block (seeded by rank).  No collective in the data path.

Extra keys on the same line (one GPU):
per_config   stencil27_128 and banded_8M, FP32, every plain format (ELL too)
fp64         the three matrices in FP64 (the reference's double columns)
lowp         BF16 / FP16 values with per-row scales (CSR with 16-bit column
             deltas, ELL with 16-bit offsets) on the stencil and banded
             matrices: time, speedup over the fastest FP32 plain kernel, max
             and mean relative error against the FP64 product (computed by
             the engine's FP64 CSR kernel, which the tests hold to 1e-12)
load_ceiling the load probe (mfp_probe_spmv_loads) on power_law_4M: the
             time of the SpMV's loads alone, a floor for every format
hybrid_widths the power-law hybrid at the headline's 2/3-quantile ELL width
             and at the width that moves the fewest bytes

--impl reference times the reference's own CPU loop
(cpu_csr_spmv_single_thread_naive, compiled from its sources into
oracle/_ref) on all host threads over the same matrix.
"""
from __future__ import annotations

import argparse
import csv
import datetime
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path
from types import SimpleNamespace

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SpMV GB/s & % HBM peak per format; selector/BF16 speedup vs plain at tolerance"
UNIT = "GB/s"
FALLBACK_HBM_GBS = 6650.0
ROWS = 4_194_304
WORKLOAD = ("power_law_4M: 4,194,304 x 4,194,304, row lengths Zipf(2.0) clipped to [1, 50000], "
            "distinct uniform columns, values and x U[-1,1], FP32")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def algorithmic_bytes(rows, cols, nnz, vs=4):
    return nnz * (vs + 4) + (rows + 1) * 4 + cols * vs + rows * vs


def lowp_algorithmic_bytes(rows, cols, nnz):
    """16-bit values + uint32 column ids + per-row FP32 scales; x and y FP32."""
    return nnz * 6 + rows * 4 + (rows + 1) * 4 + cols * 4 + rows * 4


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def traffic_table():
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if self.gpu_id:
                cmd += ["-i", self.gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.file.read())) if len(r) >= 9]
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU loop
# ---------------------------------------------------------------------------
def cpu_baseline_reference(m, threads: int, reps: int, warmup: int = 1):
    """Times the reference CPU loop (oracle/_ref) or, if absent, the oracle port.
    m: rows, cols, nnz, row_ptr, columns and data (values, any float type)."""
    from oracle import load_oracle, load_ref
    ref = load_ref()
    nbytes = algorithmic_bytes(m.rows, m.cols, m.nnz)
    y = np.empty(m.rows, np.float32)
    times = []
    if ref is not None:
        import ctypes as C
        data64 = np.ascontiguousarray(m.data, np.float64)
        h = ref.lib.ref_bench_create(0, threads, m.rows, m.cols, C.c_void_p(m.row_ptr.ctypes.data),
                                     C.c_void_p(m.columns.ctypes.data), C.c_void_p(data64.ctypes.data))
        for i in range(warmup + reps):
            t = ref.lib.ref_bench_run(h, C.c_void_p(y.ctypes.data))
            if i >= warmup:
                times.append(t)
        ref.lib.ref_bench_destroy(h)
        kind = "reference"
    else:
        orc = load_oracle()
        x = np.ones(m.cols, np.float32)
        data32 = np.ascontiguousarray(m.data, np.float32)
        for i in range(warmup + reps):
            _, t = orc.csr_spmv_parallel(threads, m.rows, m.row_ptr, m.columns, data32, x)
            if i >= warmup:
                times.append(t)
        kind = "port"
    mean = sum(times) / len(times)
    return {"value": nbytes / mean / 1e9, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"full matrix ({m.rows} rows, {m.nnz} nnz), FP32 CSR, x = 1, "
                      f"{threads} thread(s), mean of {reps} passes after {warmup} warm-up",
            "seconds_per_spmv": mean}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import synth_power_law  # the seeded generator alone: no engine library is loaded
    t = time.time()
    rows, cols, rp, ci, va = synth_power_law(args.rows, 0, ROWS)
    m = SimpleNamespace(rows=rows, cols=cols, nnz=int(ci.size), row_ptr=rp, columns=ci, data=va)
    log(f"[bench] generated power-law matrix: {rows} rows, {m.nnz} nnz in {time.time() - t:.1f}s")
    threads = os.cpu_count() or 1
    t0 = time.time()
    cb = cpu_baseline_reference(m, threads, reps=args.steps, warmup=args.warmup)
    cfg = {"workload": WORKLOAD, "rows": m.rows, "cols": m.cols, "nnz": m.nnz,
           "formats": ["CPU CSR (reference loop)"],
           "parallelism": f"{threads} host threads, contiguous row ranges (rank 0 only)"}
    out = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["seconds_per_spmv"] * 1e3,
           "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded)", "config": cfg,
           "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
           "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "wall_s": time.time() - t0}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------
def time_launches(launch, n, flush, stream):
    """Device time (ms) of `n` calls of launch(), L2 flushed before each."""
    import torch
    out = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    for a, b in ev:
        flush.fill_(1.0)
        a.record(stream)
        launch()
        b.record(stream)
    torch.cuda.synchronize()
    for a, b in ev:
        out.append(a.elapsed_time(b))
    return out


def fmt_entry(ms_list, nbytes, peak, fbytes=None):
    mean_ms = sum(ms_list) / len(ms_list)
    gbs = nbytes / (mean_ms * 1e-3) / 1e9
    e = {"ms": round(mean_ms, 5), "ms_median": round(statistics.median(ms_list), 5), "gbs": round(gbs, 1),
         "frac": round(gbs / peak, 4)}
    if fbytes is not None:
        e["format_bytes"] = int(fbytes)
        e["format_gbs"] = round(fbytes / (mean_ms * 1e-3) / 1e9, 1)
    return e


def measure_plain(name, m, formats, steps, warmup, flush, stream, peak, hybrid_width):
    """Every format of `formats` on matrix m (dtype of m), built on the device
    from one device CSR.  Returns {label: entry}."""
    import torch

    from matrix_format_performance_b200 import synth
    from matrix_format_performance_b200.device import HYBRID, LABELS, DeviceMatrix
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).cuda()
    ci = torch.from_numpy(m.columns.view(np.int32)).cuda()
    va = torch.from_numpy(m.data).cuda()
    x = torch.from_numpy(synth.vector(0, m.cols).astype(m.dtype)).cuda()
    y = torch.empty(m.rows, dtype=x.dtype, device="cuda")
    vs = np.dtype(m.dtype).itemsize
    nbytes = algorithmic_bytes(m.rows, m.cols, m.nnz, vs)
    out = {}
    for f in formats:
        dm = DeviceMatrix.from_device_csr(rp, ci, va, m.cols, f, ell_width=hybrid_width if f == HYBRID else None)
        fb = dm.info().format_bytes
        time_launches(lambda: dm.spmv(x, y, stream), warmup, flush, stream)
        out[LABELS[f]] = fmt_entry(time_launches(lambda: dm.spmv(x, y, stream), steps, flush, stream), nbytes,
                                   peak, fb)
        dm.close()
    del rp, ci, va
    return {"rows": m.rows, "cols": m.cols, "nnz": int(m.nnz), "algorithmic_bytes": int(nbytes),
            "formats": out, "fastest": min(out, key=lambda k: out[k]["ms"])}


def byte_model_width(m, vs: int, row_bytes: int = 1, cap: int = 64) -> int:
    """The hybrid ELL width that moves the fewest bytes: w slots of (value,
    column) for every row against (value, column, row offset: 1 byte in a
    handle's tail) for each tail element past w, plus one 4-byte base per
    256-element tile of the tail."""
    lens = np.diff(m.row_ptr.astype(np.int64))
    best, best_b = 0, None
    for w in range(0, min(cap, int(lens.max())) + 1):
        tail = int(np.maximum(lens - w, 0).sum())
        b = w * m.rows * (vs + 4) + tail * (vs + 4 + row_bytes) + (tail + 255) // 256 * 4
        if best_b is None or b < best_b:
            best, best_b = w, b
    return best


def fp64_product(m64, x32):
    """y = A x and sum_j |a_ij x_j| in FP64 by the engine's FP64 CSR kernel
    (held to 1e-12 of the extended-precision oracle by the parity tests)."""
    import torch

    from matrix_format_performance_b200.device import CSR_SCALAR, DeviceMatrix
    rp = torch.from_numpy(m64.row_ptr.view(np.int32)).cuda()
    ci = torch.from_numpy(m64.columns.view(np.int32)).cuda()
    va = torch.from_numpy(m64.data).cuda()
    x = torch.from_numpy(x32.astype(np.float64)).cuda()
    y = torch.empty(m64.rows, dtype=torch.float64, device="cuda")
    ab = torch.empty_like(y)
    dm = DeviceMatrix.from_device_csr(rp, ci, va, m64.cols, CSR_SCALAR)
    dm.spmv(x, y)
    dm.close()
    va.abs_()
    dm = DeviceMatrix.from_device_csr(rp, ci, va, m64.cols, CSR_SCALAR)
    dm.spmv(x.abs(), ab)
    dm.close()
    torch.cuda.synchronize()
    return y, ab


def measure_lowp(name, m64, fastest_fp32, steps, warmup, flush, stream, peak):
    import torch

    from matrix_format_performance_b200 import synth
    from matrix_format_performance_b200.device import BF16, F16, DeviceMatrix
    x32 = synth.vector(0, m64.cols).astype(np.float32)
    y64, ab = fp64_product(m64, x32)
    x = torch.from_numpy(x32).cuda()
    y = torch.empty(m64.rows, device="cuda")
    nbytes = lowp_algorithmic_bytes(m64.rows, m64.cols, m64.nnz)
    out = {}
    for vt in (BF16, F16):
        for build in (DeviceMatrix.from_csr_lowp, DeviceMatrix.from_ell_lowp):
            dm = build(m64, vt, True)
            time_launches(lambda: dm.spmv(x, y, stream), warmup, flush, stream)
            e = fmt_entry(time_launches(lambda: dm.spmv(x, y, stream), steps, flush, stream), nbytes, peak)
            rel = (y.double() - y64).abs() / ab.clamp_min(1e-300)
            rel = rel[ab > 0]
            e["speedup_vs_fastest_fp32"] = round(fastest_fp32[1] / e["ms"], 3)
            e["max_rel_err_vs_fp64"] = float(rel.max()) if rel.numel() else 0.0
            e["mean_rel_err_vs_fp64"] = float(rel.mean()) if rel.numel() else 0.0
            out[dm.label] = e
            dm.close()
    best = min(out, key=lambda k: out[k]["ms"])
    return {"rows": m64.rows, "nnz": int(m64.nnz), "algorithmic_bytes": int(nbytes),
            "fastest_fp32": {"format": fastest_fp32[0], "ms": fastest_fp32[1]}, "layouts": out,
            "best": best, "best_speedup": out[best]["speedup_vs_fastest_fp32"],
            "error_reference": "FP64 product by the engine's FP64 CSR kernel; error per row relative to "
                               "sum_j |a_ij x_j|"}


def measure_load_ceiling(m, steps, warmup, flush, stream, peak, best_ms):
    """The probe's loads alone on matrix m (FP32): a floor for every format."""
    import ctypes as C

    import torch

    from matrix_format_performance_b200 import synth
    from matrix_format_performance_b200._capi import call
    va = torch.from_numpy(m.data).cuda()
    ci = torch.from_numpy(m.columns.view(np.int32)).cuda()
    x = torch.from_numpy(synth.vector(0, m.cols).astype(np.float32)).cuda()
    out = torch.empty(1 << 16, device="cuda")
    s = C.c_void_p(stream.cuda_stream)

    def probe(mode, xpath):
        return lambda: call("mfp_probe_spmv_loads", mode, xpath, m.nnz, C.c_void_p(va.data_ptr()),
                            C.c_void_p(ci.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                            out.numel(), s)
    res = {}
    for key, mode, xpath in (("stream_only", 0, 0), ("gather_only", 1, 0), ("loads_ldg", 2, 0),
                             ("loads_l2_only", 2, 1), ("loads_no_l1_allocate", 2, 2)):
        time_launches(probe(mode, xpath), warmup, flush, stream)
        ms = statistics.median(time_launches(probe(mode, xpath), steps, flush, stream))
        res[key] = {"ms": round(ms, 5)}
        if mode != 1:
            res[key]["stream_gbs"] = round(m.nnz * 8 / (ms * 1e-3) / 1e9, 1)
        if mode != 0:
            res[key]["gathers_per_ms"] = round(m.nnz / ms / 1e6, 1)
    # where the gather limit sits: the same gathers held in L1 (16 KB of x),
    # and gathers through TMA tile::gather4 (all of them, or half beside ld)
    time_launches(probe(3, 0), warmup, flush, stream)
    ms = statistics.median(time_launches(probe(3, 0), steps, flush, stream))
    res["gather_l1_resident"] = {"ms": round(ms, 5), "gathers_per_ms": round(m.nnz / ms / 1e6, 1)}

    def probe4(mode):
        return lambda: call("mfp_probe_spmv_gather4", mode, m.nnz, m.cols, C.c_void_p(ci.data_ptr()),
                            C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), out.numel(), s)
    for key, mode in (("gather_tma_gather4", 4), ("gather_half_tma_half_ld", 5)):
        time_launches(probe4(mode), warmup, flush, stream)
        ms = statistics.median(time_launches(probe4(mode), steps, flush, stream))
        n = m.nnz // 256 * 256
        res[key] = {"ms": round(ms, 5), "gathers_per_ms": round(n / ms / 1e6, 1),
                    "error_ctas": int(torch.isnan(out[:4096]).sum().item())}
    floor = min(res[k]["ms"] for k in ("loads_ldg", "loads_l2_only", "loads_no_l1_allocate"))
    nbytes = algorithmic_bytes(m.rows, m.cols, m.nnz)
    res["floor_ms"] = floor
    res["floor_algorithmic_gbs"] = round(nbytes / (floor * 1e-3) / 1e9, 1)
    res["floor_frac_of_hbm"] = round(nbytes / (floor * 1e-3) / 1e9 / peak, 4)
    res["best_format_ms"] = best_ms
    res["best_format_over_floor"] = round(best_ms / floor, 3)
    res["note"] = ("loads of an SpMV without the rows (values + column ids streamed, x gathered); units: "
                   "gathers_per_ms in millions; gather_l1_resident folds every gather into 16 KB of x")
    return res


def headline_matrix(args, rank, ws):
    """(this rank's CSR, the global matrix's rows / cols / nnz, hybrid width, row range)."""
    from matrix_format_performance_b200 import formats as F
    from matrix_format_performance_b200 import synth
    from matrix_format_performance_b200.partition import rank_shard
    t = time.time()
    if args.scaling == "weak":
        m = synth.power_law(rows=args.rows, seed=rank, cols=ROWS).astype(np.float32)
        glob = (m.rows * ws, m.cols, int(m.nnz) * ws)  # each rank's nnz differs slightly; recomputed below
        shard, lo, hi = m, 0, m.rows
    else:
        m = synth.power_law(rows=args.rows, seed=0, cols=ROWS).astype(np.float32)
        glob = (m.rows, m.cols, int(m.nnz))
        shard, lo, hi = rank_shard(m, rank, ws) if ws > 1 else (m, 0, m.rows)
    hyb_w = F.row_length_quantile(m, 2 / 3)
    log(f"[bench] rank {rank}: rows [{lo}, {hi}) of {m.rows}, {shard.nnz} nnz ({args.scaling} scaling) "
        f"in {time.time() - t:.1f}s")
    return shard, m, glob, hyb_w, (lo, hi)


def run_engine(args):
    import torch
    import torch.distributed as dist

    from matrix_format_performance_b200 import synth
    from matrix_format_performance_b200.device import FORMAT_NAMES, LABELS, DeviceMatrix, device_info

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = device_info(local)
    peak, peak_src = measured_peak()
    m, full, glob, hyb_w, (lo, hi) = headline_matrix(args, rank, ws)
    x = synth.vector(1000 + (rank if args.scaling == "weak" else 0), m.cols).astype(np.float32)
    formats = [FORMAT_NAMES[n] for n in args.formats.split(",")]
    mats = {}
    t = time.time()
    for f in formats:
        cfg = {"kernel": args.csr_kernel} if f in (0, 1, 2) and args.csr_kernel else None
        mats[f] = DeviceMatrix.build(m, f, sm_count=dev.sm_count, shared_mem=int(dev.shared_mem_per_block),
                                     hybrid_width=hyb_w, config=cfg)
    log(f"[bench] rank {rank}: formats uploaded in {time.time() - t:.1f}s (hybrid ELL width {hyb_w})")
    maxlen = int(full.row_lengths().max())
    skipped = {"GPU ELL": f"padding: width {maxlen} x {full.rows} rows = {maxlen * full.rows * 8 / 1e12:.2f} TB"}
    # bytes of one SpMV: the global matrix (strong) or this rank's block (weak)
    nbytes_rank = algorithmic_bytes(m.rows, m.cols, m.nnz)
    nbytes_global = algorithmic_bytes(*glob) if args.scaling == "strong" else None
    fbytes = {f: mats[f].info().format_bytes for f in formats}
    xt = torch.from_numpy(x).cuda()
    ys = {f: torch.empty(m.rows, device="cuda") for f in formats}
    flush = torch.empty(int(2 * dev.l2_bytes) // 4 + 1, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def step(record):
        for f in formats:
            flush.fill_(1.0)
            if record is not None:
                record[f][0].record(stream)
            mats[f].spmv(xt, ys[f], stream)
            if record is not None:
                record[f][1].record(stream)

    for _ in range(args.warmup):
        step(None)
    torch.cuda.synchronize()
    gpu_uuid = None
    try:
        gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    sampler = ClockSampler(gpu_uuid)
    if rank == 0:
        sampler.start()
        time.sleep(0.3)
    events = [{f: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for f in formats}
              for _ in range(args.steps)]
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    wall0 = torch.cuda.Event(enable_timing=True)
    wall1 = torch.cuda.Event(enable_timing=True)
    wall0.record(stream)
    for k in range(args.steps):
        step(events[k])
    wall1.record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clocks = sampler.stop() if rank == 0 else None
    per_fmt_ms = {f: [events[k][f][0].elapsed_time(events[k][f][1]) for k in range(args.steps)] for f in formats}
    kernel_ms = sum(sum(v) for v in per_fmt_ms.values())
    bracket_ms = wall0.elapsed_time(wall1)

    # e2e: host x in, host y out, through the host-buffer API (page-locked
    # vectors; one x copied in and one y copied out per step)
    e_steps = max(1, args.steps)
    hx = torch.from_numpy(x).pin_memory().numpy()
    hys = [torch.empty(m.rows, dtype=torch.float32).pin_memory().numpy() for _ in range(e_steps)]
    for f in formats:  # warm-up; the first pipelined call makes the handle's copy streams
        mats[f].spmv_host(hx, hys[0], stream)
        mats[f].spmv_host_batch([hx] * 2, hys[:1] * 2, stream)
    torch.cuda.synchronize()

    def timed(fn):
        if ws > 1:
            dist.barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    def pipelined():
        for f in formats:
            mats[f].spmv_host_batch([hx] * e_steps, hys, stream)

    def single_calls():
        for k in range(e_steps):
            for f in formats:
                mats[f].spmv_host(hx, hys[k], stream)
    e2e_ms = timed(pipelined)
    e2e_single_ms = timed(single_calls)

    # max over ranks; weak scaling sums the ranks' own bytes
    tt = torch.tensor([kernel_ms, bracket_ms, e2e_ms, e2e_single_ms], dtype=torch.float64, device="cuda")
    nb = torch.tensor([float(nbytes_rank)], dtype=torch.float64, device="cuda")
    if ws > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dist.all_reduce(nb, op=dist.ReduceOp.SUM)
    kernel_ms, bracket_ms, e2e_ms, e2e_single_ms = tt.tolist()
    job_bytes = nbytes_global if args.scaling == "strong" else int(nb.item())
    value = job_bytes * len(formats) * args.steps / (kernel_ms * 1e-3) / 1e9
    e2e_value = job_bytes * len(formats) * e_steps / (e2e_ms * 1e-3) / 1e9
    e2e_single_value = job_bytes * len(formats) * e_steps / (e2e_single_ms * 1e-3) / 1e9
    launch_counts = {f: mats[f].info().kernel_launches for f in formats}
    for f in formats:
        mats[f].close()

    if rank == 0:
        per_format = {LABELS[f]: fmt_entry(per_fmt_ms[f], nbytes_rank, peak, fbytes[f]) for f in formats}
        dom = max(formats, key=lambda f: sum(per_fmt_ms[f]))
        dom_ms = sum(per_fmt_ms[dom]) / args.steps
        achieved = nbytes_rank / (dom_ms * 1e-3) / 1e9
        tr = traffic_table().get(LABELS[dom])
        roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(achieved / peak, 4), "peak_source": f"{peak_src} (hbm_gbs)",
                    "traffic": (tr or {}).get("dram_bytes_per_launch"), "kernel": LABELS[dom],
                    "algorithmic_bytes_per_launch": nbytes_rank}
        cfg = {"workload": WORKLOAD, "rows": glob[0], "cols": glob[1], "nnz": glob[2],
               "rows_rank0": m.rows, "nnz_rank0": int(m.nnz), "formats": [LABELS[f] for f in formats],
               "skipped": skipped, "hybrid_ell_width": hyb_w,
               "l2": "flushed before every timed launch (write of 2x L2 bytes); matrix arrays also exceed L2",
               "parallelism": (f"strong: one matrix in {ws} contiguous row block(s) balanced by nonzeros, "
                               f"x replicated, no collective" if args.scaling == "strong" else
                               f"weak: one {m.rows}-row block per rank ({ws} rank(s)), no collective")}
        out = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(kernel_ms / args.steps, 5),
               "ms_per_step_bracket": round(bracket_ms / args.steps, 5),
               "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded power-law; stands in for the reference's SuiteSparse set)",
               "config": cfg, "frac_of_hbm_peak": round(value / peak, 4),
               "per_format": per_format, "roofline": roofline,
               "e2e": {"value": round(e2e_value, 1), "unit": UNIT,
                       "h2d_bytes_per_step": int(m.cols * 4 * len(formats) * ws),
                       "d2h_bytes_per_step": int(glob[0] * 4 * len(formats)) if args.scaling == "strong"
                       else int(m.rows * 4 * len(formats) * ws), "steps": e_steps,
                       "mode": "mfp_matrix_spmv_host_batch per format over the steps: a step's copies overlap "
                               "the neighbouring steps' kernels",
                       "single_call_value": round(e2e_single_value, 1)},
               "gpu_launches": args.steps * sum(launch_counts[f] for f in formats),
               "clocks": clocks}
        if ws == 1 and not args.no_extras:
            extras_t = time.time()
            sampler2 = ClockSampler(gpu_uuid)
            sampler2.start()
            out.update(run_extras(args, full, x, per_format, flush, stream, peak, hyb_w))
            out["extras_clocks"] = sampler2.stop()
            out["extras_wall_s"] = round(time.time() - extras_t, 1)
        if ws == 1 and not args.no_cpu_baseline:
            try:
                cb = cpu_baseline_reference(full, threads=1, reps=args.cpu_reps)
                out["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            except Exception as e:  # the baseline is reported, never required for the GPU number
                out["cpu_baseline"] = {"error": str(e)}
        print(json.dumps(out), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_extras(args, power_law, x, per_format, flush, stream, peak, hyb_w):
    """The rest of the metric on one GPU: stencil / banded per format, FP64,
    reduced precision, the load ceiling of the power-law matrix and its
    hybrid at the byte model's ELL width."""
    from matrix_format_performance_b200 import formats as F
    from matrix_format_performance_b200 import synth
    from matrix_format_performance_b200.device import (COO, CSR_ADAPTIVE, CSR_SCALAR, CSR_VECTOR, ELL, HYBRID,
                                                       SCOO)
    steps, warmup = args.steps, args.warmup
    plain = [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE, ELL, COO, SCOO, HYBRID]
    no_ell = [f for f in plain if f != ELL]
    res = {"per_config": {}, "fp64": {}, "lowp": {}}
    best_pl = min(per_format.values(), key=lambda e: e["ms"])["ms"]
    t = time.time()
    res["load_ceiling"] = {"power_law_4M": measure_load_ceiling(power_law, steps, warmup, flush, stream, peak,
                                                                best_pl)}
    log(f"[bench] load ceiling in {time.time() - t:.1f}s")
    # the hybrid at the byte model's ELL width beside the 2/3-quantile width of
    # the headline (the reference's own sweep varies the width too)
    t = time.time()
    wb = byte_model_width(power_law, 4)
    hw = {"quantile_width": hyb_w, "byte_model_width": wb,
          "note": "byte model: w*rows*(4+4) + tail*(4+4+1) + tail tiles*4 bytes, minimised over w"}
    for label, w in (("quantile", hyb_w), ("byte_model", wb)):
        e = measure_plain("power_law_4M", power_law, [HYBRID], steps, warmup, flush, stream, peak, w)
        hw[label] = e["formats"]["GPU Hybrid (atomic)"]
        hw[label]["format_bytes_over_algorithmic"] = round(hw[label]["format_bytes"] / e["algorithmic_bytes"], 3)
    res["hybrid_widths"] = {"power_law_4M": hw}
    log(f"[bench] hybrid widths in {time.time() - t:.1f}s")
    pl64 = synth.power_law(seed=0)
    t = time.time()
    res["fp64"]["power_law_4M"] = measure_plain("power_law_4M", pl64, no_ell, steps, warmup, flush, stream, peak,
                                                hyb_w)
    del pl64
    log(f"[bench] power-law FP64 in {time.time() - t:.1f}s")
    for name, gen in (("stencil27_128", lambda: synth.stencil_27(128, seed=0)),
                      ("banded_8M", lambda: synth.banded(seed=0))):
        t = time.time()
        m64 = gen()
        w = F.row_length_quantile(m64, 2 / 3)
        m32 = m64.astype(np.float32)
        res["per_config"][name] = measure_plain(name, m32, plain, steps, warmup, flush, stream, peak, w)
        del m32
        res["fp64"][name] = measure_plain(name, m64, plain, steps, warmup, flush, stream, peak, w)
        pc = res["per_config"][name]
        fastest = (pc["fastest"], pc["formats"][pc["fastest"]]["ms"])
        res["lowp"][name] = measure_lowp(name, m64, fastest, steps, warmup, flush, stream, peak)
        del m64
        log(f"[bench] {name} in {time.time() - t:.1f}s")
    return res


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--scaling", choices=["strong", "weak"], default="strong",
                    help="multi-GPU: split one matrix by rows (strong) or one matrix per rank (weak)")
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--cpu-reps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="only the power-law FP32 headline")
    ap.add_argument("--csr-kernel", type=int, default=0,
                    help="CSR kernel: 0 auto, 1 row-block, 2 streaming (2048-element chunks), 3 streaming (1024)")
    ap.add_argument("--formats", default="csr,csr_vector,csr_adaptive,coo,scoo,hybrid",
                    help="comma list of: csr, csr_vector, csr_adaptive, coo, scoo, hybrid")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "engine":
        log("[bench] warm-up raised to 3 (the timing rules require at least 3)")
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
