#!/usr/bin/env python
"""SpMV benchmark on the power-law configuration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Workload (one "step"): y = A*x once through each plain format the layout
admits -- CSR scalar, CSR vector, CSR-Adaptive, COO, SCOO, hybrid ELL+COO --
on a 4,194,304 x 4,194,304 matrix whose row lengths are Zipf(2.0) clipped to
[1, 50000] (distinct uniform columns, values and x uniform[-1, 1], FP32).
ELL is skipped: its padding (width 50,000 x 4,194,304 rows) does not fit,
which is also why the reference's driver drops such matrices.

value    algorithmic bytes of all SpMVs of all ranks / max-over-ranks device
         time of the kernels (CUDA events on the launching stream; L2 flushed
         before every launch).  Bytes per SpMV:
         nnz*(4+4) + (rows+1)*4 + cols*4 + rows*4.
e2e      the same bytes / time of mfp_matrix_spmv_host (host x in, host y out,
         page-locked buffers, copies inside the timed region).
Multi-GPU: one rank per GPU, each owns its own 4,194,304-row block of a
global matrix (weak scaling); no collective in the data path.

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

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SpMV GB/s & % HBM peak per format; selector/BF16 speedup vs plain at tolerance"
UNIT = "GB/s"
FALLBACK_HBM_GBS = 6650.0
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


def build_workload(rows: int, seed: int):
    from matrix_format_performance_b200 import synth
    t = time.time()
    m = synth.power_law(rows=rows, seed=seed, cols=4_194_304).astype(np.float32)
    x = synth.vector(1000, m.cols).astype(np.float32)
    log(f"[bench] generated power-law block seed={seed}: {m.rows} rows, {m.nnz} nnz in {time.time() - t:.1f}s")
    return m, x


def cpu_baseline_reference(m, threads: int, reps: int, warmup: int = 1):
    """Times the reference CPU loop (oracle/_ref) or, if absent, the oracle port."""
    from oracle import load_oracle, load_ref
    ref = load_ref()
    nbytes = algorithmic_bytes(m.rows, m.cols, m.nnz)
    y = np.empty(m.rows, np.float32)
    times = []
    if ref is not None:
        import ctypes as C
        data64 = m.data.astype(np.float64)
        h = ref.lib.ref_bench_create(0, threads, m.rows, m.cols, C.c_void_p(m.row_ptr.ctypes.data),
                                     C.c_void_p(m.columns.ctypes.data), C.c_void_p(data64.ctypes.data))
        used = len(range(threads))
        for i in range(warmup + reps):
            t = ref.lib.ref_bench_run(h, C.c_void_p(y.ctypes.data))
            if i >= warmup:
                times.append(t)
        ref.lib.ref_bench_destroy(h)
        kind = "reference"
    else:
        orc = load_oracle()
        x = np.ones(m.cols, np.float32)
        for i in range(warmup + reps):
            _, t = orc.csr_spmv_parallel(threads, m.rows, m.row_ptr, m.columns, m.data, x)
            if i >= warmup:
                times.append(t)
        used = threads
        kind = "port"
    mean = sum(times) / len(times)
    return {"value": nbytes / mean / 1e9, "unit": UNIT, "cores": used, "kind": kind,
            "sample": f"full matrix ({m.rows} rows, {m.nnz} nnz), FP32 CSR, x = 1, "
                      f"{used} thread(s), mean of {reps} passes after {warmup} warm-up",
            "seconds_per_spmv": mean}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    m, _ = build_workload(args.rows, seed=0)
    threads = os.cpu_count() or 1
    t0 = time.time()
    cb = cpu_baseline_reference(m, threads, reps=args.steps, warmup=args.warmup)
    out = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["seconds_per_spmv"] * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded)", "config": config_dict(m, ws, formats=["CPU CSR (reference loop)"]),
           "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
           "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "wall_s": time.time() - t0}
    print(json.dumps(out), flush=True)


def config_dict(m, ws, formats, skipped=None):
    return {"workload": WORKLOAD, "rows_per_rank": m.rows, "cols": m.cols, "nnz_per_rank": int(m.nnz),
            "formats": formats, "skipped": skipped or {},
            "l2": "flushed before every timed launch (write of 2x L2 bytes); matrix arrays also exceed L2",
            "parallelism": f"row blocks, one {m.rows}-row block per rank ({ws} rank(s)), no collective"}


def run_engine(args):
    import torch
    import torch.distributed as dist

    from matrix_format_performance_b200 import formats as F
    from matrix_format_performance_b200.device import LABELS, DeviceMatrix, device_info

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = device_info(local)
    m, x = build_workload(args.rows, seed=rank)
    hyb_w = F.row_length_quantile(m, 2 / 3)
    from matrix_format_performance_b200.device import FORMAT_NAMES
    formats = [FORMAT_NAMES[n] for n in args.formats.split(",")]
    mats = {}
    t = time.time()
    for f in formats:
        cfg = {"kernel": args.csr_kernel} if f in (0, 1, 2) and args.csr_kernel else None
        mats[f] = DeviceMatrix.build(m, f, sm_count=dev.sm_count, shared_mem=int(dev.shared_mem_per_block),
                                     hybrid_width=hyb_w, config=cfg)
    log(f"[bench] rank {rank}: formats uploaded in {time.time() - t:.1f}s (hybrid ELL width {hyb_w})")
    skipped = {"GPU ELL": f"padding: width {int(m.row_lengths().max())} x {m.rows} rows "
                          f"= {int(m.row_lengths().max()) * m.rows * 8 / 1e12:.2f} TB"}
    nbytes = algorithmic_bytes(m.rows, m.cols, m.nnz)
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

    # e2e: host x in, host y out, through mfp_matrix_spmv_host
    hx = torch.from_numpy(x).pin_memory().numpy()
    hy = torch.empty(m.rows, dtype=torch.float32).pin_memory().numpy()
    for f in formats:
        mats[f].spmv_host(hx, hy, stream)
    e_steps = max(1, min(args.steps, 5))
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e_steps):
        for f in formats:
            mats[f].spmv_host(hx, hy, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)

    # max over ranks
    tt = torch.tensor([kernel_ms, bracket_ms, e2e_ms], dtype=torch.float64, device="cuda")
    if ws > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    kernel_ms, bracket_ms, e2e_ms = tt.tolist()
    total_bytes = nbytes * len(formats) * args.steps * ws
    value = total_bytes / (kernel_ms * 1e-3) / 1e9
    e2e_value = nbytes * len(formats) * e_steps * ws / (e2e_ms * 1e-3) / 1e9

    if rank == 0:
        peak, peak_src = measured_peak()
        per_format = {}
        for f in formats:
            mean_ms = sum(per_fmt_ms[f]) / len(per_fmt_ms[f])
            gbs = nbytes / (mean_ms * 1e-3) / 1e9
            per_format[LABELS[f]] = {"ms": round(mean_ms, 5), "gbs": round(gbs, 1), "frac": round(gbs / peak, 4),
                                     "format_bytes": int(fbytes[f]),
                                     "format_gbs": round(fbytes[f] / (mean_ms * 1e-3) / 1e9, 1)}
        dom = max(formats, key=lambda f: sum(per_fmt_ms[f]))
        dom_ms = sum(per_fmt_ms[dom]) / args.steps
        achieved = nbytes / (dom_ms * 1e-3) / 1e9
        tr = traffic_table().get(LABELS[dom])
        roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(achieved / peak, 4), "peak_source": f"{peak_src} (hbm_gbs)",
                    "traffic": (tr or {}).get("dram_bytes_per_launch"), "kernel": LABELS[dom],
                    "algorithmic_bytes_per_launch": nbytes}
        out = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(kernel_ms / args.steps, 5),
               "ms_per_step_bracket": round(bracket_ms / args.steps, 5),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded power-law; stands in for the reference's SuiteSparse set)",
               "config": config_dict(m, ws, [LABELS[f] for f in formats], skipped),
               "frac_of_hbm_peak": round(value / peak, 4),
               "per_format": per_format, "roofline": roofline,
               "e2e": {"value": round(e2e_value, 1), "unit": UNIT,
                       "h2d_bytes_per_step": int(m.cols * 4 * len(formats) * ws),
                       "d2h_bytes_per_step": int(m.rows * 4 * len(formats) * ws), "steps": e_steps},
               "gpu_launches": args.steps * sum(mats[f].info().kernel_launches for f in formats),
               "clocks": clocks}
        if ws == 1 and not args.no_cpu_baseline:
            try:
                cb = cpu_baseline_reference(m, threads=1, reps=args.cpu_reps)
                out["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            except Exception as e:  # the baseline is reported, never required for the GPU number
                out["cpu_baseline"] = {"error": str(e)}
        print(json.dumps(out), flush=True)
    for f in formats:
        mats[f].close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--rows", type=int, default=4_194_304)
    ap.add_argument("--cpu-reps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
