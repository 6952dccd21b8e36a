"""bench.py: its helpers and the JSON line the driver reads.

CPU: the hybrid ELL width of the byte model; the reference arm's line.
GPU: the engine arm's line on a small power-law matrix.
"""
import importlib.util
import pathlib

import numpy as np
import pytest

from matrix_format_performance_b200 import synth


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", pathlib.Path(__file__).parents[1] / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_bench_byte_model_width():
    """bench.byte_model_width: the hybrid ELL width that moves the fewest
    bytes, checked against a direct count on small matrices."""
    bench = _bench()
    for m, vs in ((synth.power_law(rows=50_000, seed=3), 4), (synth.stencil_27(12), 8), (synth.uniform(3000, 0, 9), 4)):
        lens = np.diff(m.row_ptr.astype(np.int64))

        def cost(w):
            tail = int(np.maximum(lens - w, 0).sum())
            return w * m.rows * (vs + 4) + tail * (vs + 5) + (tail + 255) // 256 * 4
        w = bench.byte_model_width(m, vs)
        assert cost(w) == min(cost(k) for k in range(0, min(64, int(lens.max())) + 1))


def _run_bench(*args, timeout=900):
    import json
    import os
    import subprocess
    import sys
    root = pathlib.Path(__file__).parents[1]
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, str(root / "bench.py"), *args], cwd=root, env=env, capture_output=True,
                         text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_reference_arm_line():
    """bench.py --impl reference on a small matrix: the driver's keys, a
    positive GB/s from the reference's own loop, e2e with no copies."""
    import pytest
    oracle = pytest.importorskip("oracle")
    try:
        oracle.load_synth()
    except Exception as e:  # the generator library is built by the oracle recipe
        pytest.skip(f"oracle generator not built: {e}")
    d = _run_bench("--impl", "reference", "--rows", "20000", "--steps", "2", "--warmup", "1")
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1


@pytest.mark.gpu
def test_engine_arm_line():
    """bench.py on a 200,000-row power-law matrix: every key of the driver's
    contract, the roofline and e2e objects, clocks and the launch count."""
    d = _run_bench("--rows", "200000", "--steps", "3", "--warmup", "3", "--no-extras", "--no-cpu-baseline")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "gpu_launches", "clocks", "per_format"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    assert "workload" in d["config"]
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and 0 < r["frac"] and r["peak"] > 0
    assert abs(r["achieved"] / r["peak"] - r["frac"]) < 1e-3
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] >= 3 * len(d["per_format"])
