"""CPU tests of bench.py's helpers (no GPU): the hybrid ELL width of the
byte model."""
import importlib.util
import pathlib

import numpy as np

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
            return w * m.rows * (vs + 4) + tail * (vs + 6) + (tail + 255) // 256 * 4
        w = bench.byte_model_width(m, vs)
        assert cost(w) == min(cost(k) for k in range(0, min(64, int(lens.max())) + 1))
