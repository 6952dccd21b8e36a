"""The cuSPARSE yardstick computes the same product (tolerance check against
the oracle), so its times are comparable with the engine's."""
import numpy as np
import pytest

from matrix_format_performance_b200 import synth


@pytest.mark.gpu
@pytest.mark.parametrize("fmt,alg", [(0, 0), (0, 1), (0, 2), (1, 0)])
def test_cusparse_matches_oracle(oracle_lib, fmt, alg):
    import torch
    from matrix_format_performance_b200 import yardstick as Y
    m = synth.power_law(rows=30_000, seed=9).astype(np.float32)
    x = synth.vector(2, m.cols).astype(np.float32)
    idx = m.row_ptr if fmt == 0 else np.repeat(np.arange(m.rows, dtype=np.uint32), np.diff(m.row_ptr.astype(np.int64)))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    y = torch.full((m.rows,), float("nan"), device="cuda")
    Y.spmv(fmt, alg, m.rows, m.cols, m.nnz, t(idx.view(np.int32)), t(m.columns.view(np.int32)), t(m.data), t(x), y)
    ys, ab = oracle_lib.csr_spmv_exact(m.rows, m.row_ptr, m.columns, m.data.astype(np.float64), x.astype(np.float64))
    assert np.all(np.abs(y.cpu().numpy().astype(np.float64) - ys) <= 1e-5 * ab)
