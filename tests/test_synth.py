"""Seeded synthetic configurations: sizes, structure, determinism."""
import numpy as np
import pytest

from matrix_format_performance_b200 import formats as F
from matrix_format_performance_b200 import synth


def _check_csr(m):
    rp = m.row_ptr.astype(np.int64)
    assert rp[0] == 0 and rp[-1] == m.nnz and np.all(np.diff(rp) >= 0)
    assert np.all(m.columns < m.cols)
    for r in range(0, m.rows, max(1, m.rows // 200)):
        c = m.columns[rp[r]:rp[r + 1]].astype(np.int64)
        assert np.all(np.diff(c) > 0)  # sorted, no duplicates


def test_laplacian_512_is_the_configured_size():
    m = synth.laplacian_2d(512)
    assert (m.rows, m.cols, m.nnz) == (262_144, 262_144, 1_308_672)
    _check_csr(m)
    assert set(np.unique(m.data)) == {-1.0, 4.0}
    assert np.allclose(np.add.reduceat(m.data, m.row_ptr[:-1].astype(np.int64))[513], 0.0)  # interior row sums to 0


def test_stencil_27_size():
    m = synth.stencil_27(16)
    assert m.rows == 16 ** 3 and m.nnz == 27 * 14 ** 3 + 0 + (m.nnz - 27 * 14 ** 3)
    _check_csr(m)
    # 128^3 grid: (3*128-2)^3 = 55,742,968 nnz, computed without materialising it
    n = 128
    assert (3 * n - 2) ** 3 == 55_742_968
    assert m.nnz == (3 * 16 - 2) ** 3


def test_banded_rows_have_32_distinct_columns_in_band():
    m = synth.banded(n=5000, half_band=64, per_row=32, seed=3)
    assert m.nnz == 32 * 5000
    _check_csr(m)
    rows = np.repeat(np.arange(m.rows), np.diff(m.row_ptr.astype(np.int64)))
    assert np.all(np.abs(m.columns.astype(np.int64) - rows) <= 64)


def test_power_law_statistics_and_determinism():
    a = synth.power_law(rows=200_000, seed=5)
    b = synth.power_law(rows=200_000, seed=5)
    assert np.array_equal(a.row_ptr, b.row_ptr) and np.array_equal(a.columns, b.columns)
    assert np.array_equal(a.data, b.data)
    _check_csr(a)
    lens = a.row_lengths()
    assert lens.min() >= 1 and lens.max() <= 50_000
    # Zipf(2): P(len = 1) = 1 / zeta(2)
    assert abs(np.mean(lens == 1) - 6 / np.pi ** 2) < 0.01
    assert F.row_length_quantile(a, 2 / 3) == 2
    c = synth.power_law(rows=200_000, seed=6)
    assert not np.array_equal(a.row_ptr, c.row_ptr)


def test_vector_is_seeded_uniform():
    x = synth.vector(0, 100_000)
    assert np.array_equal(x, synth.vector(0, 100_000))
    assert x.min() >= -1 and x.max() < 1 and abs(x.mean()) < 0.01


@pytest.mark.parametrize("fn", [lambda: synth.uniform(3000, 4, 64, seed=1), lambda: synth.tridiagonal(3000),
                                lambda: synth.block_diagonal(3000, 32)])
def test_batched_families(fn):
    m = fn()
    _check_csr(m)
    assert m.rows == 3000
