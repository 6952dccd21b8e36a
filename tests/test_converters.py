"""The engine's host converters (libmfp_spmv.so) are bit-exact with the reference.

Runs on CPU: the converters are plain host code in the C ABI library.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden
from matrix_format_performance_b200 import formats as F
from matrix_format_performance_b200 import synth
from matrix_format_performance_b200._capi import MfpError


def _coo(g):
    return F.matrix_class(int(g["rows"][0]), int(g["cols"][0]), g["row_ids"], g["col_ids"], g["values"])


@pytest.mark.parametrize("case", golden_cases())
@pytest.mark.parametrize("dt,s", [(np.float32, "f32"), (np.float64, "f64")])
def test_converters_match_reference_fixtures(case, dt, s):
    g = load_golden(case)
    c = F.csr_matrix_class(_coo(g), dt)
    assert np.array_equal(c.row_ptr, g[f"csr_row_ptr_{s}"])
    assert np.array_equal(c.columns, g[f"csr_columns_{s}"])
    assert np.array_equal(c.data, g[f"csr_data_{s}"])
    st = F.get_rows_statistics(c)
    assert [st.min_elements_in_rows, st.max_elements_in_rows, st.avg_elements_in_rows] == list(g["stats_u32"])
    assert st.elements_in_rows_std_deviation == g["stats_std"][0]
    assert F.ell_matrix_class.estimate_size(c) == int(g[f"ell_width_{s}"][0]) * c.rows
    if f"ell_data_{s}" in g:
        e = F.ell_matrix_class(c)
        assert e.elements_in_rows == int(g[f"ell_width_{s}"][0])
        assert np.array_equal(e.data, g[f"ell_data_{s}"]) and np.array_equal(e.columns, g[f"ell_columns_{s}"])
    o = F.coo_matrix_class(c)
    assert np.array_equal(o.data, g[f"coo_data_{s}"]) and np.array_equal(o.cols_, g[f"coo_cols_{s}"])
    assert np.array_equal(o.rows_, g[f"coo_rows_{s}"])
    h = F.hybrid_matrix_class(c)
    if f"hyb_ell_data_{s}" in g:
        h.allocate(c, 0.2)
        assert h.ell_matrix.elements_in_rows == int(g[f"hyb_width_{s}"][0])
        assert np.array_equal(h.ell_matrix.data, g[f"hyb_ell_data_{s}"])
        assert np.array_equal(h.ell_matrix.columns, g[f"hyb_ell_columns_{s}"])
    else:
        hw = int(g[f"hyb_width_{s}"][0])
        h.coo_matrix = F.coo_matrix_class(c, hw)
    assert np.array_equal(h.coo_matrix.data, g[f"hyb_coo_data_{s}"])
    assert np.array_equal(h.coo_matrix.cols_, g[f"hyb_coo_cols_{s}"])
    assert np.array_equal(h.coo_matrix.rows_, g[f"hyb_coo_rows_{s}"])
    for tag, sm, smem in (("scoo", 148, 49152), ("scoo_small", 4, 1024)):
        sc = F.scoo_matrix_class(sm, smem, c)
        assert [sc.slices_count, sc.slice_size, sc.lane_size] == list(g[f"{tag}_params_{s}"])
        assert np.array_equal(sc.values, g[f"{tag}_values_{s}"])
        assert np.array_equal(sc.c_index, g[f"{tag}_c_index_{s}"])
        assert np.array_equal(sc.r_index, g[f"{tag}_r_index_{s}"])
        assert np.array_equal(sc.slices_ptr, g[f"{tag}_slices_ptr_{s}"])
    assert np.array_equal(F.fill_row_blocks(c, 64), g["rowblocks"])


def test_hybrid_width_rule_percent_sweep(oracle_lib):
    g = load_golden("powerlaw_small")
    c = F.csr_matrix_class(_coo(g), np.float32)
    for pct in (0.0, 0.2, 0.35, 0.7, 1.0):
        h = F.hybrid_matrix_class(c)
        import ctypes as C
        w = C.c_uint32()
        from matrix_format_performance_b200._capi import call
        call("mfp_hybrid_width", c.rows, F.ptr(c.row_ptr), pct, C.byref(w))
        assert w.value == oracle_lib.hybrid_width(c.rows, c.row_ptr, pct)


def test_row_length_quantile():
    rp = np.array([0, 1, 2, 3, 5, 8, 13], np.uint32)  # lengths 1,1,1,2,3,5
    c = F.csr_matrix_class.from_arrays(6, 20, rp, np.zeros(13, np.uint32), np.ones(13, np.float32))
    assert F.row_length_quantile(c, 0.5) == 1
    assert F.row_length_quantile(c, 2 / 3) == 2
    assert F.row_length_quantile(c, 1.0) == 5


def test_fill_row_blocks_other_bin_sizes(oracle_lib):
    g = load_golden("powerlaw_small")
    c = F.csr_matrix_class(_coo(g), np.float32)
    for per_wg in (1, 7, 64, 256, 4096):
        assert np.array_equal(F.fill_row_blocks(c, per_wg), oracle_lib.fill_row_blocks(c.rows, c.row_ptr, per_wg))


def test_rejects_non_general_storage():
    g = load_golden("laplacian_16")
    m = _coo(g)
    m.storage_scheme = 1
    with pytest.raises(MfpError, match="Only general matrices"):
        F.csr_matrix_class(m, np.float32)


def test_rejects_out_of_range_ids():
    m = F.matrix_class(3, 3, [0, 3], [0, 1], [1.0, 2.0])
    with pytest.raises(MfpError, match="row id 3"):
        F.csr_matrix_class(m, np.float32)
    m = F.matrix_class(3, 3, [0, 1], [0, 9], [1.0, 2.0])
    with pytest.raises(MfpError, match="col id 9"):
        F.csr_matrix_class(m, np.float64)


def test_empty_matrix_and_zero_rows():
    m = F.matrix_class(5, 4, [], [], [])
    c = F.csr_matrix_class(m, np.float32)
    assert c.nnz == 0 and np.array_equal(c.row_ptr, np.zeros(6, np.uint32))
    st = F.get_rows_statistics(c)
    assert (st.min_elements_in_rows, st.max_elements_in_rows, st.avg_elements_in_rows) == (0, 0, 0)
    z = F.csr_matrix_class.from_arrays(0, 4, np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.float32))
    with pytest.raises(MfpError):
        F.get_rows_statistics(z)


def test_compare_results_matches_reference_rule():
    a = np.array([1.0, 2.0, 3.0], np.float32)
    err, bad = F.compare_results(a, a.copy())
    assert err == 0.0 and bad is None
    b = a.copy()
    b[1] = 2.5
    err, bad = F.compare_results(b, a)
    assert err == pytest.approx(0.25 / 14.0) and bad == 1


@pytest.mark.parametrize("kind", ["power_law", "stencil", "banded"])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_scoo_sort_cols_orders_each_slice_by_column_stably(kind, dt):
    """The reference's disabled sort_cols block (scoo_matrix_class.cpp:102-138)
    restated with a stable sort: per slice, the elements ordered by column,
    equal columns in CSR order; slices_ptr and parameters unchanged."""
    m = {"power_law": lambda: synth.power_law(rows=40_000, seed=3),
         "stencil": lambda: synth.stencil_27(24, seed=1),
         "banded": lambda: synth.banded(n=30_000, seed=2)}[kind]().astype(dt)
    plain = F.scoo_matrix_class(148, 49152, m)
    srt = F.scoo_matrix_class(148, 49152, m, sort_cols=True)
    np.testing.assert_array_equal(srt.slices_ptr, plain.slices_ptr)
    assert (srt.slices_count, srt.slice_size, srt.lane_size) == (plain.slices_count, plain.slice_size,
                                                                   plain.lane_size)
    sp = plain.slices_ptr
    for s in range(plain.slices_count):
        b, e = int(sp[s]), int(sp[s + 1])
        if b >= e:
            continue
        p = np.argsort(plain.c_index[b:e], kind="stable")
        np.testing.assert_array_equal(srt.c_index[b:e], plain.c_index[b:e][p])
        np.testing.assert_array_equal(srt.r_index[b:e], plain.r_index[b:e][p])
        np.testing.assert_array_equal(srt.values[b:e].view(np.uint8), plain.values[b:e][p].view(np.uint8))
