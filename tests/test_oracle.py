"""Pins the oracle (oracle/oracle.c) to the reference.

Every array the oracle restates is compared bit for bit with what the
reference's own code returned for the same input: the committed fixtures in
tests/golden/ (made by tests/golden/make_golden.py from the compiled
reference), and, when oracle/_ref was built here, fresh random inputs run
through the reference live.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden


def _csr(g, s):
    return g[f"csr_row_ptr_{s}"], g[f"csr_columns_{s}"], g[f"csr_data_{s}"]


@pytest.mark.parametrize("case", golden_cases())
@pytest.mark.parametrize("dt,s", [(np.float32, "f32"), (np.float64, "f64")])
def test_oracle_converters_match_golden(oracle_lib, case, dt, s):
    g = load_golden(case)
    rows = int(g["rows"][0])
    rp, ci, d = oracle_lib.csr_from_coo(rows, g["row_ids"], g["col_ids"], g["values"], dt)
    grp, gci, gd = _csr(g, s)
    assert np.array_equal(rp, grp) and np.array_equal(ci, gci) and np.array_equal(d, gd)
    mn, mx, avg, sd = oracle_lib.rows_statistics(rows, rp)
    assert [mn, mx, avg] == list(g["stats_u32"]) and sd == g["stats_std"][0]
    w = int(g[f"ell_width_{s}"][0])
    assert w == mx
    if f"ell_data_{s}" in g:
        ed, ec = oracle_lib.ell(rows, rp, ci, d, w)
        assert np.array_equal(ed, g[f"ell_data_{s}"]) and np.array_equal(ec, g[f"ell_columns_{s}"])
    cd, cc, cr = oracle_lib.coo(rows, rp, ci, d, 0)
    assert np.array_equal(cd, g[f"coo_data_{s}"]) and np.array_equal(cc, g[f"coo_cols_{s}"])
    assert np.array_equal(cr, g[f"coo_rows_{s}"])
    hw = oracle_lib.hybrid_width(rows, rp, 0.2)
    assert hw == int(g[f"hyb_width_{s}"][0])
    hd, hc, hr = oracle_lib.coo(rows, rp, ci, d, hw)
    assert np.array_equal(hd, g[f"hyb_coo_data_{s}"]) and np.array_equal(hr, g[f"hyb_coo_rows_{s}"])
    if f"hyb_ell_data_{s}" in g:
        ed, ec = oracle_lib.ell(rows, rp, ci, d, hw)
        assert np.array_equal(ed, g[f"hyb_ell_data_{s}"]) and np.array_equal(ec, g[f"hyb_ell_columns_{s}"])
    for tag, sm, smem in (("scoo", 148, 49152), ("scoo_small", 4, 1024)):
        prm, v, cx, rx, sp = oracle_lib.scoo(rows, rp, ci, d, sm, smem)
        assert list(prm) == list(g[f"{tag}_params_{s}"])
        assert np.array_equal(v, g[f"{tag}_values_{s}"]) and np.array_equal(cx, g[f"{tag}_c_index_{s}"])
        assert np.array_equal(rx, g[f"{tag}_r_index_{s}"]) and np.array_equal(sp, g[f"{tag}_slices_ptr_{s}"])
    assert np.array_equal(oracle_lib.fill_row_blocks(rows, grp), g["rowblocks"])


@pytest.mark.parametrize("case", golden_cases())
@pytest.mark.parametrize("dt,s", [(np.float32, "f32"), (np.float64, "f64")])
def test_oracle_spmv_matches_golden(oracle_lib, case, dt, s):
    g = load_golden(case)
    rows, cols = int(g["rows"][0]), int(g["cols"][0])
    rp, ci, d = _csr(g, s)
    one = np.ones(cols, dt)
    assert np.array_equal(oracle_lib.csr_spmv(rows, rp, ci, d, one), g[f"y1_{s}"])
    assert np.array_equal(oracle_lib.csr_spmv(rows, rp, ci, d, one, reduce_order=True), g[f"y1ro_{s}"])
    x = g["x"].astype(dt)
    assert np.array_equal(oracle_lib.csr_spmv(rows, rp, ci, d, x), g[f"yx_{s}"])
    assert np.array_equal(oracle_lib.csr_spmv(rows, rp, ci, d, x, reduce_order=True), g[f"yxro_{s}"])
    yp, _ = oracle_lib.csr_spmv_parallel(3, rows, rp, ci, d, x)
    assert np.array_equal(yp, g[f"yx_{s}"])
    if f"ell_data_{s}" in g:
        w = int(g[f"ell_width_{s}"][0])
        ye = oracle_lib.ell_spmv(rows, w, g[f"ell_data_{s}"], g[f"ell_columns_{s}"], x)
        # padding adds +0 to every row sum: same bits as the CSR loop
        assert np.array_equal(ye, g[f"yx_{s}"])


def test_oracle_extended_precision_is_closer(oracle_lib):
    g = load_golden("powerlaw_small")
    rows = int(g["rows"][0])
    rp, ci, d = _csr(g, "f64")
    x = g["x"]
    y, ab = oracle_lib.csr_spmv_exact(rows, rp, ci, d, x)
    y64 = oracle_lib.csr_spmv(rows, rp, ci, d, x)
    assert np.all(np.abs(y - y64) <= 1e-13 * np.maximum(ab, 1e-300))
    assert np.all(ab >= np.abs(y))


def _random_coo(rng, rows, cols, max_len):
    lens = rng.integers(0, max_len + 1, size=rows)
    r, c = [], []
    for i, n in enumerate(lens):
        n = min(int(n), cols)
        r += [i] * n
        c += list(rng.choice(cols, size=n, replace=False))
    v = rng.uniform(-1, 1, size=len(r))
    p = rng.permutation(len(r))
    from matrix_format_performance_b200.formats import matrix_class
    return matrix_class(rows, cols, np.array(r, np.uint32)[p], np.array(c, np.uint32)[p], v[p])


@pytest.mark.parametrize("seed", range(4))
def test_oracle_matches_live_reference(oracle_lib, ref_lib, seed):
    if ref_lib is None:
        pytest.skip("oracle/_ref not built (no reference sources on this machine)")
    rng = np.random.default_rng(1000 + seed)
    m = _random_coo(rng, int(rng.integers(1, 400)), int(rng.integers(1, 300)), int(rng.integers(1, 40)))
    for dt in (np.float32, np.float64):
        rp, ci, d = ref_lib.csr(m, dt)
        orp, oci, od = oracle_lib.csr_from_coo(m.rows, m.row_ids, m.col_ids, m.data, dt)
        assert np.array_equal(rp, orp) and np.array_equal(ci, oci) and np.array_equal(d, od)
        assert ref_lib.rows_statistics(m) == oracle_lib.rows_statistics(m.rows, rp)
        for sm, smem in ((148, 49152), (3, 4096), (1, 256)):
            prm, v, cx, rx, sp = ref_lib.scoo(m, dt, sm, smem)
            oprm, ov, ocx, orx, osp = oracle_lib.scoo(m.rows, rp, ci, d, sm, smem)
            assert prm == oprm and np.array_equal(sp, osp) and np.array_equal(rx, orx)
        assert np.array_equal(ref_lib.fill_row_blocks(m.rows, rp), oracle_lib.fill_row_blocks(m.rows, rp))
        y = ref_lib.spmv_ones(m, dt)
        assert np.array_equal(y, oracle_lib.csr_spmv(m.rows, rp, ci, d, np.ones(m.cols, dt)))
        for pct in (0.0, 0.2, 0.35, 1.0):
            w, *_ = ref_lib.hybrid(m, dt, pct)
            assert w == oracle_lib.hybrid_width(m.rows, rp, pct)


def test_reference_measurement_record(ref_lib):
    if ref_lib is None:
        pytest.skip("oracle/_ref not built")
    from matrix_format_performance_b200.formats import measurement_class
    e, bw, fl = ref_lib.measurement("GPU CSR", 1.25e-4, 123456789.0, 2.5e7)
    m = measurement_class("GPU CSR", 1.25e-4, 123456789.0, 2.5e7)
    assert (m.elapsed, m.effective_bandwidth, m.computational_throughput) == (e, bw, fl)
