"""On-device format conversion (mfp_dev_*) against the host converters (needs a B200).

The host converters are pinned to the reference's own (test_converters.py,
test_oracle.py); the device kernels must reproduce their arrays bit for bit:
ELL / COO / hybrid tail / SCOO from CSR, row statistics, SCOO x windows, and
CSR from COO triplets in any input order (stable for repeated entries).
Handles built from a device CSR must give the same y bits as handles built
from the host converters' arrays.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden_cases, load_golden
from matrix_format_performance_b200 import _capi, convert, formats as F
from matrix_format_performance_b200 import synth
from matrix_format_performance_b200._capi import MfpError, call
from matrix_format_performance_b200.device import (COO, CSR_ADAPTIVE, CSR_SCALAR, CSR_VECTOR, ELL, HYBRID, SCOO,
                                                   DeviceMatrix)

pytestmark = pytest.mark.gpu


def dev(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a).cuda()


def host(t, dtype=None):
    a = t.cpu().numpy()
    if a.dtype == np.int32:
        a = a.view(np.uint32)
    return a


def bits(a):
    a = np.asarray(a)
    return a.view(np.uint64 if a.dtype.itemsize == 8 else np.uint32)


def sparse_rows_matrix(dt):
    """100,003 rows, most empty; one 9,000-element row; runs of empty rows
    inside every 2048-element output tile."""
    rng = np.random.default_rng(5)
    rows, cols = 100_003, 60_000
    lens = np.zeros(rows, np.int64)
    lens[::997] = rng.integers(1, 40, size=lens[::997].size)
    lens[50_001] = 9_000
    lens[rows - 1] = 3
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    ci = np.concatenate([np.sort(rng.choice(cols, size=n, replace=False)) for n in lens if n]).astype(np.uint32)
    v = rng.uniform(-1, 1, size=ci.size).astype(dt)
    return F.csr_matrix_class.from_arrays(rows, cols, rp, ci, v, dt)


def tiny_matrices(dt):
    out = {
        "empty_matrix": F.csr_matrix_class.from_arrays(7, 5, np.zeros(8, np.uint32), np.zeros(0, np.uint32),
                                                       np.zeros(0, dt), dt),
        "one_row": F.csr_matrix_class.from_arrays(1, 9, [0, 4], [0, 2, 5, 8], np.arange(1, 5, dtype=dt), dt),
        "one_col": F.csr_matrix_class.from_arrays(5, 1, [0, 1, 1, 2, 3, 3], [0, 0, 0], np.ones(3, dt), dt),
    }
    return out


MATS = {}


def mat(name, dt):
    key = (name, np.dtype(dt).name)
    if key not in MATS:
        if name == "sparse_rows":
            m = sparse_rows_matrix(dt)
        elif name in ("empty_matrix", "one_row", "one_col"):
            m = tiny_matrices(dt)[name]
        else:
            m = {"laplacian_512": lambda: synth.laplacian_2d(512),
                 "power_law_300k": lambda: synth.power_law(rows=300_000, seed=11),
                 "stencil_40": lambda: synth.stencil_27(40, seed=2),
                 "banded_200k": lambda: synth.banded(n=200_000, seed=4),
                 "uniform_rect": lambda: synth.uniform(50_000, 0, 40, seed=9, cols=70_001)}[name]().astype(dt)
        MATS[key] = m
    return MATS[key]


NAMES = ["laplacian_512", "power_law_300k", "stencil_40", "banded_200k", "uniform_rect", "sparse_rows",
         "empty_matrix", "one_row", "one_col"]
DTS = [np.float32, np.float64]


def on_device(m):
    return dev(m.row_ptr), dev(m.columns), dev(m.data)


@pytest.mark.parametrize("name", NAMES)
def test_rows_statistics_bit_identical(name):
    m = mat(name, np.float32)
    want = F.get_rows_statistics(m)
    got = convert.rows_statistics(dev(m.row_ptr))
    for f in ("min_elements_in_rows", "max_elements_in_rows", "avg_elements_in_rows"):
        assert getattr(got, f) == getattr(want, f), f
    assert bits(np.float64(got.elements_in_rows_std_deviation)) == bits(np.float64(want.elements_in_rows_std_deviation))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dt", DTS)
def test_coo_and_tails_identical(name, dt):
    m = mat(name, dt)
    rp, ci, v = on_device(m)
    starts = sorted({0, 1, 3, F.row_length_quantile(m, 2 / 3) if m.rows else 0})
    for s in starts:
        want = F.coo_matrix_class(m, s)
        od, oc, orow = convert.coo_from_csr(rp, ci, v, s)
        assert convert.coo_count(rp, s) == want.elements_count
        np.testing.assert_array_equal(host(orow), want.rows_, err_msg=f"rows start={s}")
        np.testing.assert_array_equal(host(oc), want.cols_, err_msg=f"cols start={s}")
        np.testing.assert_array_equal(bits(host(od)), bits(want.data), err_msg=f"data start={s}")


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dt", DTS)
def test_ell_identical(name, dt):
    m = mat(name, dt)
    rp, ci, v = on_device(m)
    widths = [1, 4]
    if m.rows and F.ell_matrix_class.estimate_size(m) <= 40_000_000:
        widths.append(None)
    for w in widths:
        want = F.ell_matrix_class(m, w) if w is not None else F.ell_matrix_class(m)
        ed, ec, width = convert.ell_from_csr(rp, ci, v, w)
        assert width == want.elements_in_rows
        np.testing.assert_array_equal(host(ec), want.columns, err_msg=f"width={w}")
        np.testing.assert_array_equal(bits(host(ed)), bits(want.data), err_msg=f"width={w}")


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dt", DTS)
@pytest.mark.parametrize("smem", [49152, 232448])
def test_scoo_identical(name, dt, smem):
    m = mat(name, dt)
    want = F.scoo_matrix_class(148, smem, m)
    rp, ci, v = on_device(m)
    ov, oc, orow, sp = convert.scoo_from_csr(rp, ci, v, want.params)
    np.testing.assert_array_equal(host(sp), want.slices_ptr)
    np.testing.assert_array_equal(host(orow), want.r_index)
    np.testing.assert_array_equal(host(oc), want.c_index)
    np.testing.assert_array_equal(bits(host(ov)), bits(want.values))
    # x windows per slice
    win_h = np.empty(2 * want.slices_count, np.uint32)
    call("mfp_scoo_x_windows", m.nnz, F.ptr(want.c_index), F.ptr(want.slices_ptr), want.slices_count, F.ptr(win_h))
    win_d = torch.empty(2 * want.slices_count, dtype=torch.int32, device="cuda")
    call("mfp_dev_scoo_x_windows", m.nnz, convert._p(oc), sp.data_ptr(),
         want.slices_count, win_d.data_ptr(), None)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(win_d), win_h)


@pytest.mark.parametrize("name", ["laplacian_512", "power_law_300k", "banded_200k", "uniform_rect", "sparse_rows"])
def test_hybrid_identical(name):
    m = mat(name, np.float32)
    rp, ci, v = on_device(m)
    for pct in (0.0, 0.2):
        w = F.hybrid_width(m, pct)
        assert convert.hybrid_width(rp, pct) == w
        if m.rows * w > 60_000_000:
            continue
        want = F.hybrid_matrix_class(m)
        want.allocate(m, pct)
        (ed, ec), (cd, cc, cr) = convert.hybrid_from_csr(rp, ci, v, w)
        np.testing.assert_array_equal(host(ec), want.ell_matrix.columns)
        np.testing.assert_array_equal(bits(host(ed)), bits(want.ell_matrix.data))
        np.testing.assert_array_equal(host(cr), want.coo_matrix.rows_)
        np.testing.assert_array_equal(host(cc), want.coo_matrix.cols_)
        np.testing.assert_array_equal(bits(host(cd)), bits(want.coo_matrix.data))


def triplets(m, order, seed=0, duplicates=0):
    rng = np.random.default_rng(seed)
    r = np.repeat(np.arange(m.rows, dtype=np.uint32), np.diff(m.row_ptr.astype(np.int64)))
    c = m.columns.copy()
    v = m.data.astype(np.float64) + rng.uniform(-1e-3, 1e-3, size=m.nnz)  # doubles not exact in float32
    if duplicates and m.nnz:
        pick = rng.integers(0, m.nnz, size=duplicates)
        r = np.concatenate([r, r[pick]])
        c = np.concatenate([c, c[pick]])
        v = np.concatenate([v, rng.uniform(-1, 1, size=duplicates)])
    if order == "shuffled":
        p = rng.permutation(r.size)
    elif order == "column_major":
        p = np.lexsort((r, c))
    else:
        p = np.arange(r.size)
    return F.matrix_class(m.rows, m.cols, r[p], c[p], v[p])


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", ["sorted", "shuffled", "column_major"])
@pytest.mark.parametrize("dt", DTS)
def test_csr_from_coo_identical(name, order, dt):
    m = mat(name, np.float32)
    t = triplets(m, order, seed=hash((name, order)) & 0xffff)
    want = F.csr_matrix_class(t, dt)
    rp, co, d = convert.csr_from_coo(t.rows, t.cols, dev(t.row_ids), dev(t.col_ids), dev(t.data),
                                     torch.float32 if dt == np.float32 else torch.float64)
    np.testing.assert_array_equal(host(rp), want.row_ptr)
    np.testing.assert_array_equal(host(co), want.columns)
    np.testing.assert_array_equal(bits(host(d)), bits(want.data))


@pytest.mark.parametrize("name", ["power_law_300k", "sparse_rows", "one_row"])
def test_csr_from_coo_repeated_entries_keep_input_order(name):
    m = mat(name, np.float32)
    t = triplets(m, "shuffled", seed=3, duplicates=max(1, m.nnz // 10))
    want = F.csr_matrix_class(t, np.float64)
    rp, co, d = convert.csr_from_coo(t.rows, t.cols, dev(t.row_ids), dev(t.col_ids), dev(t.data), torch.float64)
    np.testing.assert_array_equal(host(rp), want.row_ptr)
    np.testing.assert_array_equal(host(co), want.columns)
    np.testing.assert_array_equal(bits(host(d)), bits(want.data))


def test_invalid_ids_and_csr_are_reported():
    r = dev(np.array([0, 1, 5], np.uint32))
    c = dev(np.array([0, 1, 1], np.uint32))
    v = dev(np.ones(3))
    with pytest.raises(MfpError, match="row id >= rows 3 at element 2"):
        convert.csr_from_coo(3, 3, r, c, v)
    with pytest.raises(MfpError, match="col id >= cols 1"):
        convert.csr_from_coo(6, 1, r, c, v)
    with pytest.raises(MfpError, match="not a CSR row pointer"):
        convert.check_csr(dev(np.array([0, 2, 1, 3], np.uint32)), dev(np.zeros(3, np.uint32)), 4)
    with pytest.raises(MfpError, match="column id >= cols 4 at element 1"):
        convert.check_csr(dev(np.array([0, 2, 3], np.uint32)), dev(np.array([0, 4, 1], np.uint32)), 4)
    convert.check_csr(dev(np.array([0, 2, 3], np.uint32)), dev(np.array([0, 3, 1], np.uint32)), 4)


@pytest.mark.parametrize("name", ["laplacian_512", "power_law_300k", "stencil_40", "sparse_rows", "empty_matrix"])
@pytest.mark.parametrize("fmt", [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE, ELL, COO, SCOO, HYBRID])
@pytest.mark.parametrize("dt", DTS)
def test_handle_from_device_csr_gives_the_same_bits(name, fmt, dt):
    m = mat(name, dt)
    if fmt == ELL and F.ell_matrix_class.estimate_size(m) > 40_000_000:
        pytest.skip("ELL padding too large for this matrix")
    hw = F.row_length_quantile(m, 2 / 3) if (fmt == HYBRID and m.rows) else 0
    ref = DeviceMatrix.build(m, fmt, hybrid_width=hw if fmt == HYBRID else None)
    rp, ci, v = on_device(m)
    dm = DeviceMatrix.from_device_csr(rp, ci, v, m.cols, fmt, ell_width=hw if fmt == HYBRID else None)
    del rp, ci, v  # the handle owns copies
    x = dev(synth.vector(1, max(m.cols, 1))[:m.cols].astype(dt))
    y1 = torch.full((m.rows,), float("nan"), dtype=x.dtype, device="cuda")
    y2 = y1.clone()
    ref.spmv(x, y1)
    dm.spmv(x, y2)
    torch.cuda.synchronize()
    assert np.array_equal(bits(host(y1)), bits(host(y2)))
    a, b = ref.info(), dm.info()
    assert (a.format_bytes, a.algorithmic_bytes, a.kernel_launches) == (b.format_bytes, b.algorithmic_bytes,
                                                                         b.kernel_launches)
    if fmt not in (ELL, HYBRID):
        assert a.nnz == b.nnz
    ref.close()
    dm.close()


@pytest.mark.parametrize("case", golden_cases())
def test_golden_fixtures_convert_on_device(case):
    g = load_golden(case)
    for s, dt in (("f32", np.float32), ("f64", np.float64)):
        m = F.csr_matrix_class.from_arrays(int(g["rows"][0]), int(g["cols"][0]), g[f"csr_row_ptr_{s}"],
                                           g[f"csr_columns_{s}"], g[f"csr_data_{s}"], dt)
        rp, ci, v = on_device(m)
        if f"coo_rows_{s}" in g:
            od, oc, orow = convert.coo_from_csr(rp, ci, v)
            np.testing.assert_array_equal(host(orow), g[f"coo_rows_{s}"])
            np.testing.assert_array_equal(host(oc), g[f"coo_cols_{s}"])
            np.testing.assert_array_equal(bits(host(od)), bits(g[f"coo_data_{s}"].astype(dt)))
        if f"ell_columns_{s}" in g:
            ed, ec, w = convert.ell_from_csr(rp, ci, v)
            assert w == int(g[f"ell_width_{s}"][0])
            np.testing.assert_array_equal(host(ec), g[f"ell_columns_{s}"])
            np.testing.assert_array_equal(bits(host(ed)), bits(g[f"ell_data_{s}"].astype(dt)))
        st = convert.rows_statistics(rp)
        assert [st.min_elements_in_rows, st.max_elements_in_rows, st.avg_elements_in_rows] == list(g["stats_u32"])
        assert bits(np.float64(st.elements_in_rows_std_deviation)) == bits(np.float64(g["stats_std"][0]))
        for tag in ("scoo", "scoo_small"):
            p = _capi.ScooParams(*[int(t) for t in g[f"{tag}_params_{s}"]])
            ov, oc, orow, sp = convert.scoo_from_csr(rp, ci, v, p)
            np.testing.assert_array_equal(host(sp), g[f"{tag}_slices_ptr_{s}"])
            np.testing.assert_array_equal(host(orow), g[f"{tag}_r_index_{s}"])
            np.testing.assert_array_equal(host(oc), g[f"{tag}_c_index_{s}"])
            np.testing.assert_array_equal(bits(host(ov)), bits(g[f"{tag}_values_{s}"].astype(dt)))
        w = int(g[f"hyb_width_{s}"][0])
        assert convert.hybrid_width(rp, 0.2) == w
        (ed, ec), (cd, cc, cr) = convert.hybrid_from_csr(rp, ci, v, w)
        if f"hyb_ell_columns_{s}" in g:  # fixtures keep the ELL part only where it is small
            np.testing.assert_array_equal(host(ec), g[f"hyb_ell_columns_{s}"])
            np.testing.assert_array_equal(bits(host(ed)), bits(g[f"hyb_ell_data_{s}"].astype(dt)))
        np.testing.assert_array_equal(host(cr), g[f"hyb_coo_rows_{s}"])
        np.testing.assert_array_equal(host(cc), g[f"hyb_coo_cols_{s}"])
        np.testing.assert_array_equal(bits(host(cd)), bits(g[f"hyb_coo_data_{s}"].astype(dt)))
        t = F.matrix_class(int(g["rows"][0]), int(g["cols"][0]), g["row_ids"], g["col_ids"], g["values"])
        rp2, co2, d2 = convert.csr_from_coo(t.rows, t.cols, dev(t.row_ids), dev(t.col_ids), dev(t.data),
                                            torch.float32 if s == "f32" else torch.float64)
        np.testing.assert_array_equal(host(rp2), g[f"csr_row_ptr_{s}"])
        np.testing.assert_array_equal(host(co2), g[f"csr_columns_{s}"])
        np.testing.assert_array_equal(bits(host(d2)), bits(g[f"csr_data_{s}"].astype(dt)))


def test_full_size_power_law_conversions():
    """4,194,304-row power-law matrix: COO and SCOO from CSR, and CSR back
    from shuffled triplets, on the device against the host converters."""
    m = synth.power_law(rows=4_194_304, seed=0)
    rp, ci, v = on_device(m)
    want = F.scoo_matrix_class(148, 49152, m)
    ov, oc, orow, sp = convert.scoo_from_csr(rp, ci, v, want.params)
    np.testing.assert_array_equal(host(sp), want.slices_ptr)
    np.testing.assert_array_equal(host(orow), want.r_index)
    np.testing.assert_array_equal(host(oc), want.c_index)
    np.testing.assert_array_equal(bits(host(ov)), bits(want.values))
    del ov, oc, sp
    t = triplets(m, "shuffled", seed=1)
    want = F.csr_matrix_class(t, np.float32)
    rp2, co2, d2 = convert.csr_from_coo(t.rows, t.cols, dev(t.row_ids), dev(t.col_ids), dev(t.data))
    np.testing.assert_array_equal(host(rp2), want.row_ptr)
    np.testing.assert_array_equal(host(co2), want.columns)
    np.testing.assert_array_equal(bits(host(d2)), bits(want.data))


def test_scratch_pool_is_kept_and_released():
    m = mat("power_law_300k", np.float32)
    t = triplets(m, "shuffled", seed=7)
    convert.csr_from_coo(t.rows, t.cols, dev(t.row_ids), dev(t.col_ids), dev(t.data))
    assert convert.scratch_bytes() >= m.nnz * 16  # keys and payloads of both sort buffers stay mapped
    convert.release_scratch()
    assert convert.scratch_bytes() == 0


@pytest.mark.parametrize("name", ["laplacian_512", "power_law_300k", "stencil_40", "sparse_rows", "one_row",
                                  "empty_matrix"])
@pytest.mark.parametrize("dt", DTS)
def test_scoo_sort_cols_on_device_identical(name, dt):
    m = mat(name, dt)
    want = F.scoo_matrix_class(148, 49152, m, sort_cols=True)
    plain = F.scoo_matrix_class(148, 49152, m)
    v, c, r = dev(plain.values), dev(plain.c_index), dev(plain.r_index)
    convert.scoo_sort_cols(v, c, r, m.rows, m.cols, plain.slice_size)
    np.testing.assert_array_equal(host(c), want.c_index)
    np.testing.assert_array_equal(host(r), want.r_index)
    np.testing.assert_array_equal(bits(host(v)), bits(want.values))
