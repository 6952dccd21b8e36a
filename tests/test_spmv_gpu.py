"""Parity of every sm_100a format kernel with the oracle (needs a B200).

Criteria
  exact      CSR scalar (one thread per row, CSR order) and ELL (slots in
             order) equal the reference CPU loop bit for bit; CSR vector with
             32 lanes equals the reference's reduce-order loop for rows whose
             elements are staged in one chunk.
  tolerance  every format, per row: |y - y*| <= TOL * sum_j |a_ij x_j|, with
             y* the extended-precision product of the same (rounded) inputs;
             TOL = 1e-5 for float32 and 1e-12 for float64.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden_cases, load_golden
from matrix_format_performance_b200 import formats as F
from matrix_format_performance_b200 import synth
from matrix_format_performance_b200._capi import call
from matrix_format_performance_b200.device import (COO, CSR_ADAPTIVE, CSR_SCALAR, CSR_VECTOR, ELL, HYBRID, SCOO,
                                                   DeviceMatrix)

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.float32): 1e-5, np.dtype(np.float64): 1e-12}
ALL = [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE, ELL, COO, SCOO, HYBRID]
NEVER = 0xFFFFFFFF
EXACT_SCALAR = {"long_row_threshold": NEVER, "assist_threshold": NEVER}
EXACT_VECTOR = {"long_row_threshold": NEVER, "assist_threshold": NEVER, "vector_lanes": 32}


def run(m, fmt, x, config=None, hybrid_width=None, reps=1):
    dm = DeviceMatrix.build(m, fmt, config=config, hybrid_width=hybrid_width)
    xt = torch.from_numpy(np.ascontiguousarray(x, m.dtype)).cuda()
    outs = []
    for _ in range(reps):
        yt = torch.full((m.rows,), float("nan"), dtype=xt.dtype, device="cuda")
        dm.spmv(xt, yt)
        torch.cuda.synchronize()
        outs.append(yt.cpu().numpy())
    dm.close()
    return outs if reps > 1 else outs[0]


def check_tol(oracle_lib, m, x, y, what=""):
    ys, ab = oracle_lib.csr_spmv_exact(m.rows, m.row_ptr, m.columns, m.data, x.astype(m.dtype))
    err = np.abs(y.astype(np.float64) - ys)
    bound = TOL[m.dtype] * ab
    bad = np.nonzero(~(err <= bound))[0]
    assert bad.size == 0, (f"{what}: {bad.size} rows out of tolerance, first {bad[:5]}, "
                           f"err {err[bad[:5]]}, bound {bound[bad[:5]]}")


def golden_csr(g, s):
    dt = np.float32 if s == "f32" else np.float64
    return F.csr_matrix_class.from_arrays(int(g["rows"][0]), int(g["cols"][0]), g[f"csr_row_ptr_{s}"],
                                          g[f"csr_columns_{s}"], g[f"csr_data_{s}"], dt)


def single_chunk_windows(m, block=256, chunk=2048):
    rp = m.row_ptr.astype(np.int64)
    for r0 in range(0, m.rows, block):
        r1 = min(m.rows, r0 + block)
        if rp[r1] - (rp[r0] & ~3) > chunk:
            return False
    return True


@pytest.mark.parametrize("case", golden_cases())
@pytest.mark.parametrize("s", ["f32", "f64"])
def test_exact_formats_match_reference_bits(case, s):
    g = load_golden(case)
    m = golden_csr(g, s)
    x = g["x"].astype(m.dtype)
    assert np.array_equal(run(m, CSR_SCALAR, x, EXACT_SCALAR), g[f"yx_{s}"])
    assert np.array_equal(run(m, ELL, x), g[f"yx_{s}"])
    yv = run(m, CSR_VECTOR, x, EXACT_VECTOR)
    if single_chunk_windows(m):
        assert np.array_equal(yv, g[f"yxro_{s}"])
    ones = np.ones(m.cols, m.dtype)
    assert np.array_equal(run(m, CSR_SCALAR, ones, EXACT_SCALAR), g[f"y1_{s}"])


@pytest.mark.parametrize("case", golden_cases())
@pytest.mark.parametrize("s", ["f32", "f64"])
@pytest.mark.parametrize("fmt", ALL)
def test_all_formats_within_tolerance_on_fixtures(oracle_lib, case, s, fmt):
    g = load_golden(case)
    m = golden_csr(g, s)
    x = g["x"].astype(m.dtype)
    check_tol(oracle_lib, m, x, run(m, fmt, x), f"{case}/{s}/fmt{fmt}")


def _synthetic():
    return {
        "laplacian_512": synth.laplacian_2d(512),
        "power_law_300k": synth.power_law(rows=300_000, seed=11),
        "stencil_40": synth.stencil_27(40, seed=2),
        "banded_200k": synth.banded(n=200_000, seed=4),
        "uniform_rect": synth.uniform(50_000, 0, 40, seed=9, cols=70_001),
    }


SYN = {}


def syn(name):
    if name not in SYN:
        SYN[name] = _synthetic()[name]
    return SYN[name]


@pytest.mark.parametrize("name", ["laplacian_512", "power_law_300k", "stencil_40", "banded_200k", "uniform_rect"])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("fmt", ALL)
def test_synthetic_configs_within_tolerance(oracle_lib, name, dt, fmt):
    m = syn(name).astype(dt)
    if fmt == ELL and F.ell_matrix_class.estimate_size(m) > 50_000_000:
        pytest.skip("ELL padding too large for this matrix (the reference skips it too)")
    x = synth.vector(0, m.cols).astype(dt)
    hw = F.row_length_quantile(m, 2 / 3) if fmt == HYBRID else None
    check_tol(oracle_lib, m, x, run(m, fmt, x, hybrid_width=hw), f"{name}/{dt.__name__}/fmt{fmt}")


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_scalar_and_ell_exact_on_laplacian_512(oracle_lib, dt):
    m = syn("laplacian_512").astype(dt)
    x = synth.vector(0, m.cols).astype(dt)
    y_ref = oracle_lib.csr_spmv(m.rows, m.row_ptr, m.columns, m.data, x)
    assert np.array_equal(run(m, CSR_SCALAR, x, EXACT_SCALAR), y_ref)
    assert np.array_equal(run(m, ELL, x), y_ref)
    # default (streaming) configuration: exact except rows split between two CTA ranges
    y = run(m, CSR_SCALAR, x)
    assert np.count_nonzero(y != y_ref) <= 2 * 148 * 8


def _long_rows_matrix(dt):
    rng = np.random.default_rng(77)
    lens = rng.integers(0, 9, size=6000)
    lens[[5, 1234, 5999]] = [50_000, 9_000, 4_097]
    lens[[10, 11, 12]] = [3000, 0, 700]
    cols = 200_000
    rp = np.zeros(lens.size + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(cols, size=int(n), replace=False)) for n in lens]).astype(np.uint32)
    v = rng.uniform(-1, 1, size=ci.size)
    return F.csr_matrix_class.from_arrays(lens.size, cols, rp.astype(np.uint32), ci, v.astype(dt), dt)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("fmt", ALL)
def test_long_rows_split_and_repeatable(oracle_lib, dt, fmt):
    m = _long_rows_matrix(dt)
    if fmt == ELL:
        pytest.skip("ELL width 50,000")
    x = synth.vector(3, m.cols).astype(dt)
    ys = run(m, fmt, x, reps=3, hybrid_width=4)
    check_tol(oracle_lib, m, x, ys[0], f"long rows fmt{fmt}")
    # deterministic: plan counters reset between launches, sums in a fixed order
    assert np.array_equal(ys[0], ys[1]) and np.array_equal(ys[1], ys[2])


@pytest.mark.parametrize("name", ["laplacian_512", "power_law_300k", "stencil_40", "banded_200k", "uniform_rect"])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("fmt", [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE])
def test_warp_tile_csr_kernel(oracle_lib, name, dt, fmt):
    """kernel 4: 256 consecutive elements per warp, rows from row_ptr, the COO
    reduction and fix-up; repeatable bit for bit."""
    m = syn(name).astype(dt)
    x = synth.vector(5, m.cols).astype(dt)
    ys = run(m, fmt, x, {"kernel": 4}, reps=2)
    check_tol(oracle_lib, m, x, ys[0], f"{name}/{dt.__name__}/tile fmt{fmt}")
    assert np.array_equal(ys[0], ys[1])


@pytest.mark.parametrize("lanes", [2, 4, 8, 16, 32])
def test_vector_lane_counts(oracle_lib, lanes):
    m = syn("power_law_300k").astype(np.float32)
    x = synth.vector(1, m.cols).astype(np.float32)
    check_tol(oracle_lib, m, x, run(m, CSR_VECTOR, x, {"vector_lanes": lanes}), f"lanes {lanes}")


@pytest.mark.parametrize("cfg", [{"long_row_threshold": 300, "piece_nnz": 256}, {"assist_threshold": 8},
                                 {"bin_nnz": 64}, {"bin_nnz": 700, "long_row_threshold": 5000}, {"kernel": 4}])
@pytest.mark.parametrize("fmt", [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE])
def test_csr_plan_configurations(oracle_lib, cfg, fmt):
    m = _long_rows_matrix(np.float64)
    x = synth.vector(5, m.cols)
    check_tol(oracle_lib, m, x, run(m, fmt, x, cfg), f"cfg {cfg} fmt{fmt}")


@pytest.mark.parametrize("fmt", ALL)
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_empty_rows_and_empty_matrix(fmt, dt):
    rp = np.array([0, 0, 3, 3, 3, 4, 4], np.uint32)
    ci = np.array([0, 2, 5, 1], np.uint32)
    m = F.csr_matrix_class.from_arrays(6, 7, rp, ci, np.array([1, 2, 3, 4], dt), dt)
    x = np.arange(1, 8).astype(dt)
    y = run(m, fmt, x, hybrid_width=1)
    assert np.array_equal(y, np.array([0, 1 + 6 + 18, 0, 0, 8, 0], dt))
    z = F.csr_matrix_class.from_arrays(5, 3, np.zeros(6, np.uint32), np.zeros(0, np.uint32), np.zeros(0, dt), dt)
    assert np.array_equal(run(z, fmt, np.ones(3, dt), hybrid_width=0), np.zeros(5, dt))


def test_coo_tiles_sharing_rows(oracle_lib):
    # one row spans many 2048-element tiles, separated by long runs of empty rows
    rng = np.random.default_rng(5)
    lens = np.zeros(100_000, np.int64)
    lens[0] = 3
    lens[17] = 20_000
    lens[18] = 1
    lens[60_000] = 9_000
    lens[99_999] = 2
    cols = 30_000
    rp = np.zeros(lens.size + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(cols, size=int(n), replace=False)) for n in lens if n]).astype(np.uint32)
    m = F.csr_matrix_class.from_arrays(lens.size, cols, rp.astype(np.uint32), ci, rng.uniform(-1, 1, ci.size), np.float64)
    x = synth.vector(2, cols)
    ys = run(m, COO, x, reps=3)
    check_tol(oracle_lib, m, x, ys[0], "coo tiles")
    assert np.array_equal(ys[0], ys[2])


@pytest.mark.parametrize("nnz_valid", [100, 5_000, 70_000])
def test_coo_drops_row_ids_beyond_rows(oracle_lib, nnz_valid):
    """Row ids >= rows are dropped: y past `rows` (here a guard region of the
    same allocation, which the ids point into) is never written."""
    rng = np.random.default_rng(nnz_valid)
    rows, cols, guard = 3_000, 500, 64
    r = np.sort(rng.integers(0, rows, size=nnz_valid)).astype(np.uint32)
    r = np.concatenate([r, np.array([rows, rows + 3, rows + 3, rows + 40], np.uint32)])
    c = rng.integers(0, cols, size=r.size).astype(np.uint32)
    v = rng.uniform(-1, 1, size=r.size).astype(np.float32)
    x = rng.uniform(-1, 1, size=cols).astype(np.float32)
    rp = np.zeros(rows + 1, np.int64)
    np.add.at(rp, r[:nnz_valid].astype(np.int64) + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    ys, ab = oracle_lib.csr_spmv_exact(rows, rp, c[:nnz_valid], v[:nnz_valid], x)
    d_v, d_c, d_r, d_x = (torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda()
                          for a in (v, c, r, x))
    y = torch.full((rows + guard,), 7.0, device="cuda")
    nbytes = C.c_size_t()
    call("mfp_coo_workspace_bytes", rows, r.size, C.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    call("mfp_coo_spmv_f32", rows, cols, r.size, *(C.c_void_p(t.data_ptr()) for t in (d_v, d_c, d_r, d_x, y, ws)),
         nbytes.value, stream)
    torch.cuda.synchronize()
    got = y.cpu().numpy()
    assert np.all(got[rows:] == 7.0)
    assert np.all(np.abs(got[:rows].astype(np.float64) - ys) <= 1e-5 * ab)


@pytest.mark.parametrize("name", ["power_law_300k", "stencil_40"])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_raw_hybrid_entry_point_matches_handle(oracle_lib, name, dt):
    """mfp_hybrid_spmv_* on the reference layout (the ELL kernel, then the COO
    passes adding the tail) against the oracle, and the handle on the same
    layout."""
    m = syn(name).astype(dt)
    x = synth.vector(12, m.cols).astype(dt)
    w = F.row_length_quantile(m, 2 / 3)
    hm = F.hybrid_matrix_class(m)
    hm.allocate_width(m, w)
    e, c = hm.ell_matrix, hm.coo_matrix
    dv = lambda a: torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda()  # noqa: E731
    d_ed, d_ec, d_cd, d_cc, d_cr, d_x = (dv(a) for a in (e.data, e.columns, c.data, c.cols_, c.rows_, x))
    nb = C.c_size_t()
    call("mfp_hybrid_workspace_bytes", m.rows, c.elements_count, C.byref(nb))
    ws = torch.empty(max(1, nb.value), dtype=torch.uint8, device="cuda")
    y = torch.full((m.rows,), float("nan"), dtype=d_x.dtype, device="cuda")
    fn = "mfp_hybrid_spmv_f32" if dt == np.float32 else "mfp_hybrid_spmv_f64"
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    call(fn, m.rows, m.cols, w, p(d_ed), p(d_ec), c.elements_count, p(d_cd), p(d_cc), p(d_cr), p(d_x), p(y), p(ws),
         nb.value, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    y_raw = y.cpu().numpy()
    check_tol(oracle_lib, m, x, y_raw, f"raw hybrid {name}")
    y_handle = run(m, HYBRID, x, hybrid_width=w)
    check_tol(oracle_lib, m, x, y_handle, f"hybrid handle {name}")


def test_device_pointer_entry_points_and_unaligned_arrays(oracle_lib):
    m = syn("power_law_300k").astype(np.float32)
    x = synth.vector(4, m.cols).astype(np.float32)
    # offset every array by one element so the 16-byte paths are not taken
    def dev(a):
        t = torch.empty(a.size + 1, dtype=torch.from_numpy(a[:1]).dtype, device="cuda")
        t[1:] = torch.from_numpy(a).cuda()
        return t, t.data_ptr() + a.itemsize
    keep = []  # the tensors must outlive the raw pointers handed to the library

    def dev_keep(a):
        t, p = dev(a)
        keep.append(t)
        return p
    d_v = dev_keep(m.data)
    d_c = dev_keep(m.columns.view(np.int32))
    d_r = dev_keep(m.row_ptr.view(np.int32))
    xt = torch.from_numpy(x).cuda()
    yt = torch.full((m.rows,), float("nan"), device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for algo in (0, 1, 2):
        plan = C.c_void_p()
        call("mfp_csr_plan_create", m.rows, m.cols, m.nnz, F.ptr(m.row_ptr), algo, None, C.byref(plan))
        call("mfp_csr_spmv_f32", plan, C.c_void_p(d_v), C.c_void_p(d_c), C.c_void_p(d_r), C.c_void_p(xt.data_ptr()),
             C.c_void_p(yt.data_ptr()), stream)
        torch.cuda.synchronize()
        check_tol(oracle_lib, m, x, yt.cpu().numpy(), f"unaligned csr algo {algo}")
        call("mfp_csr_plan_destroy", plan)
    coo = F.coo_matrix_class(m)
    d_cv = dev_keep(coo.data)
    d_cc = dev_keep(coo.cols_.view(np.int32))
    d_cr = dev_keep(coo.rows_.view(np.int32))
    nbytes = C.c_size_t()
    call("mfp_coo_workspace_bytes", m.rows, m.nnz, C.byref(nbytes))
    ws = torch.zeros(nbytes.value, dtype=torch.uint8, device="cuda")
    yt.fill_(float("nan"))
    call("mfp_coo_spmv_f32", m.rows, m.cols, m.nnz, C.c_void_p(d_cv), C.c_void_p(d_cc), C.c_void_p(d_cr),
         C.c_void_p(xt.data_ptr()), C.c_void_p(yt.data_ptr()), C.c_void_p(ws.data_ptr()), nbytes.value, stream)
    torch.cuda.synchronize()
    check_tol(oracle_lib, m, x, yt.cpu().numpy(), "unaligned coo")
    err = C.c_uint32()
    call("mfp_workspace_error", C.c_void_p(ws.data_ptr()), C.byref(err))
    assert err.value == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_scoo_tiles_and_chunk_fallback(oracle_lib, dtype):
    """SCOO slices reduced in warp tiles (rows crossing tiles summed in tile
    order), and a slice of more than 512 tiles (a 140,000-element row plus
    neighbours) that takes the whole-CTA chunk path; empty rows on both
    sides; the same bits on a second run."""
    rng = np.random.default_rng(31)
    rows, cols = 3000, 200_000
    lens = rng.integers(0, 4, rows)
    lens[1500] = 140_000          # > 512 tiles of 256 in its slice
    lens[700] = 130_000 // 2      # ~254 tiles: the tile path with a long carry chain
    lens[701:705] = 0
    lens[2990:] = 0
    rp = np.zeros(rows + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    colv = np.concatenate([np.sort(rng.choice(cols, n, replace=False)) if n else np.zeros(0, np.int64)
                           for n in lens]).astype(np.uint32)
    vals = rng.uniform(-1, 1, int(rp[-1]))
    m = F.csr_matrix_class.from_arrays(rows, cols, rp.astype(np.uint32), colv, vals, dtype)
    x = synth.vector(5, cols).astype(dtype)
    a, b = run(m, SCOO, x, reps=2)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    check_tol(oracle_lib, m, x, a, "scoo tiles / chunks")


def compact_row_bytes(rows, dtype):
    """(bytes per row id, wide tiles) of a COO handle: 1 when at most one
    256-element tile in 8 spans more than 256 rows (those wide tiles read
    4-byte rows; float32 only, float64 needs none), else 2 when every tile
    spans at most 65,536 rows, else 4."""
    rows = np.asarray(rows, np.int64)
    if rows.size == 0:
        return 4, 0
    span = np.maximum.reduceat(rows - np.repeat(rows[::256], 256)[:rows.size], np.arange(0, rows.size, 256))
    wide = int((span > 0xFF).sum())
    if wide <= span.size // 8 and (wide == 0 or np.dtype(dtype) == np.float32):
        return 1, wide
    return (2 if span.max() <= 0xFFFF else 4), 0


def gapped_rows_matrix(dtype, gap, holes=()):
    """Rows of 4-8 elements separated by `gap` - 1 empty rows (a 256-element
    tile spans about 43 * gap rows), and no elements in the row ranges
    `holes` (start, length)."""
    rng = np.random.default_rng(11)
    rows, cols = 200_000, 5000
    lens = np.zeros(rows, np.int64)
    lens[::gap] = rng.integers(4, 9, lens[::gap].size)
    for a, n in holes:
        lens[a:a + n] = 0
    rp = np.zeros(rows + 1, np.uint32)
    rp[1:] = np.cumsum(lens)
    colv = np.concatenate([np.sort(rng.choice(cols, n, replace=False)) for n in lens if n]).astype(np.uint32)
    return F.csr_matrix_class.from_arrays(rows, cols, rp, colv, rng.uniform(-1, 1, colv.size), dtype)


COMPACT_CASES = {"gap_3": (3, ()), "gap_200": (200, ()),
                 "holes": (1, ((5_000, 300), (50_000, 1_000), (120_000, 70_000), (199_000, 500)))}


@pytest.mark.parametrize("case", ["power_law_300k", "gap_3", "gap_200", "holes"])
@pytest.mark.parametrize("fmt", [COO, SCOO, HYBRID])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_compact_rows_give_the_bits_of_32_bit_rows(oracle_lib, case, fmt, dtype):
    """COO, SCOO and hybrid handles keep their rows as offsets.  COO and the
    hybrid's tail: 8-bit offsets from each 256-element tile's first row when
    at most one tile in 8 spans more than 256 rows, those wide tiles reading
    the 32-bit rows (the power-law matrix; rows with 2 empty rows between
    them; in float32, empty row ranges of 300 to 70,000 rows, which also
    make one tile span more than 65,536 rows: 32-bit rows in float64), else
    16-bit (199 empty rows between rows).
    SCOO: 16-bit offsets from the slice's first row.  The same bits as the
    raw entry points on the 32-bit row ids, and the handle's byte count
    charges the row bytes read."""
    m = syn(case).astype(dtype) if case == "power_law_300k" else gapped_rows_matrix(dtype, *COMPACT_CASES[case])
    x = synth.vector(13, m.cols).astype(dtype)
    xt = torch.from_numpy(x).cuda()
    sfx = "f32" if dtype == np.float32 else "f64"
    keep = []

    def dev(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        keep.append(t)
        return C.c_void_p(t.data_ptr())
    yr = torch.full((m.rows,), float("nan"), dtype=xt.dtype, device="cuda")
    vs = np.dtype(dtype).itemsize
    if fmt == COO:
        c = F.coo_matrix_class(m)
        nbytes = C.c_size_t()
        call("mfp_coo_workspace_bytes", m.rows, m.nnz, C.byref(nbytes))
        ws = torch.zeros(nbytes.value, dtype=torch.uint8, device="cuda")
        call(f"mfp_coo_spmv_{sfx}", m.rows, m.cols, m.nnz, dev(c.data), dev(c.cols_.view(np.int32)),
             dev(c.rows_.view(np.int32)), C.c_void_p(xt.data_ptr()), C.c_void_p(yr.data_ptr()),
             C.c_void_p(ws.data_ptr()), nbytes.value, None)
        dm = DeviceMatrix.from_coo(c)
        n_ids, tiles = m.nnz, -(-m.nnz // 256)
    elif fmt == SCOO:
        c = F.scoo_matrix_class(148, 49152, m)
        call(f"mfp_scoo_spmv_{sfx}", m.rows, m.cols, c.slices_count, c.slice_size, dev(c.values),
             dev(c.c_index.view(np.int32)), dev(c.r_index.view(np.int32)), dev(c.slices_ptr.view(np.int32)), None, 0,
             None, C.c_void_p(xt.data_ptr()), C.c_void_p(yr.data_ptr()), None)
        dm = DeviceMatrix.from_scoo(c)
        n_ids, tiles = m.nnz, 0
    else:
        hm = F.hybrid_matrix_class(m)
        hm.allocate_width(m, 2)
        e, c = hm.ell_matrix, hm.coo_matrix
        nbytes = C.c_size_t()
        call("mfp_hybrid_workspace_bytes", m.rows, c.elements_count, C.byref(nbytes))
        ws = torch.zeros(max(1, nbytes.value), dtype=torch.uint8, device="cuda")
        call(f"mfp_hybrid_spmv_{sfx}", m.rows, m.cols, e.elements_in_rows, dev(e.data),
             dev(e.columns.view(np.int32)), c.elements_count, dev(c.data), dev(c.cols_.view(np.int32)),
             dev(c.rows_.view(np.int32)), C.c_void_p(xt.data_ptr()), C.c_void_p(yr.data_ptr()),
             C.c_void_p(ws.data_ptr()), nbytes.value, None)
        dm = DeviceMatrix.from_hybrid(hm)
        n_ids, tiles = c.elements_count, -(-c.elements_count // 256)
    torch.cuda.synchronize()
    yh = torch.full((m.rows,), float("nan"), dtype=xt.dtype, device="cuda")
    dm.spmv(xt, yh)
    torch.cuda.synchronize()
    info = dm.info()
    dm.close()
    assert np.array_equal(yr.cpu().numpy().view(np.uint8), yh.cpu().numpy().view(np.uint8))
    check_tol(oracle_lib, m, x, yh.cpu().numpy(), "compact rows")
    if fmt == COO:
        rb, wide = compact_row_bytes(c.rows_, dtype)
        holes64 = case == "holes" and dtype == np.float64  # a tile spans 70,043 rows: 32-bit rows
        assert rb == (2 if case == "gap_200" else 4 if holes64 else 1)
        assert (wide > 0) == (case == "holes" and dtype == np.float32)
        assert info.format_bytes == (m.nnz * (vs + 4 + rb) + (4 * tiles if rb < 4 else 0) + wide * 256 * 3
                                     + m.cols * vs + m.rows * vs)
    elif fmt == SCOO:
        assert info.format_bytes == m.nnz * (vs + 6) + (c.slices_count + 1) * 4 + m.cols * vs + m.rows * vs


def test_compact_rows_fall_back_when_a_tile_spans_more_than_16_bits(oracle_lib):
    """A COO tile whose rows span more than 65,535 (long runs of empty rows)
    keeps 32-bit rows; the handle's y is right either way."""
    rows, cols = 300_000, 1000
    rng = np.random.default_rng(5)
    r = np.sort(np.concatenate([rng.integers(0, 10, 200), [70_000, 150_000, 299_999], rng.integers(0, rows, 400)]))
    lens = np.bincount(r, minlength=rows)
    rp = np.zeros(rows + 1, np.uint32)
    rp[1:] = np.cumsum(lens)
    colv = np.concatenate([np.sort(rng.choice(cols, n, replace=False)) for n in lens if n]).astype(np.uint32)
    m = F.csr_matrix_class.from_arrays(rows, cols, rp, colv, rng.uniform(-1, 1, len(colv)), np.float32)
    x = synth.vector(3, cols).astype(np.float32)
    dm = DeviceMatrix.build(m, COO)
    info = dm.info()
    xt = torch.from_numpy(x).cuda()
    y = torch.full((rows,), float("nan"), device="cuda")
    dm.spmv(xt, y)
    torch.cuda.synchronize()
    dm.close()
    assert info.format_bytes == m.nnz * 12 + cols * 4 + rows * 4  # 32-bit rows kept
    check_tol(oracle_lib, m, x, y.cpu().numpy(), "coo fallback rows")


def test_raw_scoo_row_ids_outside_their_slice_stay_in_bounds(oracle_lib):
    """mfp_scoo_spmv_f32 on caller arrays where one element's row id points
    into the previous slice (inside a long row the warp tiles carry across
    tiles) and another's beyond the matrix: the slice's shared-memory
    accumulator is never indexed out of range, every other row keeps the
    bits of the unchanged arrays, and the two rows get finite values (which
    the invalid input leaves unspecified)."""
    m = syn("power_law_300k").astype(np.float32)
    sc = F.scoo_matrix_class(148, 49152, m)
    sp = sc.slices_ptr.astype(np.int64)
    s = int(np.argmax(np.diff(sp)[1:])) + 1            # a slice > 0 with many elements
    e1, e2 = int(sp[s]) + 300, int(sp[s + 1]) - 1
    bad = sc.r_index.copy()
    rows_hit = [int(bad[e1]), int(bad[e2])]
    assert rows_hit[0] != rows_hit[1]
    bad[e1] = s * sc.slice_size - 1                       # a row of the previous slice
    bad[e2] = m.rows + 5                                  # beyond the matrix
    x = synth.vector(12, m.cols).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    v, ci, sp_d = d(sc.values), d(sc.c_index.view(np.int32)), d(sc.slices_ptr.view(np.int32))
    outs = []
    for ri in (sc.r_index, bad):
        rt = d(ri.view(np.int32))
        yt = torch.full((m.rows,), float("nan"), device="cuda")
        call("mfp_scoo_spmv_f32", m.rows, m.cols, sc.slices_count, sc.slice_size, C.c_void_p(v.data_ptr()),
             C.c_void_p(ci.data_ptr()), C.c_void_p(rt.data_ptr()), C.c_void_p(sp_d.data_ptr()), None, 0, None,
             C.c_void_p(xt.data_ptr()), C.c_void_p(yt.data_ptr()), None)
        torch.cuda.synchronize()
        outs.append(yt.cpu().numpy())
    good, y = outs
    check_tol(oracle_lib, m, x, good, "raw scoo")
    others = np.ones(m.rows, bool)
    others[rows_hit] = False
    assert np.array_equal(good[others].view(np.uint32), y[others].view(np.uint32))
    assert np.all(np.isfinite(y[rows_hit]))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("fmt", ["coo", "csr0", "csr1", "csr2", "ell"])
def test_load_widths_agree(oracle_lib, fmt, dtype):
    """Kernels read a thread's 32-byte sector with one 256-bit load on
    32-byte-aligned arrays, with 16-byte loads on 16-byte-aligned arrays and
    element by element otherwise; the three give the same bits (COO warp
    pass, CSR vector (warp tiles), ELL; FP32 and FP64).  CSR scalar and
    CSR-Adaptive, whose rows of a few thousand elements are reduced by a
    whole CTA, give the same bits for both vector widths."""
    m = syn("stencil_40" if fmt == "ell" else "power_law_300k").astype(dtype)
    x = synth.vector(9, m.cols).astype(dtype)
    xt = torch.from_numpy(x).cuda()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    sfx = "f32" if dtype == np.float32 else "f64"
    outs = []
    for off in (0, 16, np.dtype(dtype).itemsize):  # bytes past a 256-byte-aligned allocation
        keep = []

        def dev(a):
            raw = torch.zeros(a.nbytes + off, dtype=torch.uint8, device="cuda")
            raw[off:].copy_(torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).ravel()))
            keep.append(raw)
            return C.c_void_p(raw.data_ptr() + off)
        yraw = torch.zeros(m.rows * x.itemsize + off, dtype=torch.uint8, device="cuda")
        yp = C.c_void_p(yraw.data_ptr() + off)
        if fmt == "coo":
            coo = F.coo_matrix_class(m)
            nbytes = C.c_size_t()
            call("mfp_coo_workspace_bytes", m.rows, m.nnz, C.byref(nbytes))
            ws = torch.zeros(nbytes.value, dtype=torch.uint8, device="cuda")
            call(f"mfp_coo_spmv_{sfx}", m.rows, m.cols, m.nnz, dev(coo.data), dev(coo.cols_.view(np.int32)),
                 dev(coo.rows_.view(np.int32)), C.c_void_p(xt.data_ptr()), yp, C.c_void_p(ws.data_ptr()),
                 nbytes.value, stream)
        elif fmt == "ell":
            e = F.ell_matrix_class(m)
            call(f"mfp_ell_spmv_{sfx}", m.rows, m.cols, e.elements_in_rows, dev(e.data), dev(e.columns.view(np.int32)),
                 C.c_void_p(xt.data_ptr()), yp, stream)
        else:
            plan = C.c_void_p()
            call("mfp_csr_plan_create", m.rows, m.cols, m.nnz, F.ptr(m.row_ptr), int(fmt[3]), None, C.byref(plan))
            call(f"mfp_csr_spmv_{sfx}", plan, dev(m.data), dev(m.columns.view(np.int32)),
                 dev(m.row_ptr.view(np.int32)), C.c_void_p(xt.data_ptr()), yp, stream)
            torch.cuda.synchronize()
            call("mfp_csr_plan_destroy", plan)
        torch.cuda.synchronize()
        outs.append(yraw[off:].cpu().numpy().view(dtype).copy())
    assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8))
    if fmt in ("csr0", "csr2"):  # a whole-CTA row shares its elements among threads differently element by element
        check_tol(oracle_lib, m, x, outs[2], f"{fmt} {sfx} unaligned")
    else:
        assert np.array_equal(outs[0].view(np.uint8), outs[2].view(np.uint8))
    check_tol(oracle_lib, m, x, outs[0], f"{fmt} {sfx} load widths")


@pytest.mark.parametrize("fmt", [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE, ELL, COO, SCOO, HYBRID])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_pipelined_host_batch_equals_device_calls(fmt, dtype):
    """mfp_matrix_spmv_host_batch: 1, 2 and 5 independent host vectors, page
    locked or not, give the bits of one device call per vector."""
    m = syn("stencil_40").astype(dtype)
    dm = DeviceMatrix.build(m, fmt, hybrid_width=20)
    try:
        for n, pinned in ((1, True), (2, False), (5, True)):
            xs = [synth.vector(20 + i, m.cols).astype(dtype) for i in range(n)]
            if pinned:
                xs = [torch.from_numpy(x).pin_memory().numpy() for x in xs]
                ys = [torch.full((m.rows,), float("nan"), dtype=torch.from_numpy(xs[0][:1]).dtype).pin_memory().numpy()
                      for _ in range(n)]
            else:
                ys = [np.full(m.rows, np.nan, dtype) for _ in range(n)]
            dm.spmv_host_batch(xs, ys)
            for x, y in zip(xs, ys):
                xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
                yt = torch.empty(m.rows, dtype=xt.dtype, device="cuda")
                dm.spmv(xt, yt)
                torch.cuda.synchronize()
                assert np.array_equal(y.view(np.uint8), yt.cpu().numpy().view(np.uint8))
        dm.spmv_host_batch([], [])
    finally:
        dm.close()


@pytest.mark.parametrize("fmt", [CSR_ADAPTIVE, COO, HYBRID])
def test_host_buffer_call_equals_device_call(fmt):
    m = syn("stencil_40").astype(np.float32)
    x = synth.vector(8, m.cols).astype(np.float32)
    dm = DeviceMatrix.build(m, fmt, hybrid_width=27)
    y_host = np.empty(m.rows, np.float32)
    dm.spmv_host(x, y_host)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty(m.rows, device="cuda")
    dm.spmv(xt, yt)
    torch.cuda.synchronize()
    assert np.array_equal(y_host, yt.cpu().numpy())
    info = dm.info()
    assert info.nnz == m.nnz and info.algorithmic_bytes == m.nnz * 8 + (m.rows + 1) * 4 + m.cols * 4 + m.rows * 4


@pytest.mark.parametrize("fmt", ALL)
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_host_call_with_page_locked_buffers(fmt, dt):
    """Page-locked host y: formats that store rows in order write it directly
    (no copy-out); the result equals the device-buffer call bit for bit."""
    m = syn("stencil_40").astype(dt)
    x = synth.vector(8, m.cols).astype(dt)
    dm = DeviceMatrix.build(m, fmt, hybrid_width=27)
    hx = torch.from_numpy(x).pin_memory().numpy()
    hy_t = torch.full((m.rows,), float("nan"), dtype=torch.from_numpy(x[:1]).dtype).pin_memory()
    hy = hy_t.numpy()
    for _ in range(2):
        dm.spmv_host(hx, hy)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty(m.rows, dtype=xt.dtype, device="cuda")
    dm.spmv(xt, yt)
    torch.cuda.synchronize()
    assert np.array_equal(hy, yt.cpu().numpy())
    dm.close()


@pytest.mark.parametrize("fmt", [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE, COO, SCOO, HYBRID])
def test_full_size_power_law_float32(oracle_lib, fmt):
    """The power-law configuration at full size (4,194,304 rows, ~31M nnz)."""
    if "power_law_full" not in SYN:
        SYN["power_law_full"] = synth.power_law(seed=0).astype(np.float32)
    m = SYN["power_law_full"]
    x = synth.vector(0, m.cols).astype(np.float32)
    hw = F.row_length_quantile(m, 2 / 3)
    y = run(m, fmt, x, hybrid_width=hw)
    check_tol(oracle_lib, m, x, y, f"power-law full fmt{fmt}")
    # size-independent checksum: sum_i y_i = sum_j (column sum of A)_j x_j
    colsum = np.bincount(m.columns, weights=m.data.astype(np.float64), minlength=m.cols)
    assert abs(y.astype(np.float64).sum() - colsum @ x.astype(np.float64)) < 1e-3 * np.abs(m.data).sum() ** 0.5


STREAM_CASES = ["laplacian_16", "powerlaw_small", "edge_long_row", "edge_empty_rows", "random_rect"]


@pytest.mark.parametrize("kernel", [2, 3])
@pytest.mark.parametrize("fmt", [CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE])
@pytest.mark.parametrize("s", ["f32", "f64"])
def test_streaming_csr_kernel(oracle_lib, kernel, fmt, s):
    """The streaming CSR kernel (persistent CTAs, TMA chunks) on fixtures, synthetic and long-row matrices."""
    cfg = {"kernel": kernel}
    for case in STREAM_CASES:
        g = load_golden(case)
        m = golden_csr(g, s)
        x = g["x"].astype(m.dtype)
        check_tol(oracle_lib, m, x, run(m, fmt, x, cfg), f"stream{kernel} {case}/{s}/fmt{fmt}")
    dt = np.float32 if s == "f32" else np.float64
    for m in (syn("power_law_300k").astype(dt), _long_rows_matrix(dt), syn("uniform_rect").astype(dt)):
        x = synth.vector(6, m.cols).astype(dt)
        ys = run(m, fmt, x, cfg, reps=2)
        check_tol(oracle_lib, m, x, ys[0], f"stream{kernel} synthetic fmt{fmt}")
        assert np.array_equal(ys[0], ys[1])


@pytest.mark.parametrize("kernel", [2, 3])
def test_streaming_scalar_exact_within_cta_ranges(oracle_lib, kernel):
    """Scalar streaming keeps CSR order (exact) except rows split between CTA ranges."""
    m = syn("laplacian_512").astype(np.float32)
    x = synth.vector(0, m.cols).astype(np.float32)
    y_ref = oracle_lib.csr_spmv(m.rows, m.row_ptr, m.columns, m.data, x)
    y = run(m, CSR_SCALAR, x, {"kernel": kernel, "assist_threshold": NEVER})
    assert np.count_nonzero(y != y_ref) <= 2 * 148 * 8


@pytest.mark.parametrize("name", ["laplacian_512", "power_law_300k", "stencil_40", "banded_200k", "uniform_rect"])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_scoo_sort_cols_layout(oracle_lib, name, dt):
    """SCOO with each slice in column order (the reference's sort_cols option):
    rows unordered within slices, shared-memory atomics; host-built and
    device-built handles both within tolerance."""
    m = syn(name).astype(dt)
    x = synth.vector(6, m.cols).astype(dt)
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dm = DeviceMatrix.from_scoo(F.scoo_matrix_class(148, 49152, m, sort_cols=True))
    yt = torch.full((m.rows,), float("nan"), dtype=xt.dtype, device="cuda")
    dm.spmv(xt, yt)
    torch.cuda.synchronize()
    check_tol(oracle_lib, m, x, yt.cpu().numpy(), f"{name}/sort_cols host-built")
    dm.close()
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).cuda()
    ci = torch.from_numpy(m.columns.view(np.int32)).cuda()
    va = torch.from_numpy(m.data).cuda()
    dm = DeviceMatrix.from_device_csr(rp, ci, va, m.cols, SCOO, scoo_sort_cols=True)
    yt.fill_(float("nan"))
    dm.spmv(xt, yt)
    torch.cuda.synchronize()
    check_tol(oracle_lib, m, x, yt.cpu().numpy(), f"{name}/sort_cols device-built")
    dm.close()
