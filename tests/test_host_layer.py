"""The C++ host layer (matrix_format_performance_b200/host): the reference's
class and operator interface over the C ABI.

CPU: the Matrix Market reader, and the matrix classes built from a file in
C++ are bit-exact with the fixtures the reference's own sources produced.
GPU: the main.cpp-style driver runs every operator on small matrices and
writes the reference's result files with its labels; every GPU result passes
the reference's compare_results check (relative squared error <= 1e-9).
"""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import golden_cases, load_golden
from matrix_format_performance_b200 import build as B
from matrix_format_performance_b200 import formats as F
from matrix_format_performance_b200 import synth

ROOT = Path(__file__).resolve().parent.parent


def write_mtx(path: Path, rows, cols, ri, ci, v, symmetry="general", field="real"):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {symmetry}\n% written by the tests\n")
        f.write(f"{rows} {cols} {len(ri)}\n")
        for r, c, x in zip(ri, ci, v):
            f.write(f"{int(r) + 1} {int(c) + 1}" + ("" if field == "pattern" else f" {float(x)!r}") + "\n")


@pytest.fixture(scope="module")
def classes_check(tmp_path_factory):
    return B.host_compile(ROOT / "tests" / "cpp" / "host_classes_check.cpp",
                          tmp_path_factory.mktemp("cpp") / "host_classes_check")


@pytest.mark.parametrize("case", golden_cases())
def test_host_classes_match_reference_fixtures(classes_check, tmp_path, case):
    g = load_golden(case)
    mtx = tmp_path / "m.mtx"
    write_mtx(mtx, int(g["rows"][0]), int(g["cols"][0]), g["row_ids"], g["col_ids"], g["values"])
    out = tmp_path / "out"
    out.mkdir()
    subprocess.run([str(classes_check), str(mtx), str(out)], check=True)

    def arr(name, dt):
        return np.fromfile(out / f"{name}.bin", dtype=dt)
    for dt, s in ((np.float32, "f32"), (np.float64, "f64")):
        for k in ("csr_row_ptr", "csr_columns", "coo_cols", "coo_rows", "hyb_coo_cols", "hyb_coo_rows",
                  "scoo_params", "scoo_c_index", "scoo_r_index", "scoo_slices_ptr", "scoo_small_params",
                  "scoo_small_c_index", "scoo_small_r_index", "scoo_small_slices_ptr"):
            assert np.array_equal(arr(f"{k}_{s}", np.uint32), g[f"{k}_{s}"]), (k, s)
        for k in ("csr_data", "coo_data", "hyb_coo_data", "scoo_values", "scoo_small_values"):
            assert np.array_equal(arr(f"{k}_{s}", dt), g[f"{k}_{s}"]), (k, s)
        assert np.array_equal(arr(f"stats_u32_{s}", np.uint32), g["stats_u32"])
        assert arr(f"stats_std_{s}", np.float64)[0] == g["stats_std"][0]
        if f"ell_data_{s}" in g:
            assert arr(f"ell_width_{s}", np.uint32)[0] == g[f"ell_width_{s}"][0]
            assert np.array_equal(arr(f"ell_data_{s}", dt), g[f"ell_data_{s}"])
            assert np.array_equal(arr(f"ell_columns_{s}", np.uint32), g[f"ell_columns_{s}"])
        if f"hyb_ell_data_{s}" in g:
            assert arr(f"hyb_width_{s}", np.uint32)[0] == g[f"hyb_width_{s}"][0]
            assert np.array_equal(arr(f"hyb_ell_data_{s}", dt), g[f"hyb_ell_data_{s}"])
            assert np.array_equal(arr(f"hyb_ell_columns_{s}", np.uint32), g[f"hyb_ell_columns_{s}"])


def test_reader_symmetric_and_pattern(classes_check, tmp_path):
    """symmetric files are expanded (mirrored off-diagonal entries), pattern
    entries read as 1: the CSR of the expanded file equals the general one."""
    ri, ci, v = [0, 1, 2, 2], [0, 0, 1, 2], [4.0, -1.0, -2.5, 3.0]
    write_mtx(tmp_path / "s.mtx", 3, 3, ri, ci, v, symmetry="symmetric")
    gri = [0, 1, 0, 2, 1, 2]
    gci = [0, 0, 1, 1, 2, 2]
    gv = [4.0, -1.0, -1.0, -2.5, -2.5, 3.0]
    write_mtx(tmp_path / "g.mtx", 3, 3, gri, gci, gv)
    write_mtx(tmp_path / "p.mtx", 3, 3, gri, gci, gv, field="pattern")
    res = {}
    for n in ("s", "g", "p"):
        out = tmp_path / n
        out.mkdir()
        subprocess.run([str(classes_check), str(tmp_path / f"{n}.mtx"), str(out)], check=True)
        res[n] = (np.fromfile(out / "csr_row_ptr_f64.bin", np.uint32), np.fromfile(out / "csr_columns_f64.bin", np.uint32),
                  np.fromfile(out / "csr_data_f64.bin", np.float64))
    for a, b in zip(res["s"], res["g"]):
        assert np.array_equal(a, b)
    assert np.array_equal(res["p"][2], np.ones(6)) and np.array_equal(res["p"][1], res["g"][1])


def test_reader_rejects_malformed(classes_check, tmp_path):
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    r = subprocess.run([str(classes_check), str(bad), str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 2 and "coordinate" in r.stderr
    bad.write_text("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n")
    r = subprocess.run([str(classes_check), str(bad), str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 2 and "out of range" in r.stderr


@pytest.mark.gpu
def test_driver_runs_every_operator(tmp_path):
    drv = B.build_driver()
    files = []
    # row lengths capped at 200 so that every matrix also runs the ELL operator
    mats = {"powerlaw_20k.mtx": synth.power_law(rows=20_000, k_hi=200, seed=3),
            "uniform_30k.mtx": synth.uniform(30_000, 0, 40, seed=4),
            "banded_50k.mtx": synth.banded(n=50_000, seed=5),
            "laplacian_64.mtx": synth.laplacian_2d(64)}
    for name, m in mats.items():
        rows = np.repeat(np.arange(m.rows), np.diff(m.row_ptr.astype(np.int64)))
        write_mtx(tmp_path / name, m.rows, m.cols, rows, m.columns, m.data)
        files.append(str(tmp_path / name))
    (tmp_path / "list.txt").write_text("\n".join(files) + "\n")
    r = subprocess.run([str(drv), str(tmp_path / "list.txt")], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "ERROR" not in r.stderr, r.stderr[-2000:]
    labels = {"CPU CSR", "CPU CSR Parallel", "GPU CSR", "GPU CSR (vector)", "GPU CSR-Adaptive",
              "GPU CSR (cuSparse)", "GPU ELL",
              "GPU COO", "GPU SCOO", "GPU Hybrid (TODO)", "GPU Hybrid (atomic)"}
    info = json.loads((tmp_path / "matrices_info.json").read_text())
    assert set(info) == set(mats)
    for prec in ("float", "double"):
        t = json.loads((tmp_path / f"{prec}.json").read_text())
        bw = json.loads((tmp_path / f"{prec}_effective_bandwidth.json").read_text())
        err = json.loads((tmp_path / f"{prec}_max_error.json").read_text())
        assert set(t) == set(mats)
        for name in mats:
            assert labels <= set(t[name]), (prec, name, set(t[name]))
            assert all(v > 0 for v in t[name].values())
            assert all(v > 0 for k, v in bw[name].items())
            assert max(err[name].values()) <= 1e-9, (prec, name, err[name])
        for name, m in mats.items():
            assert info[name]["nnz"] == m.nnz and info[name]["rows"] == m.rows


@pytest.mark.gpu
def test_driver_hybrid_sweep(tmp_path):
    """--hybrid-sweep: the reference's disabled sweep (percent 0, 0.35, 0.70),
    keyed by percent; a percent whose ELL part exceeds 64x the CSR layout is
    skipped (the power-law matrix's 0.70 width)."""
    drv = B.build_driver()
    mats = {"banded_20k.mtx": synth.banded(n=20_000, seed=6),
            "powerlaw_20k.mtx": synth.power_law(rows=20_000, k_hi=2_000, seed=7)}
    for name, m in mats.items():
        rows = np.repeat(np.arange(m.rows), np.diff(m.row_ptr.astype(np.int64)))
        write_mtx(tmp_path / name, m.rows, m.cols, rows, m.columns, m.data)
    (tmp_path / "list.txt").write_text("\n".join(str(tmp_path / n) for n in mats) + "\n")
    r = subprocess.run([str(drv), "--hybrid-sweep", str(tmp_path / "list.txt")], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    for prec in ("float", "double"):
        t = json.loads((tmp_path / f"{prec}.json").read_text())
        err = json.loads((tmp_path / f"{prec}_max_error.json").read_text())
        for name, m in mats.items():
            stats = F.get_rows_statistics(m)
            csr_bytes = m.nnz * (4 if prec == "float" else 8) + m.nnz * 4
            for pct in (0, 35, 70):
                w = int(stats.avg_elements_in_rows + (stats.max_elements_in_rows - stats.avg_elements_in_rows) * pct / 100)
                fits = w * m.rows * ((4 if prec == "float" else 8) + 4) <= 64 * csr_bytes
                for label in ("GPU Hybrid (TODO)", "GPU Hybrid (atomic)"):
                    key = f"{label} {pct}%"
                    assert (key in t[name]) == fits, (prec, name, key, w)
                    if fits:
                        assert t[name][key] > 0 and err[name][key] <= 1e-9
