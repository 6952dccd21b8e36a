"""ctypes bindings of the oracle libraries (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libmfp_ref.so"
SYNTH_SO = HERE / "libmfp_synth.so"
# the reference checkout: MFP_REFERENCE_SRC, else the default of oracle/Makefile
REFERENCE_SRC = os.environ.get("MFP_REFERENCE_SRC")

vp, u32, u64, i32, i64, f64 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_longlong, C.c_double


def _p(a):
    if a is None:
        return None
    if a.size == 0:
        return None
    assert a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


def _ref_dir() -> Path | None:
    """The reference checkout the recipe would compile, or None when absent."""
    if REFERENCE_SRC:
        d = Path(REFERENCE_SRC)
    else:
        r = subprocess.run(["make", "-s", "-C", str(HERE), "print-ref"], capture_output=True, text=True)
        d = Path(r.stdout.strip()) if r.returncode == 0 and r.stdout.strip() else None
    return d if d is not None and (d / "common" / "matrix_converter.cpp").exists() else None


def build(ref: bool | None = None) -> None:
    """Builds liboracle.so and libmfp_synth.so, and _ref/libmfp_ref.so when the
    reference sources exist (MFP_REFERENCE_SRC, else oracle/Makefile's REF)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so", "libmfp_synth.so"], check=True)
    src = _ref_dir()
    if ref is None:
        ref = src is not None
    if ref:
        if src is None:
            raise FileNotFoundError("reference sources not found: set MFP_REFERENCE_SRC")
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={src}"], check=True)


class Oracle:
    """The C restatement (oracle.c)."""

    def __init__(self, path: Path = ORACLE_SO):
        self.lib = C.CDLL(str(path))
        L = self.lib
        for n in ("oracle_csr_spmv_f32", "oracle_csr_spmv_f64", "oracle_csr_spmv_reduce_order_f32",
                  "oracle_csr_spmv_reduce_order_f64"):
            getattr(L, n).argtypes = [u32, vp, vp, vp, vp, vp]
            getattr(L, n).restype = None
        for n in ("oracle_ell_spmv_f32", "oracle_ell_spmv_f64"):
            getattr(L, n).argtypes = [u32, u32, vp, vp, vp, vp]
            getattr(L, n).restype = None
        L.oracle_csr_spmv_ld.argtypes = [u32, vp, vp, vp, vp, vp, vp]
        L.oracle_csr_spmv_ld.restype = None
        L.oracle_csr_spmv_parallel.argtypes = [u32, i32, u32, vp, vp, vp, vp, vp]
        L.oracle_csr_spmv_parallel.restype = f64
        for n in ("oracle_csr_from_coo_f32", "oracle_csr_from_coo_f64"):
            getattr(L, n).argtypes = [u32, u32, vp, vp, vp, vp, vp, vp]
        L.oracle_rows_statistics.argtypes = [u32, vp, vp, C.POINTER(f64)]
        L.oracle_rows_statistics.restype = None
        for n in ("oracle_ell_from_csr_f32", "oracle_ell_from_csr_f64"):
            getattr(L, n).argtypes = [u32, vp, vp, vp, u32, vp, vp]
            getattr(L, n).restype = None
        for n in ("oracle_coo_from_csr_f32", "oracle_coo_from_csr_f64"):
            getattr(L, n).argtypes = [u32, vp, vp, vp, u32, vp, vp, vp]
            getattr(L, n).restype = u32
        L.oracle_hybrid_width.argtypes = [u32, vp, f64]
        L.oracle_hybrid_width.restype = u32
        L.oracle_scoo_params.argtypes = [u32, u32, u64, u32, vp]
        L.oracle_scoo_params.restype = None
        for n in ("oracle_scoo_from_csr_f32", "oracle_scoo_from_csr_f64"):
            getattr(L, n).argtypes = [u32, vp, vp, vp, u32, u32, vp, vp, vp, vp]
            getattr(L, n).restype = None
        L.oracle_fill_row_blocks.argtypes = [i32, u32, vp, u32, vp]
        L.oracle_fill_row_blocks.restype = u32

    @staticmethod
    def _sfx(dtype) -> str:
        return "f64" if np.dtype(dtype) == np.float64 else "f32"

    # -- SpMV ---------------------------------------------------------------
    def csr_spmv(self, rows, row_ptr, cols, data, x, reduce_order=False) -> np.ndarray:
        y = np.empty(rows, data.dtype)
        xx = np.ascontiguousarray(x, data.dtype)  # keep alive across the call
        fn = f"oracle_csr_spmv{'_reduce_order' if reduce_order else ''}_{self._sfx(data.dtype)}"
        getattr(self.lib, fn)(rows, _p(row_ptr), _p(cols), _p(data), _p(xx), _p(y))
        return y

    def ell_spmv(self, rows, width, data, cols, x) -> np.ndarray:
        y = np.empty(rows, data.dtype)
        xx = np.ascontiguousarray(x, data.dtype)
        getattr(self.lib, f"oracle_ell_spmv_{self._sfx(data.dtype)}")(rows, width, _p(data), _p(cols), _p(xx), _p(y))
        return y

    def csr_spmv_exact(self, rows, row_ptr, cols, data, x) -> tuple[np.ndarray, np.ndarray]:
        """(y, sum |a x|) in extended precision; data/x are converted to float64 exactly."""
        y = np.empty(rows, np.float64)
        ab = np.empty(rows, np.float64)
        dd = np.ascontiguousarray(data, np.float64)
        xx = np.ascontiguousarray(x, np.float64)
        self.lib.oracle_csr_spmv_ld(rows, _p(row_ptr), _p(cols), _p(dd), _p(xx), _p(y), _p(ab))
        return y, ab

    def csr_spmv_parallel(self, threads, rows, row_ptr, cols, data, x) -> tuple[np.ndarray, float]:
        y = np.empty(rows, data.dtype)
        xx = np.ascontiguousarray(x, data.dtype)
        t = self.lib.oracle_csr_spmv_parallel(threads, int(data.dtype == np.float64), rows, _p(row_ptr), _p(cols),
                                              _p(data), _p(xx), _p(y))
        return y, t

    # -- converters ---------------------------------------------------------
    def csr_from_coo(self, rows, row_ids, col_ids, values, dtype):
        nnz = values.size
        rp = np.empty(rows + 1, np.uint32)
        ci = np.empty(nnz, np.uint32)
        d = np.empty(nnz, dtype)
        getattr(self.lib, f"oracle_csr_from_coo_{self._sfx(dtype)}")(rows, nnz, _p(row_ids), _p(col_ids),
                                                                     _p(values), _p(rp), _p(ci), _p(d))
        return rp, ci, d

    def rows_statistics(self, rows, row_ptr):
        out = np.empty(3, np.uint32)
        sd = C.c_double()
        self.lib.oracle_rows_statistics(rows, _p(row_ptr), _p(out), C.byref(sd))
        return int(out[0]), int(out[1]), int(out[2]), sd.value

    def ell(self, rows, row_ptr, cols, data, width):
        ed = np.empty(rows * width, data.dtype)
        ec = np.empty(rows * width, np.uint32)
        getattr(self.lib, f"oracle_ell_from_csr_{self._sfx(data.dtype)}")(rows, _p(row_ptr), _p(cols), _p(data),
                                                                          width, _p(ed), _p(ec))
        return ed, ec

    def coo(self, rows, row_ptr, cols, data, start=0):
        fn = getattr(self.lib, f"oracle_coo_from_csr_{self._sfx(data.dtype)}")
        n = fn(rows, _p(row_ptr), _p(cols), _p(data), start, None, None, None)
        cd = np.empty(n, data.dtype)
        cc = np.empty(n, np.uint32)
        cr = np.empty(n, np.uint32)
        fn(rows, _p(row_ptr), _p(cols), _p(data), start, _p(cd) or C.c_void_p(1), _p(cc), _p(cr))
        return cd, cc, cr

    def hybrid_width(self, rows, row_ptr, percent) -> int:
        return int(self.lib.oracle_hybrid_width(rows, _p(row_ptr), percent))

    def scoo_params(self, rows, sm_count, smem, dtype):
        out = np.empty(3, np.uint32)
        self.lib.oracle_scoo_params(rows, sm_count, smem, np.dtype(dtype).itemsize, _p(out))
        return int(out[0]), int(out[1]), int(out[2])

    def scoo(self, rows, row_ptr, cols, data, sm_count, smem):
        slices, size, lane = self.scoo_params(rows, sm_count, smem, data.dtype)
        nnz = data.size
        v = np.empty(nnz, data.dtype)
        ci = np.empty(nnz, np.uint32)
        ri = np.empty(nnz, np.uint32)
        sp = np.empty(slices + 1, np.uint32)
        getattr(self.lib, f"oracle_scoo_from_csr_{self._sfx(data.dtype)}")(rows, _p(row_ptr), _p(cols), _p(data),
                                                                           slices, size, _p(v), _p(ci), _p(ri),
                                                                           _p(sp))
        return (slices, size, lane), v, ci, ri, sp

    def fill_row_blocks(self, rows, row_ptr, per_wg=64) -> np.ndarray:
        n = self.lib.oracle_fill_row_blocks(0, rows, _p(row_ptr), per_wg, None)
        out = np.empty(n + 1, np.uint32)
        self.lib.oracle_fill_row_blocks(1, rows, _p(row_ptr), per_wg, _p(out))
        return out


class RefLib:
    """The reference's own code (oracle/_ref/libmfp_ref.so)."""

    def __init__(self, path: Path = REF_SO):
        self.lib = C.CDLL(str(path))
        L = self.lib
        coo_in = [u32, u32, u32, vp, vp, vp]
        for s in ("f32", "f64"):
            getattr(L, f"ref_csr_{s}").argtypes = coo_in + [vp, vp, vp]
            getattr(L, f"ref_ell_{s}").argtypes = coo_in + [i64, vp, vp]
            getattr(L, f"ref_ell_{s}").restype = u32
            getattr(L, f"ref_coo_{s}").argtypes = coo_in + [i64, vp, vp, vp]
            getattr(L, f"ref_coo_{s}").restype = u32
            getattr(L, f"ref_hybrid_{s}").argtypes = coo_in + [f64, vp, vp, vp, vp, vp, vp, vp]
            getattr(L, f"ref_hybrid_{s}").restype = None
            getattr(L, f"ref_scoo_{s}").argtypes = coo_in + [u32, C.c_size_t, vp, vp, vp, vp, vp]
            getattr(L, f"ref_scoo_{s}").restype = None
            getattr(L, f"ref_spmv_{s}").argtypes = coo_in + [i32, vp]
            getattr(L, f"ref_spmv_{s}").restype = None
        L.ref_rows_statistics.argtypes = coo_in + [vp, C.POINTER(f64)]
        L.ref_rows_statistics.restype = None
        L.ref_fill_row_blocks.argtypes = [i32, u32, vp, vp]
        L.ref_fill_row_blocks.restype = u32
        L.ref_measurement.argtypes = [C.c_char_p, f64, f64, f64, vp]
        L.ref_measurement.restype = None
        L.ref_bench_create.argtypes = [i32, u32, u32, u32, vp, vp, vp]
        L.ref_bench_create.restype = vp
        L.ref_bench_run.argtypes = [vp, vp]
        L.ref_bench_run.restype = f64
        L.ref_bench_destroy.argtypes = [vp]
        L.ref_bench_destroy.restype = None

    @staticmethod
    def _sfx(dtype) -> str:
        return "f64" if np.dtype(dtype) == np.float64 else "f32"

    @staticmethod
    def _coo(m):
        return (m.rows, m.cols, m.nnz, _p(m.row_ids), _p(m.col_ids), _p(m.data))

    def csr(self, m, dtype):
        rp = np.empty(m.rows + 1, np.uint32)
        ci = np.empty(m.nnz, np.uint32)
        d = np.empty(m.nnz, dtype)
        getattr(self.lib, f"ref_csr_{self._sfx(dtype)}")(*self._coo(m), _p(rp), _p(ci), _p(d))
        return rp, ci, d

    def rows_statistics(self, m):
        out = np.empty(3, np.uint32)
        sd = C.c_double()
        self.lib.ref_rows_statistics(*self._coo(m), _p(out), C.byref(sd))
        return int(out[0]), int(out[1]), int(out[2]), sd.value

    def ell(self, m, dtype, width=-1):
        fn = getattr(self.lib, f"ref_ell_{self._sfx(dtype)}")
        w = fn(*self._coo(m), width, None, None)
        d = np.empty(m.rows * w, dtype)
        c = np.empty(m.rows * w, np.uint32)
        if d.size:
            fn(*self._coo(m), width, _p(d), _p(c))
        return w, d, c

    def coo(self, m, dtype, start=-1):
        fn = getattr(self.lib, f"ref_coo_{self._sfx(dtype)}")
        n = fn(*self._coo(m), start, None, None, None)
        d = np.empty(n, dtype)
        c = np.empty(n, np.uint32)
        r = np.empty(n, np.uint32)
        if n:
            fn(*self._coo(m), start, _p(d), _p(c), _p(r))
        return d, c, r

    def hybrid(self, m, dtype, percent):
        fn = getattr(self.lib, f"ref_hybrid_{self._sfx(dtype)}")
        w, n = C.c_uint32(), C.c_uint32()
        fn(*self._coo(m), percent, C.byref(w), C.byref(n), None, None, None, None, None)
        ed = np.empty(m.rows * w.value, dtype)
        ec = np.empty(m.rows * w.value, np.uint32)
        cd = np.empty(n.value, dtype)
        cc = np.empty(n.value, np.uint32)
        cr = np.empty(n.value, np.uint32)
        dummy = np.empty(1, np.uint32)
        fn(*self._coo(m), percent, C.byref(w), C.byref(n), _p(ed) or _p(dummy), _p(ec) or _p(dummy),
           _p(cd) or _p(dummy), _p(cc) or _p(dummy), _p(cr) or _p(dummy))
        return w.value, ed, ec, cd, cc, cr

    def scoo(self, m, dtype, sm_count, smem):
        fn = getattr(self.lib, f"ref_scoo_{self._sfx(dtype)}")
        prm = np.empty(3, np.uint32)
        fn(*self._coo(m), sm_count, smem, _p(prm), None, None, None, None)
        v = np.empty(m.nnz, dtype)
        ci = np.empty(m.nnz, np.uint32)
        ri = np.empty(m.nnz, np.uint32)
        sp = np.empty(int(prm[0]) + 1, np.uint32)
        dummy = np.empty(1, np.float64)
        fn(*self._coo(m), sm_count, smem, _p(prm), _p(v) or _p(dummy), _p(ci) or _p(dummy), _p(ri) or _p(dummy),
           _p(sp))
        return (int(prm[0]), int(prm[1]), int(prm[2])), v, ci, ri, sp

    def spmv_ones(self, m, dtype, reduce_order=False) -> np.ndarray:
        """The reference CPU loop, y = A * 1 (its x is fixed to 1)."""
        y = np.empty(m.rows, dtype)
        getattr(self.lib, f"ref_spmv_{self._sfx(dtype)}")(*self._coo(m), int(reduce_order), _p(y))
        return y

    def fill_row_blocks(self, rows, row_ptr) -> np.ndarray:
        n = self.lib.ref_fill_row_blocks(0, rows, _p(row_ptr), None)
        out = np.empty(n + 1, np.uint32)
        self.lib.ref_fill_row_blocks(1, rows, _p(row_ptr), _p(out))
        return out

    def measurement(self, fmt: str, elapsed, nbytes, ops):
        out = np.empty(3, np.float64)
        self.lib.ref_measurement(fmt.encode(), elapsed, nbytes, ops, _p(out))
        return tuple(out)


_oracle = None
_ref = None


def load_oracle() -> Oracle:
    global _oracle
    if _oracle is None:
        if not ORACLE_SO.exists():
            build(ref=False)
        _oracle = Oracle()
    return _oracle


def load_ref() -> RefLib | None:
    """The compiled reference, or None when it was not built (no reference sources)."""
    global _ref
    if _ref is None and REF_SO.exists():
        _ref = RefLib()
    return _ref


_synth = None


def load_synth() -> C.CDLL:
    """The seeded matrix generator alone (libmfp_synth.so: the engine's
    generator source built without the engine), so the benchmark's reference
    arm maps no engine library."""
    global _synth
    if _synth is None:
        if not SYNTH_SO.exists():
            build(ref=False)
        _synth = C.CDLL(str(SYNTH_SO))
        _synth.mfp_synth_csr.restype = i32
        _synth.mfp_synth_csr.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    return _synth


def synth_power_law(rows: int, seed: int, cols: int, alpha: float = 2.0, k_lo: int = 1, k_hi: int = 50_000):
    """(rows, cols, row_ptr, columns, values float64) of the seeded power-law
    matrix: the same arrays as the engine's synth.power_law."""
    from matrix_format_performance_b200._capi import SynthParams  # a ctypes struct; loads no library
    lib = load_synth()
    p = SynthParams(1, seed, rows, cols, alpha, k_lo, k_hi, 0)
    r, c, n = C.c_uint32(), C.c_uint32(), C.c_uint64()
    if lib.mfp_synth_csr(C.byref(p), C.byref(r), C.byref(c), C.byref(n), None, None, None):
        raise RuntimeError("mfp_synth_csr (size query) failed")
    rp = np.empty(r.value + 1, np.uint32)
    ci = np.empty(max(1, n.value), np.uint32)
    va = np.empty(max(1, n.value), np.float64)
    if lib.mfp_synth_csr(C.byref(p), C.byref(r), C.byref(c), C.byref(n), _p(rp), C.c_void_p(ci.ctypes.data),
                         C.c_void_p(va.ctypes.data)):
        raise RuntimeError("mfp_synth_csr failed")
    return r.value, c.value, rp, ci[:n.value], va[:n.value]
