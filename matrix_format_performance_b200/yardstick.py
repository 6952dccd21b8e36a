"""cuSPARSE yardstick (libmfp_yardstick.so): cusparseSpMV on the engine's CSR
and COO layouts, for comparison with the engine's kernels.  Library code,
not the engine's SpMV path."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libmfp_yardstick.so"
_lib = None
CSR, COO = 0, 1
ALG_DEFAULT, ALG1, ALG2 = 0, 1, 2


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} not found: python -m matrix_format_performance_b200.build")
        lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
        vp, u32 = C.c_void_p, C.c_uint32
        lib.mfp_cusparse_spmv.argtypes = [C.c_int, C.c_int, C.c_int, u32, u32, u32, vp, vp, vp, vp, vp, u32, C.c_int,
                                          vp, C.POINTER(C.c_double)]
        lib.mfp_cusparse_spmv.restype = C.c_int
        lib.mfp_cusparse_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def spmv(fmt, alg, rows, cols, nnz, index, col_ids, values, x, y, reps=0, flush_l2=True, stream=None) -> float:
    """y = A x with cuSPARSE (torch tensors for the device arrays); with reps,
    the median time in seconds."""
    import torch
    lib = load()
    vt = 1 if values.dtype == torch.float64 else 0
    med = C.c_double(0.0)
    s = stream if stream is not None else torch.cuda.current_stream()
    st = lib.mfp_cusparse_spmv(fmt, alg, vt, rows, cols, nnz, C.c_void_p(index.data_ptr()),
                               C.c_void_p(col_ids.data_ptr()), C.c_void_p(values.data_ptr()),
                               C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), reps, int(flush_l2),
                               C.c_void_p(s.cuda_stream), C.byref(med))
    if st:
        raise RuntimeError(f"cuSPARSE: {lib.mfp_cusparse_last_error().decode()}")
    return med.value
