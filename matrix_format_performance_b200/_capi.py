"""ctypes binding of include/mfp_spmv.h (libmfp_spmv.so).

The shared library is the product; this module only declares its C
signatures.  Importing it raises if the library has not been built: there is
no Python or CPU fallback for any SpMV entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# MFP_LIBRARY selects another build of the same library (e.g. a tuning variant).
LIB_PATH = Path(os.environ.get("MFP_LIBRARY", Path(__file__).resolve().parent / "lib" / "libmfp_spmv.so"))

u32, u64, i32, f64 = C.c_uint32, C.c_uint64, C.c_int, C.c_double
vp = C.c_void_p
P_u32 = C.POINTER(C.c_uint32)


class MfpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"mfp status {status}: {message}")
        self.status = status


class RowsStatistic(C.Structure):
    _fields_ = [("min_elements_in_rows", u32), ("max_elements_in_rows", u32),
                ("avg_elements_in_rows", u32), ("elements_in_rows_std_deviation", f64)]


class ScooParams(C.Structure):
    _fields_ = [("slices_count", u32), ("slice_size", u32), ("lane_size", u32)]


class CsrConfig(C.Structure):
    _fields_ = [("long_row_threshold", u32), ("vector_lanes", u32), ("bin_nnz", u32),
                ("piece_nnz", u32), ("assist_threshold", u32), ("kernel", u32)]


class MatrixInfo(C.Structure):
    _fields_ = [("format", i32), ("value_type", i32), ("rows", u32), ("cols", u32), ("nnz", u64),
                ("format_bytes", u64), ("algorithmic_bytes", u64), ("device_bytes", u64),
                ("kernel_launches", u32)]


class Measurement(C.Structure):
    _fields_ = [("format", C.c_char * 64), ("elapsed", f64), ("effective_bandwidth", f64),
                ("computational_throughput", f64)]


class DeviceInfo(C.Structure):
    _fields_ = [("device", i32), ("sm_count", i32), ("shared_mem_per_block", u64),
                ("shared_mem_optin", u64), ("l2_bytes", u64), ("global_mem_bytes", u64),
                ("cc_major", i32), ("cc_minor", i32)]


class SynthParams(C.Structure):
    _fields_ = [("kind", i32), ("seed", u64), ("n", u32), ("cols", u32), ("alpha", f64),
                ("k_lo", u32), ("k_hi", u32), ("band", u32)]


# name -> argtypes (restype is int status unless listed in _RESTYPES)
_PROTOS = {
    "mfp_version": [],
    "mfp_status_string": [i32],
    "mfp_last_error": [],
    "mfp_get_device_info": [i32, C.POINTER(DeviceInfo)],
    "mfp_csr_from_coo_f32": [u32, u32, u32, i32, vp, vp, vp, vp, vp, vp],
    "mfp_csr_from_coo_f64": [u32, u32, u32, i32, vp, vp, vp, vp, vp, vp],
    "mfp_get_rows_statistics": [u32, vp, C.POINTER(RowsStatistic)],
    "mfp_ell_width": [u32, vp, P_u32],
    "mfp_ell_from_csr_f32": [u32, vp, vp, vp, u32, vp, vp],
    "mfp_ell_from_csr_f64": [u32, vp, vp, vp, u32, vp, vp],
    "mfp_coo_count": [u32, vp, u32, P_u32],
    "mfp_coo_from_csr_f32": [u32, vp, vp, vp, u32, vp, vp, vp],
    "mfp_coo_from_csr_f64": [u32, vp, vp, vp, u32, vp, vp, vp],
    "mfp_hybrid_width": [u32, vp, f64, P_u32],
    "mfp_row_length_quantile": [u32, vp, f64, P_u32],
    "mfp_scoo_params_compute": [u32, u32, u64, i32, C.POINTER(ScooParams)],
    "mfp_scoo_from_csr_f32": [u32, vp, vp, vp, C.POINTER(ScooParams), vp, vp, vp, vp],
    "mfp_scoo_from_csr_f64": [u32, vp, vp, vp, C.POINTER(ScooParams), vp, vp, vp, vp],
    "mfp_csr_adaptive_row_blocks": [u32, vp, u32, vp, P_u32],
    "mfp_csr_plan_create": [u32, u32, u32, vp, i32, C.POINTER(CsrConfig), C.POINTER(vp)],
    "mfp_csr_plan_destroy": [vp],
    "mfp_csr_plan_get_config": [vp, C.POINTER(i32), C.POINTER(CsrConfig), P_u32, P_u32],
    "mfp_csr_spmv_f32": [vp, vp, vp, vp, vp, vp, vp],
    "mfp_csr_spmv_f64": [vp, vp, vp, vp, vp, vp, vp],
    "mfp_ell_spmv_f32": [u32, u32, u32, vp, vp, vp, vp, vp],
    "mfp_ell_spmv_f64": [u32, u32, u32, vp, vp, vp, vp, vp],
    "mfp_coo_workspace_bytes": [u32, u32, C.POINTER(C.c_size_t)],
    "mfp_coo_spmv_f32": [u32, u32, u32, vp, vp, vp, vp, vp, vp, C.c_size_t, vp],
    "mfp_coo_spmv_f64": [u32, u32, u32, vp, vp, vp, vp, vp, vp, C.c_size_t, vp],
    "mfp_workspace_error": [vp, P_u32],
    "mfp_coo_spmv_f32_noalloc": [u32, u32, u32, vp, vp, vp, vp, vp, vp],
    "mfp_scoo_x_windows": [u32, vp, vp, u32, vp],
    "mfp_scoo_slice_order": [u32, vp, vp],
    "mfp_scoo_spmv_f32": [u32, u32, u32, u32, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp],
    "mfp_scoo_spmv_f64": [u32, u32, u32, u32, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp],
    "mfp_hybrid_workspace_bytes": [u32, u32, C.POINTER(C.c_size_t)],
    "mfp_hybrid_spmv_f32": [u32, u32, u32, vp, vp, u32, vp, vp, vp, vp, vp, vp, C.c_size_t, vp],
    "mfp_hybrid_spmv_f64": [u32, u32, u32, vp, vp, u32, vp, vp, vp, vp, vp, vp, C.c_size_t, vp],
    "mfp_lowp_quantize": [i32, u32, vp, vp, vp, vp],
    "mfp_lowp_deltas": [u32, vp, vp, vp],
    "mfp_lowp_spmv": [i32, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp],
    "mfp_lowp_error": [i32, i32, P_u32],
    "mfp_probe_spmv_loads": [i32, i32, u32, vp, vp, vp, vp, C.c_size_t, vp],
    "mfp_probe_spmv_gather4": [i32, u32, u32, vp, vp, vp, C.c_size_t, vp],
    "mfp_lowp_ell_from_csr": [i32, i32, u32, u32, vp, vp, vp, u32, vp, vp, vp],
    "mfp_lowp_ell_spmv": [i32, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp],
    "mfp_matrix_create_lowp_ell": [i32, i32, u32, u32, u32, vp, vp, vp, C.POINTER(vp)],
    "mfp_matrix_create_lowp": [i32, i32, u32, u32, u32, vp, vp, vp, C.POINTER(vp)],
    "mfp_fill_f32": [u64, vp, C.c_float, vp],
    "mfp_fill_f64": [u64, vp, f64, vp],
    "mfp_matrix_create_csr": [i32, i32, u32, u32, u32, vp, vp, vp, C.POINTER(CsrConfig), C.POINTER(vp)],
    "mfp_matrix_create_ell": [i32, u32, u32, u32, vp, vp, C.POINTER(vp)],
    "mfp_matrix_create_coo": [i32, u32, u32, u32, vp, vp, vp, C.POINTER(vp)],
    "mfp_matrix_create_scoo": [i32, u32, u32, u32, C.POINTER(ScooParams), vp, vp, vp, vp, C.POINTER(vp)],
    "mfp_matrix_create_hybrid": [i32, u32, u32, u32, vp, vp, u32, vp, vp, vp, C.POINTER(vp)],
    "mfp_matrix_destroy": [vp],
    "mfp_matrix_get_info": [vp, C.POINTER(MatrixInfo)],
    "mfp_matrix_spmv": [vp, vp, vp, vp],
    "mfp_matrix_spmv_host": [vp, vp, vp, vp],
    "mfp_matrix_spmv_host_batch": [vp, u32, vp, vp, vp],
    "mfp_measurement_make": [C.c_char_p, f64, f64, f64, C.POINTER(Measurement)],
    "mfp_compare_results_f32": [u32, vp, vp, C.POINTER(f64), P_u32],
    "mfp_compare_results_f64": [u32, vp, vp, C.POINTER(f64), P_u32],
    "mfp_matrix_time": [vp, vp, vp, u32, i32, vp, C.POINTER(f64), C.POINTER(f64)],
    "mfp_synth_csr": [C.POINTER(SynthParams), P_u32, P_u32, C.POINTER(u64), vp, vp, vp],
    "mfp_synth_vector_f64": [u64, u64, f64, f64, vp],
}
_RESTYPES = {"mfp_status_string": C.c_char_p, "mfp_last_error": C.c_char_p}

_lib = None


def load() -> C.CDLL:
    """Loads libmfp_spmv.so; raises if it is missing (build it first)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} not found: build the CUDA library with "
            "`python -m matrix_format_performance_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    for name, args in _PROTOS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, i32)
    _lib = lib
    return lib


def declared_symbols() -> list[str]:
    return list(_PROTOS)


def check(status: int) -> None:
    if status != 0:
        msg = load().mfp_last_error()
        raise MfpError(status, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))


class BatchConfig(C.Structure):
    _fields_ = [("algo", i32), ("csr", CsrConfig)]


class BatchInfo(C.Structure):
    _fields_ = [("matrices", u32), ("rows", u32), ("cols", u32), ("nnz", u32), ("algorithmic_bytes", u64),
                ("device_bytes", u64), ("config", BatchConfig), ("kernel_launches", u32)]


_PROTOS.update({
    "mfp_batch_create": [i32, u32, vp, vp, vp, vp, vp, C.POINTER(vp)],
    "mfp_batch_destroy": [vp],
    "mfp_batch_offsets": [vp, vp, vp],
    "mfp_batch_get_info": [vp, C.POINTER(BatchInfo)],
    "mfp_batch_set_config": [vp, C.POINTER(BatchConfig)],
    "mfp_batch_autotune": [vp, vp, vp, u32, vp, C.POINTER(BatchConfig), C.POINTER(f64)],
    "mfp_batch_spmv": [vp, vp, vp, vp],
    "mfp_batch_graph_launch": [vp, vp, vp, vp],
})
_PROTOS.update({
    "mfp_selector_features": [u32, u32, vp, vp, vp],
    "mfp_mlp_param_count": [],
    "mfp_mlp_forward": [vp, vp, u32, vp, vp, vp, vp],
    "mfp_mlp_backward": [vp, vp, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp],
    "mfp_mlp_adam": [vp, vp, vp, vp, u32, C.c_float, C.c_float, C.c_float, C.c_float, u32, vp],
})
_RESTYPES["mfp_mlp_param_count"] = u32


class DeviceBuildOptions(C.Structure):
    _fields_ = [("csr", C.POINTER(CsrConfig)), ("ell_width", u32), ("scoo", C.POINTER(ScooParams)),
                ("scoo_sort_cols", u32)]


ELL_WIDTH_LONGEST = 0xFFFFFFFF
_PROTOS.update({
    "mfp_dev_rows_statistics": [u32, vp, C.POINTER(RowsStatistic), vp],
    "mfp_dev_check_csr": [u32, u32, u32, vp, vp, vp],
    "mfp_dev_coo_count": [u32, vp, u32, P_u32, vp],
    "mfp_dev_coo_from_csr": [i32, u32, vp, vp, vp, u32, vp, vp, vp, vp],
    "mfp_dev_ell_from_csr": [i32, u32, vp, vp, vp, u32, vp, vp, vp],
    "mfp_dev_scoo_from_csr": [i32, u32, u32, vp, vp, vp, C.POINTER(ScooParams), vp, vp, vp, vp, vp],
    "mfp_dev_scoo_x_windows": [u32, vp, vp, u32, vp, vp],
    "mfp_dev_scoo_sort_cols": [i32, u32, u32, u32, u32, vp, vp, vp, vp],
    "mfp_scoo_sort_cols_f32": [u32, vp, vp, vp, vp],
    "mfp_scoo_sort_cols_f64": [u32, vp, vp, vp, vp],
    "mfp_scoo_spmv_unsorted_f32": [u32, u32, u32, u32, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp],
    "mfp_scoo_spmv_unsorted_f64": [u32, u32, u32, u32, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp],
    "mfp_dev_csr_from_coo": [i32, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp],
    "mfp_dev_scratch_bytes": [C.POINTER(u64)],
    "mfp_dev_scratch_release": [],
    "mfp_matrix_create_device": [i32, i32, u32, u32, u32, vp, vp, vp, C.POINTER(DeviceBuildOptions),
                                 C.POINTER(vp)],
})
