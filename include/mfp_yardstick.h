/* Vendor yardstick: cuSPARSE's generic SpMV (cusparseSpMV) on the engine's
 * CSR and COO layouts, timed the way the engine's kernels are timed, so the
 * engine's formats can be compared with NVIDIA's library on the same matrix.
 * It replaces the reference's cuSPARSE comparator, "GPU CSR (cuSparse)"
 * (gpu/gpu_matrix_multiplier.cu:135-257), whose legacy cusparse?csrmv calls
 * no longer exist.  Library code: not part of the engine's SpMV path
 * (libmfp_yardstick.so, linked against libcusparse).  Indices are passed as
 * 32-bit (uint32 ids below 2^31). */
#ifndef MFP_YARDSTICK_H
#define MFP_YARDSTICK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* format: 0 CSR (index = row_ptr, rows+1 entries), 1 COO (index = row ids,
 * nnz entries, sorted by row).  alg: 0 CUSPARSE_SPMV_ALG_DEFAULT, 1
 * CSR_ALG1 / COO_ALG1, 2 CSR_ALG2 / COO_ALG2.  value_type 0 float, 1 double.
 * Device arrays; y = A*x on `stream`.  With reps > 0, times reps launches
 * (CUDA events, L2 flushed before each when flush_l2) after one warm-up and
 * returns the median in *median_s; reps == 0 runs once.  Synchronous. */
int mfp_cusparse_spmv(int format, int alg, int value_type, uint32_t rows, uint32_t cols, uint32_t nnz,
                      const uint32_t *index, const uint32_t *col_ids, const void *values, const void *x, void *y,
                      uint32_t reps, int flush_l2, void *stream, double *median_s);
const char *mfp_cusparse_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
