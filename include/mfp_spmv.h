/*
 * mfp_spmv.h — C ABI of the B200 (sm_100a) SpMV engine.
 *
 * Drop-in boundary for the per-format SpMV path of
 * gevtushenko/matrix_format_performance.  The reference exposes that path as
 * C++ templates (gpu/gpu_matrix_multiplier.h:14-152, gpu/csr_adaptive_spmv.h:13-23,
 * gpu/scoo_spmv.h:12-23) over the layouts built by common/matrix_converter.cpp
 * and common/scoo_matrix_class.cpp.  This header flattens that surface into
 * plain C: pointers, sizes, an int status, and opaque handles.  The C++
 * compatibility headers under matrix_format_performance_b200/csrc/compat/
 * rebuild the reference's template signatures on top of it.
 *
 * Conventions
 *  - Every function returns an int status (mfp_status).  On failure a message
 *    is available from mfp_last_error() (thread-local).
 *  - "device" pointers are CUDA global-memory addresses on the current device;
 *    "host" pointers are ordinary process memory.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    Device-pointer entry points only enqueue work; they never synchronise.
 *  - Index arrays are uint32 (the reference uses unsigned int,
 *    common/matrix_converter.h:36-38).  Value arrays are float (f32) or
 *    double (f64), as the reference instantiates (gpu_matrix_multiplier.cu:1219-1302).
 *  - Device arrays passed to the SpMV entry points should start on a 32-byte
 *    boundary (cudaMalloc gives 256): kernels that read a whole 32-byte sector
 *    per thread use one 256-bit load there, two 16-byte loads on 16-byte
 *    boundaries, and unaligned arrays take a slower path.
 */
#ifndef MFP_SPMV_H
#define MFP_SPMV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MFP_VERSION 100

typedef enum mfp_status {
  MFP_SUCCESS = 0,
  MFP_ERROR_INVALID_VALUE = 1,  /* null pointer, inconsistent sizes, bad enum */
  MFP_ERROR_CUDA = 2,           /* a CUDA runtime call failed */
  MFP_ERROR_OUT_OF_MEMORY = 3,  /* device or host allocation failed */
  MFP_ERROR_TOO_LARGE = 4,      /* layout would exceed 32-bit indexing or memory */
  MFP_ERROR_NOT_SUPPORTED = 5,  /* e.g. a non-general storage scheme */
  MFP_ERROR_DEVICE_WAIT = 6     /* a bounded device-side wait gave up */
} mfp_status;

/* MFP_BF16 / MFP_F16: 16-bit stored values of the reduced-precision CSR
 * layout (x, y and the accumulation stay FP32). */
typedef enum mfp_value_type { MFP_F32 = 0, MFP_F64 = 1, MFP_BF16 = 2, MFP_F16 = 3 } mfp_value_type;

/* ------------------------------------------------------------------------- */
/* Library                                                                   */
/* ------------------------------------------------------------------------- */
int mfp_version(void);
const char *mfp_status_string(int status);
const char *mfp_last_error(void);

typedef struct mfp_device_info {
  int device;
  int sm_count;                  /* cudaDeviceProp::multiProcessorCount */
  uint64_t shared_mem_per_block; /* cudaDeviceProp::sharedMemPerBlock (48 KiB) */
  uint64_t shared_mem_optin;     /* sharedMemPerBlockOptin (227 KiB on B200) */
  uint64_t l2_bytes;
  uint64_t global_mem_bytes;
  int cc_major, cc_minor;
} mfp_device_info;
/* Replaces the property query in main.cpp:416-421. */
int mfp_get_device_info(int device, mfp_device_info *out);

/* ------------------------------------------------------------------------- */
/* Host-side format construction, bit-exact with the reference converters.   */
/* All arrays here are HOST arrays sized by the caller.                      */
/* ------------------------------------------------------------------------- */

/* csr_matrix_class<T>(matrix_class) — common/matrix_converter.cpp:15-87.
 * Input: COO triplets with double values (matrix_market::matrix_class).
 * Output: row_ptr[rows+1], columns[nnz], data[nnz]; columns sorted per row.
 * storage_scheme != 0 (non-general) -> MFP_ERROR_NOT_SUPPORTED, as the
 * reference throws at matrix_converter.cpp:19-20. */
int mfp_csr_from_coo_f32(uint32_t rows, uint32_t cols, uint32_t nnz, int storage_scheme,
                         const uint32_t *row_ids, const uint32_t *col_ids, const double *values,
                         uint32_t *row_ptr, uint32_t *columns, float *data);
int mfp_csr_from_coo_f64(uint32_t rows, uint32_t cols, uint32_t nnz, int storage_scheme,
                         const uint32_t *row_ids, const uint32_t *col_ids, const double *values,
                         uint32_t *row_ptr, uint32_t *columns, double *data);

/* matrix_rows_statistic / get_rows_statistics — matrix_converter.h:12-22,
 * matrix_converter.cpp:95-127 (integer average, population std deviation). */
typedef struct mfp_rows_statistic {
  uint32_t min_elements_in_rows;
  uint32_t max_elements_in_rows;
  uint32_t avg_elements_in_rows;
  double elements_in_rows_std_deviation;
} mfp_rows_statistic;
int mfp_get_rows_statistics(uint32_t rows, const uint32_t *row_ptr, mfp_rows_statistic *out);

/* ell_matrix_class<T> — matrix_converter.cpp:129-203.  Column-major
 * [k*rows + row], padding col=0 / value=0.  width = max row length for the
 * plain constructor (mfp_ell_width), or any fixed width (extra elements of a
 * row are dropped, matrix_converter.cpp:194-199).  Outputs sized width*rows. */
int mfp_ell_width(uint32_t rows, const uint32_t *row_ptr, uint32_t *width);
int mfp_ell_from_csr_f32(uint32_t rows, const uint32_t *row_ptr, const uint32_t *columns,
                         const float *data, uint32_t width, float *ell_data, uint32_t *ell_columns);
int mfp_ell_from_csr_f64(uint32_t rows, const uint32_t *row_ptr, const uint32_t *columns,
                         const double *data, uint32_t width, double *ell_data,
                         uint32_t *ell_columns);

/* coo_matrix_class<T> — matrix_converter.cpp:211-280.  element_start = 0 gives
 * every element; element_start = k keeps the elements at in-row position >= k
 * (the hybrid tail).  Row-major, rows ascending, columns ascending per row. */
int mfp_coo_count(uint32_t rows, const uint32_t *row_ptr, uint32_t element_start, uint32_t *count);
int mfp_coo_from_csr_f32(uint32_t rows, const uint32_t *row_ptr, const uint32_t *columns,
                         const float *data, uint32_t element_start, float *coo_data,
                         uint32_t *coo_cols, uint32_t *coo_rows);
int mfp_coo_from_csr_f64(uint32_t rows, const uint32_t *row_ptr, const uint32_t *columns,
                         const double *data, uint32_t element_start, double *coo_data,
                         uint32_t *coo_cols, uint32_t *coo_rows);

/* hybrid_matrix_class<T>::allocate width rule — matrix_converter.cpp:288-310:
 * width = (unsigned)(avg + (max - avg) * percent), avg the integer average. */
int mfp_hybrid_width(uint32_t rows, const uint32_t *row_ptr, double percent, uint32_t *width);
/* Engine extension (no reference counterpart): the q-quantile of the row
 * lengths (q = 2/3 for the power-law configuration's hybrid split). */
int mfp_row_length_quantile(uint32_t rows, const uint32_t *row_ptr, double q, uint32_t *width);

/* scoo_matrix_class<T> — common/scoo_matrix_class.cpp:13-139.
 * Parameters from (rows, sm_count, shared_mem_size, sizeof(T)) exactly as the
 * reference computes them; slices_ptr has slices_count+1 entries and the ones
 * after the last real slice stay 0 (value-initialised in the reference). */
typedef struct mfp_scoo_params {
  uint32_t slices_count;
  uint32_t slice_size;
  uint32_t lane_size;
} mfp_scoo_params;
int mfp_scoo_params_compute(uint32_t rows, uint32_t sm_count, uint64_t shared_mem_size,
                            int value_type, mfp_scoo_params *out);
int mfp_scoo_from_csr_f32(uint32_t rows, const uint32_t *row_ptr, const uint32_t *columns,
                          const float *data, const mfp_scoo_params *params, float *values,
                          uint32_t *c_index, uint32_t *r_index, uint32_t *slices_ptr);
int mfp_scoo_from_csr_f64(uint32_t rows, const uint32_t *row_ptr, const uint32_t *columns,
                          const double *data, const mfp_scoo_params *params, double *values,
                          uint32_t *c_index, uint32_t *r_index, uint32_t *slices_ptr);

/* The reference's disabled sort_cols option of scoo_matrix_class
 * (scoo_matrix_class.cpp:102-138): orders each slice's elements by column, in
 * place, on SCOO arrays built by mfp_scoo_from_csr_*.  The reference sorts with
 * std::sort (not stable: equal columns in unspecified order); this sort is
 * stable, so equal columns keep their CSR order.  Rows are then no longer
 * contiguous within a slice: SpMV goes through mfp_scoo_spmv_unsorted_* (or a
 * handle, which detects the layout). */
int mfp_scoo_sort_cols_f32(uint32_t slices_count, const uint32_t *slices_ptr, float *values,
                           uint32_t *c_index, uint32_t *r_index);
int mfp_scoo_sort_cols_f64(uint32_t slices_count, const uint32_t *slices_ptr, double *values,
                           uint32_t *c_index, uint32_t *r_index);

/* fill_row_blocks — gpu/csr_adaptive_spmv.cu:180-240, with NNZ_PER_WG as a
 * parameter (the reference fixes it at 64).  row_blocks may be NULL to count
 * only; otherwise it receives count+1 boundaries. */
int mfp_csr_adaptive_row_blocks(uint32_t rows, const uint32_t *row_ptr, uint32_t nnz_per_wg,
                                uint32_t *row_blocks, uint32_t *count);

/* ------------------------------------------------------------------------- */
/* On-device format conversion (engine extension of the host converters     */
/* above): the same layouts, identical arrays, built by CUDA kernels from    */
/* DEVICE arrays.  Functions that return a count or a status found on the    */
/* device wait for `stream`; the others only enqueue work on it.             */
/* ------------------------------------------------------------------------- */

/* get_rows_statistics of a device row_ptr (waits).  Bit-identical to
 * mfp_get_rows_statistics: the std deviation comes from an exact integer sum
 * of squared deviations, or from the host loop when that sum reaches 2^53. */
int mfp_dev_rows_statistics(uint32_t rows, const uint32_t *row_ptr, mfp_rows_statistic *out, void *stream);
/* Validates a device CSR (waits): row_ptr[0] = 0, non-decreasing,
 * row_ptr[rows] = nnz, every column < cols. */
int mfp_dev_check_csr(uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *row_ptr,
                      const uint32_t *columns, void *stream);
/* mfp_coo_count on the device (waits). */
int mfp_dev_coo_count(uint32_t rows, const uint32_t *row_ptr, uint32_t element_start, uint32_t *count,
                      void *stream);
/* coo_matrix_class (matrix_converter.cpp:211-280) from a device CSR; outputs
 * sized mfp_dev_coo_count(element_start).  value_type MFP_F32 / MFP_F64.
 * Waits for the output size when element_start > 0 or to read row_ptr[rows]. */
int mfp_dev_coo_from_csr(int value_type, uint32_t rows, const uint32_t *row_ptr, const uint32_t *columns,
                         const void *data, uint32_t element_start, void *coo_data, uint32_t *coo_cols,
                         uint32_t *coo_rows, void *stream);
/* ell_matrix_class (matrix_converter.cpp:139-203) from a device CSR:
 * column-major, padding col 0 / value 0; outputs sized width*rows. */
int mfp_dev_ell_from_csr(int value_type, uint32_t rows, const uint32_t *row_ptr, const uint32_t *columns,
                         const void *data, uint32_t width, void *ell_data, uint32_t *ell_columns,
                         void *stream);
/* scoo_matrix_class (scoo_matrix_class.cpp:58-100) from a device CSR with the
 * parameters of mfp_scoo_params_compute; slices_ptr sized slices_count+1. */
int mfp_dev_scoo_from_csr(int value_type, uint32_t rows, uint32_t nnz, const uint32_t *row_ptr,
                          const uint32_t *columns, const void *data, const mfp_scoo_params *params,
                          void *values, uint32_t *c_index, uint32_t *r_index, uint32_t *slices_ptr,
                          void *stream);
/* mfp_scoo_sort_cols_* on the device (waits): each slice's elements ordered
 * by column, stably, in place; the slice of an element is r_index / slice_size
 * (the layout of mfp_dev_scoo_from_csr). */
int mfp_dev_scoo_sort_cols(int value_type, uint32_t rows, uint32_t cols, uint32_t slice_size, uint32_t nnz,
                           void *values, uint32_t *c_index, uint32_t *r_index, void *stream);
/* mfp_scoo_x_windows on the device: [min col, max col + 1) per slice. */
int mfp_dev_scoo_x_windows(uint32_t nnz, const uint32_t *c_index, const uint32_t *slices_ptr, uint32_t slices,
                           uint32_t *windows, void *stream);
/* csr_matrix_class(matrix_market::matrix_class) (matrix_converter.cpp:15-87)
 * from device COO triplets in any order (waits): row_ptr by histogram and
 * scan, elements ordered by (row, column) with a stable radix sort, so
 * repeated (row, column) entries keep their input order like
 * mfp_csr_from_coo.  Out-of-range ids return MFP_ERROR_INVALID_VALUE. */
int mfp_dev_csr_from_coo(int value_type, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *row_ids,
                         const uint32_t *col_ids, const double *values, uint32_t *row_ptr, uint32_t *columns,
                         void *data, void *stream);
/* The converters' scratch comes from a memory pool of the current device that
 * keeps freed scratch mapped for the next conversion.  scratch_bytes reports
 * what the pool holds; scratch_release waits for the device and returns the
 * unused part to the driver. */
int mfp_dev_scratch_bytes(uint64_t *reserved);
int mfp_dev_scratch_release(void);

/* ------------------------------------------------------------------------- */
/* Device-pointer SpMV entry points: y = A * x, enqueued on `stream`.        */
/* ------------------------------------------------------------------------- */

/* CSR family.  A plan partitions the rows once per sparsity pattern (long-row
 * pieces, CSR-Adaptive row bins) and owns the scratch the pieces combine in.
 * algo: 0 = CSR scalar (one thread per row; csr_spmv_kernel,
 * gpu_matrix_multiplier.cu:22-43), 1 = CSR vector (a lane group per row;
 * csr_spmv_vector_kernel, :331-362), 2 = CSR-Adaptive (row bins;
 * csr_adaptive_spmv.cu:26-178).  Rows longer than long_row_threshold are
 * split across CTAs; rows longer than 4096 accumulate in FP64. */
typedef enum mfp_csr_algo { MFP_CSR_SCALAR = 0, MFP_CSR_VECTOR = 1, MFP_CSR_ADAPTIVE = 2 } mfp_csr_algo;
typedef struct mfp_csr_config {
  uint32_t long_row_threshold; /* 0 = default for the algo; UINT32_MAX = never split */
  uint32_t vector_lanes;       /* CSR vector lanes per row: 2..32 (power of two); 0 = auto:
                                  below a mean row length of 64 the warp-tile kernel (each
                                  warp's lanes take 8 consecutive elements of 256 and combine
                                  rows with a segmented shuffle scan; a fix-up launch adds the
                                  rows that cross tiles), else 4 lanes per row */
  uint32_t bin_nnz;            /* CSR-Adaptive elements per row bin; 0 = default */
  uint32_t piece_nnz;          /* elements per long-row piece; 0 = default (65536) */
  uint32_t assist_threshold;   /* scalar/vector: rows longer than this (and not long) are
                                  reduced by a whole warp; 0 = default (64);
                                  UINT32_MAX = never (keeps the reference summation order) */
  uint32_t kernel;             /* 0 = auto, 1 = row-block kernel (rows per CTA, long rows in
                                  pieces), 2 = streaming kernel (fixed element chunks per
                                  persistent CTA, TMA bulk prefetch), 4 = warp-tile kernel
                                  (256 consecutive elements per warp, rows from row_ptr,
                                  segmented shuffle scan + a fix-up launch) */
} mfp_csr_config;
typedef struct mfp_csr_plan mfp_csr_plan;
int mfp_csr_plan_create(uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *host_row_ptr,
                        int algo, const mfp_csr_config *config, mfp_csr_plan **plan);
int mfp_csr_plan_destroy(mfp_csr_plan *plan);
/* Reads back the resolved configuration (defaults filled in). */
int mfp_csr_plan_get_config(const mfp_csr_plan *plan, int *algo, mfp_csr_config *config,
                            uint32_t *long_rows, uint32_t *pieces);
/* Counterparts of gpu_csr_spmv / gpu_csr_vector_spmv / gpu_csr_adaptive_spmv
 * (gpu_matrix_multiplier.cu:54-133, :364-447; csr_adaptive_spmv.cu:242-321)
 * minus the per-call copies: the arrays are already on the device. */
int mfp_csr_spmv_f32(const mfp_csr_plan *plan, const float *data, const uint32_t *col_ids,
                     const uint32_t *row_ptr, const float *x, float *y, void *stream);
int mfp_csr_spmv_f64(const mfp_csr_plan *plan, const double *data, const uint32_t *col_ids,
                     const uint32_t *row_ptr, const double *x, double *y, void *stream);

/* ELL — counterpart of gpu_ell_spmv (gpu_matrix_multiplier.cu:450-550). */
int mfp_ell_spmv_f32(uint32_t rows, uint32_t cols, uint32_t width, const float *data,
                     const uint32_t *col_ids, const float *x, float *y, void *stream);
int mfp_ell_spmv_f64(uint32_t rows, uint32_t cols, uint32_t width, const double *data,
                     const uint32_t *col_ids, const double *x, double *y, void *stream);

/* COO — counterpart of gpu_coo_spmv (gpu_matrix_multiplier.cu:622-716).
 * Rows must be sorted (the coo_matrix_class layout).  A segmented reduction
 * replaces the per-element atomics, in two launches: each warp reduces 256
 * elements and writes the rows inside them; a fix-up pass adds up the rows
 * that cross those tiles, from partial sums kept in `workspace` (device memory
 * of mfp_coo_workspace_bytes bytes; no initialisation needed).  Results are
 * deterministic.  Calls that share a workspace must not overlap on the GPU.
 * Row ids must be below `rows`; elements with a larger row id are dropped
 * (never written).  Empty rows get 0. */
int mfp_coo_workspace_bytes(uint32_t rows, uint32_t nnz, size_t *bytes);
int mfp_coo_spmv_f32(uint32_t rows, uint32_t cols, uint32_t nnz, const float *data,
                     const uint32_t *col_ids, const uint32_t *row_ids, const float *x, float *y,
                     void *workspace, size_t workspace_bytes, void *stream);
int mfp_coo_spmv_f64(uint32_t rows, uint32_t cols, uint32_t nnz, const double *data,
                     const uint32_t *col_ids, const uint32_t *row_ids, const double *x, double *y,
                     void *workspace, size_t workspace_bytes, void *stream);
/* Reads a COO workspace's error word.  The two-pass COO never waits and
 * leaves it 0; it stays for callers written against a waiting COO.
 * Synchronous. */
int mfp_workspace_error(const void *workspace, uint32_t *error);

/* Load-ceiling probe (a measurement kernel; no counterpart in the reference).
 * Issues an SpMV's memory operations over nnz (value, column) pairs without
 * the rows: mode 0 streams values and column ids, mode 1 streams column ids
 * and gathers x[col], mode 2 does both (every format's loads), mode 3 is
 * mode 1 with every gather folded into x[0, 4096) (held in L1; x needs at
 * least 4096 entries).  x_path: 0 the
 * L1-cached read-only path, 1 L2 only (ld.global.cg), 2 read-only without L1
 * allocation.  One partial sum per CTA goes to `out` (at least 148 * 8 =
 * 1184 floats on a B200; fewer -> MFP_ERROR_INVALID_VALUE).  Arrays must be
 * 16-byte aligned (32-byte aligned arrays read each thread's sector with one
 * load, as the formats' kernels do).  Its time on a matrix bounds every
 * format's kernel time on that matrix from below. */
int mfp_probe_spmv_loads(int mode, int x_path, uint32_t nnz, const float *values, const uint32_t *col_ids,
                         const float *x, float *out, size_t out_len, void *stream);
/* The same probe with the x gathers done by TMA (cp.async.bulk.tensor
 * tile::gather4: four 16-byte rows of x per instruction into shared memory),
 * mode 4 all of them, mode 5 half (the other half by ld.global.nc).  x has
 * n_x entries (n_x % 4 == 0, 16-byte aligned); the last nnz % 256 elements
 * are not visited.  A CTA whose bounded wait gave up writes NaN to out. */
int mfp_probe_spmv_gather4(int mode, uint32_t nnz, uint32_t n_x, const uint32_t *col_ids, const float *x, float *out,
                           size_t out_len, void *stream);

/* COO SpMV (float) that allocates nothing.  No counterpart in the reference:
 * it serves callers that may not allocate device memory themselves (hosts
 * that own every byte through their own pool or budget, or loops that cannot
 * take cudaMalloc's latency and implicit synchronisation).  Same arguments and
 * the same result bits as mfp_coo_spmv_f32 without the workspace: it runs the
 * same two-pass COO, whose workspace lives in a fixed 4 MiB array inside the
 * library, present on every device that loads it, so nnz is limited to
 * 44,739,072 (larger -> MFP_ERROR_TOO_LARGE, before any GPU work).
 * The passes have no waits, so nothing can fail on the GPU after a successful
 * launch; the array needs no clearing (every call rewrites what it reads).
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the one array, so calls that overlap on the GPU (different
 * streams, or different host threads) race and must not be issued
 * concurrently. */
int mfp_coo_spmv_f32_noalloc(uint32_t rows, uint32_t cols, uint32_t nnz, const float *data,
                             const uint32_t *col_ids, const uint32_t *row_ids, const float *x, float *y,
                             void *stream);

/* SCOO — counterpart of gpu_scoo_spmv (gpu/scoo_spmv.cu:46-222).  One CTA per
 * slice.  x_windows (device, 2 uint32 per slice: first and one-past-last
 * column of the slice, from mfp_scoo_x_windows) lets a slice stage its x
 * window in shared memory when the window holds at most max_window elements;
 * wider slices, or x_windows == NULL, gather x from global memory. */
int mfp_scoo_x_windows(uint32_t nnz, const uint32_t *c_index, const uint32_t *slices_ptr,
                       uint32_t slices_count, uint32_t *windows);
/* slice_order (device, slices_count entries, may be NULL = natural order):
 * the order the CTAs take the slices in; mfp_scoo_slice_order gives the
 * slices by element count, heaviest first (host), which shortens the tail of
 * matrices with a few heavy slices. */
int mfp_scoo_slice_order(uint32_t slices_count, const uint32_t *slices_ptr, uint32_t *slice_order);
int mfp_scoo_spmv_f32(uint32_t rows, uint32_t cols, uint32_t slices_count, uint32_t slice_size,
                      const float *values, const uint32_t *c_index, const uint32_t *r_index,
                      const uint32_t *slices_ptr, const uint32_t *x_windows, uint32_t max_window,
                      const uint32_t *slice_order, const float *x, float *y, void *stream);
int mfp_scoo_spmv_f64(uint32_t rows, uint32_t cols, uint32_t slices_count, uint32_t slice_size,
                      const double *values, const uint32_t *c_index, const uint32_t *r_index,
                      const uint32_t *slices_ptr, const uint32_t *x_windows, uint32_t max_window,
                      const uint32_t *slice_order, const double *x, double *y, void *stream);
/* SCOO whose slices are in column order (mfp_scoo_sort_cols_*, the reference's
 * sort_cols layout): rows within a slice in any order; products are added
 * into shared-memory row accumulators with atomics, as in the reference
 * kernel, so the summation order within a row is not fixed.  Same arguments. */
int mfp_scoo_spmv_unsorted_f32(uint32_t rows, uint32_t cols, uint32_t slices_count, uint32_t slice_size,
                               const float *values, const uint32_t *c_index, const uint32_t *r_index,
                               const uint32_t *slices_ptr, const uint32_t *x_windows, uint32_t max_window,
                               const uint32_t *slice_order, const float *x, float *y, void *stream);
int mfp_scoo_spmv_unsorted_f64(uint32_t rows, uint32_t cols, uint32_t slices_count, uint32_t slice_size,
                               const double *values, const uint32_t *c_index, const uint32_t *r_index,
                               const uint32_t *slices_ptr, const uint32_t *x_windows, uint32_t max_window,
                               const uint32_t *slice_order, const double *x, double *y, void *stream);

/* Hybrid ELL + COO — counterpart of gpu_hybrid_spmv / gpu_hybrid_atomic_spmv
 * (gpu_matrix_multiplier.cu:866-1096).  The ELL kernel writes every row's ELL
 * part, then the two-pass COO adds the tail (the elements past the ELL width,
 * hybrid_matrix_class's coo_matrix) row by row, without atomics: three
 * launches.  `workspace` holds the tail's warp-tile partial sums
 * (mfp_hybrid_workspace_bytes; no initialisation needed). */
int mfp_hybrid_workspace_bytes(uint32_t rows, uint32_t coo_nnz, size_t *bytes);
int mfp_hybrid_spmv_f32(uint32_t rows, uint32_t cols, uint32_t ell_width, const float *ell_data,
                        const uint32_t *ell_cols, uint32_t coo_nnz, const float *coo_data,
                        const uint32_t *coo_cols, const uint32_t *coo_rows, const float *x, float *y,
                        void *workspace, size_t workspace_bytes, void *stream);
int mfp_hybrid_spmv_f64(uint32_t rows, uint32_t cols, uint32_t ell_width, const double *ell_data,
                        const uint32_t *ell_cols, uint32_t coo_nnz, const double *coo_data,
                        const uint32_t *coo_cols, const uint32_t *coo_rows, const double *x, double *y,
                        void *workspace, size_t workspace_bytes, void *stream);

/* ---- Reduced-precision CSR (engine extension; the reference has float and
 * double CSR only, gpu_matrix_multiplier.cu:54-129) -------------------------
 * Layout: row_ptr[rows + 1] uint32 as CSR; q[nnz] uint16 bit patterns of
 * round(a_ij / scale_i) in BF16 or FP16; scale[rows] float, scale_i =
 * max_j |a_ij| (1 for an empty or all-zero row); columns[nnz] uint32, or
 * delta[nnz] uint16 with column = base[e / MFP_LOWP_DELTA_CHUNK] + delta[e].
 * y_i = scale_i * sum_j float(q_ij) * x_j with FP32 accumulation. */
#define MFP_LOWP_DELTA_CHUNK 2048u

/* Host quantizer: q and scale from FP64 values (a_ij / scale_i rounded to
 * FP32, then to BF16 or FP16 with round-to-nearest-even). */
int mfp_lowp_quantize(int value_type, uint32_t rows, const uint32_t *row_ptr, const double *values,
                      uint16_t *q, float *scale);
/* Host delta encoder: base[k] = smallest column of chunk k, delta = column -
 * base; MFP_ERROR_NOT_SUPPORTED if a chunk's span exceeds 65535. */
int mfp_lowp_deltas(uint32_t nnz, const uint32_t *columns, uint16_t *delta, uint32_t *base);
/* y = A*x for that layout (device arrays); columns (uint32) or delta + base
 * (16-bit) is given, the other null.  With q, the indices and row_ptr
 * 16-byte aligned the launch is the pipelined kernel (TMA bulk copies into
 * shared-memory stages); otherwise a row-block kernel with plain loads.  Both
 * are within FP32 rounding of each other (their sum orders differ).  The
 * pipelined kernel sums each row in one thread: for matrices with rows longer
 * than 1,024 elements use a handle (mfp_matrix_create_lowp), which sends them
 * to the row-block kernel, where a warp shares each row longer than 128. */
int mfp_lowp_spmv(int value_type, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *row_ptr,
                  const uint16_t *q, const float *scale, const uint32_t *columns, const uint16_t *delta,
                  const uint32_t *base, const float *x, float *y, void *stream);
/* Reduced-precision ELL (engine extension): column-major slots
 * [k * rows + row] as gpu_ell_spmv's layout (matrix_converter.cpp:139-174),
 * 16-bit values q (per-row scale as above), and uint32 column ids or, with
 * index16, 16-bit offsets from the row: column = row + off - 32768
 * (MFP_ERROR_NOT_SUPPORTED when some |column - row| > 32767).  Padding slots
 * hold q = 0 and the row's last column.  width >= every row length.  Host
 * builder: q and idx hold width * rows entries (idx uint16 with index16, else
 * uint32), scale rows. */
int mfp_lowp_ell_from_csr(int value_type, int index16, uint32_t rows, uint32_t cols, const uint32_t *row_ptr,
                          const uint32_t *columns, const double *values, uint32_t width, uint16_t *q, void *idx,
                          float *scale);
/* y = A*x (device arrays; offsets or columns given, the other NULL). */
int mfp_lowp_ell_spmv(int value_type, uint32_t rows, uint32_t cols, uint32_t width, const uint16_t *q,
                      const float *scale, const uint32_t *columns, const uint16_t *offsets, const float *x, float *y,
                      void *stream);
/* Error word of the pipelined reduced-precision kernel on `device` (bit 0: a
 * stage wait gave up, the results of that launch are incomplete); `clear`
 * resets it.  Synchronous.  Engine extension, no counterpart in the reference. */
int mfp_lowp_error(int device, int clear, uint32_t *error);

/* ---- Batched SpMV (engine extension, no counterpart in the reference) ------
 * Many CSR matrices of uneven sizes as one block-diagonal CSR: matrix k's rows
 * follow matrix k-1's, its column ids are shifted into its own slice of one
 * concatenated x, and its y is a slice of one concatenated y
 * (mfp_batch_offsets).  One launch covers every matrix.  The plan (algorithm,
 * lanes, thresholds, kernel) is the default CSR scalar plan until
 * mfp_batch_set_config or mfp_batch_autotune picks another;
 * mfp_batch_graph_launch captures the launch into a CUDA graph once per
 * (x, y) pair and replays it. */
typedef struct mfp_batch mfp_batch;
typedef struct mfp_batch_config {
  int algo;              /* 0 CSR scalar, 1 CSR vector, 2 CSR-Adaptive */
  mfp_csr_config csr;    /* lanes, thresholds, kernel (0 fields = defaults) */
} mfp_batch_config;
typedef struct mfp_batch_info {
  uint32_t matrices, rows, cols, nnz; /* totals of the concatenation */
  uint64_t algorithmic_bytes;         /* sum over the matrices of nnz*(v+4)+(rows+1)*4+cols*v+rows*v */
  uint64_t device_bytes;
  mfp_batch_config config;            /* the plan in use */
  uint32_t kernel_launches;           /* launches per mfp_batch_spmv */
} mfp_batch_info;
/* Host CSR arrays per matrix: rows[k], cols[k], row_ptr[k] (rows[k]+1
 * entries, nnz = row_ptr[k][rows[k]]), columns[k], values[k] (float or
 * double).  Totals must fit 32-bit indices. */
int mfp_batch_create(int value_type, uint32_t matrices, const uint32_t *rows, const uint32_t *cols,
                     const uint32_t *const *row_ptr, const uint32_t *const *columns,
                     const void *const *values, mfp_batch **out);
int mfp_batch_destroy(mfp_batch *batch);
/* x_offsets / y_offsets receive matrices+1 entries (element offsets). */
int mfp_batch_offsets(const mfp_batch *batch, uint64_t *x_offsets, uint64_t *y_offsets);
int mfp_batch_get_info(const mfp_batch *batch, mfp_batch_info *out);
int mfp_batch_set_config(mfp_batch *batch, const mfp_batch_config *config);
/* Times every candidate plan (reps launches each, median of CUDA-event times
 * on `stream`) on the given x, y and keeps the fastest; *chosen and
 * *best_seconds (either may be NULL) receive it.  Synchronous. */
int mfp_batch_autotune(mfp_batch *batch, const void *x, void *y, uint32_t reps, void *stream,
                       mfp_batch_config *chosen, double *best_seconds);
int mfp_batch_spmv(const mfp_batch *batch, const void *x, void *y, void *stream);
/* Replays a CUDA graph of mfp_batch_spmv(x, y); the first call for an (x, y)
 * pair captures it (on an internal stream), so make that call outside any
 * stream capture of the caller's. */
int mfp_batch_graph_launch(mfp_batch *batch, const void *x, void *y, void *stream);

/* ---- Format selector (engine extension, no counterpart in the reference) --
 * Features of a CSR pattern (host):
 *   0 log10(rows)          1 log10(cols)            2 log10(nnz + 1)
 *   3 log2(1 + mean len)   4 log2(1 + std of len)   5 log2(1 + max len)
 *   6 Gini of row lengths  7 max |i - j| / max(rows, cols)   (bandwidth)
 *   8 share of nonzeros with |i - j| <= 64           9 diagonal nonzeros / min(rows, cols)
 *  10 share of empty rows  11 share of nonzeros in rows longer than 4096 */
#define MFP_SELECTOR_FEATURES 12u
int mfp_selector_features(uint32_t rows, uint32_t cols, const uint32_t *row_ptr, const uint32_t *columns,
                          float *features);

/* The selector's MLP 12 -> 64 -> 64 -> 28 (ReLU hidden layers), FP32, device
 * arrays, enqueued on `stream`.  params: W1[12][64] b1[64] W2[64][64] b2[64]
 * W3[64][28] b3[28] (mfp_mlp_param_count() floats).  All sums run in a fixed
 * order, so results are reproducible. */
#define MFP_MLP_IN 12u
#define MFP_MLP_HIDDEN 64u
#define MFP_MLP_OUT 28u
uint32_t mfp_mlp_param_count(void);
/* h1[batch][64], h2[batch][64], y[batch][28]. */
int mfp_mlp_forward(const float *params, const float *x, uint32_t batch, float *h1, float *h2, float *y,
                    void *stream);
/* Masked mean-squared error of y against target (mask 0/1, [batch][28]):
 * *loss (device) = sum mask (y - target)^2 / sum mask; grads (param count
 * floats) its gradient; work holds batch * (28 + 64 + 64) floats. */
int mfp_mlp_backward(const float *params, const float *x, const float *h1, const float *h2, const float *y,
                     const float *target, const float *mask, uint32_t batch, float *grads, float *loss,
                     float *work, void *stream);
/* One Adam step (bias-corrected; step counts from 1). */
int mfp_mlp_adam(float *params, const float *grads, float *m, float *v, uint32_t n, float lr, float beta1,
                 float beta2, float eps, uint32_t step, void *stream);

/* fill_vector — gpu_matrix_multiplier.cu:45-52. */
int mfp_fill_f32(uint64_t n, float *vec, float value, void *stream);
int mfp_fill_f64(uint64_t n, double *vec, double value, void *stream);

/* ------------------------------------------------------------------------- */
/* Device-resident matrices (the reference-facing call with host x and y).   */
/* ------------------------------------------------------------------------- */

/* A handle uploads one format once and keeps it on the device with whatever
 * plan / workspace / staging the format needs.  It replaces the caller-held
 * resizable_gpu_memory buffers of the reference (gpu/resizable_gpu_memory.h:13-44)
 * and the per-call H2D copies of every gpu_*_spmv wrapper. */
typedef enum mfp_format {
  MFP_FORMAT_CSR_SCALAR = 0,
  MFP_FORMAT_CSR_VECTOR = 1,
  MFP_FORMAT_CSR_ADAPTIVE = 2,
  MFP_FORMAT_ELL = 3,
  MFP_FORMAT_COO = 4,
  MFP_FORMAT_SCOO = 5,
  MFP_FORMAT_HYBRID = 6,
  MFP_FORMAT_CSR_LOWP = 7, /* reduced-precision CSR (engine extension) */
  MFP_FORMAT_ELL_LOWP = 8  /* reduced-precision ELL (engine extension) */
} mfp_format;
typedef struct mfp_matrix mfp_matrix;

/* CSR algorithms (format 0..2) from host CSR arrays. */
int mfp_matrix_create_csr(int format, int value_type, uint32_t rows, uint32_t cols, uint32_t nnz,
                          const uint32_t *row_ptr, const uint32_t *columns, const void *data,
                          const mfp_csr_config *config, mfp_matrix **out);
int mfp_matrix_create_ell(int value_type, uint32_t rows, uint32_t cols, uint32_t width,
                          const uint32_t *ell_columns, const void *ell_data, mfp_matrix **out);
/* COO (and the hybrid's tail, below): the handle also keeps each row id as a
 * 1-byte offset from the first row of its 256-element tile (a tile spanning
 * more than 256 rows reads the 32-bit ids; allowed for at most one tile in 8,
 * FP32 only), else as a 2-byte offset when every tile spans at most 65,536
 * rows, else only the 32-bit ids.  The SpMV reads the offsets; the result
 * bits do not depend on the choice (mfp_matrix_info.format_bytes counts it).
 * Row-ordered SCOO keeps 2-byte offsets from each slice's first row. */
int mfp_matrix_create_coo(int value_type, uint32_t rows, uint32_t cols, uint32_t nnz,
                          const uint32_t *coo_rows, const uint32_t *coo_cols,
                          const void *coo_data, mfp_matrix **out);
/* SCOO: rows within each slice may be in CSR order (the reference layout) or
 * in any order (the sort_cols layout, detected here: SpMV then uses the
 * shared-memory-atomics kernel). */
int mfp_matrix_create_scoo(int value_type, uint32_t rows, uint32_t cols, uint32_t nnz,
                           const mfp_scoo_params *params, const uint32_t *c_index,
                           const uint32_t *r_index, const uint32_t *slices_ptr,
                           const void *values, mfp_matrix **out);
int mfp_matrix_create_hybrid(int value_type, uint32_t rows, uint32_t cols, uint32_t ell_width,
                             const uint32_t *ell_columns, const void *ell_data, uint32_t coo_nnz,
                             const uint32_t *coo_rows, const uint32_t *coo_cols,
                             const void *coo_data, mfp_matrix **out);
/* Reduced-precision CSR from host CSR with FP64 values: quantized on the host
 * (mfp_lowp_quantize), 16-bit column deltas when index16 != 0 and every
 * 2048-element chunk's column span fits 16 bits (else MFP_ERROR_NOT_SUPPORTED). */
int mfp_matrix_create_lowp(int value_type, int index16, uint32_t rows, uint32_t cols, uint32_t nnz,
                           const uint32_t *row_ptr, const uint32_t *columns, const double *values,
                           mfp_matrix **out);
/* Reduced-precision ELL from host CSR with FP64 values (width = longest row). */
int mfp_matrix_create_lowp_ell(int value_type, int index16, uint32_t rows, uint32_t cols, uint32_t nnz,
                               const uint32_t *row_ptr, const uint32_t *columns, const double *values,
                               mfp_matrix **out);
/* Any of formats 0..6 from a DEVICE CSR (row_ptr, columns, data on the
 * current device), converted on the GPU with the mfp_dev_* functions; the
 * caller keeps its arrays.  options may be NULL: CSR defaults, ELL width =
 * longest row, SCOO parameters for the current device. */
#define MFP_ELL_WIDTH_LONGEST 0xFFFFFFFFu
typedef struct mfp_device_build_options {
  const mfp_csr_config *csr;   /* CSR family launch configuration (NULL = defaults) */
  uint32_t ell_width;          /* ELL / hybrid ELL part: slots per row, or MFP_ELL_WIDTH_LONGEST */
  const mfp_scoo_params *scoo; /* SCOO parameters (NULL = mfp_scoo_params_compute for this device) */
  uint32_t scoo_sort_cols;     /* SCOO: non-zero = each slice in column order (mfp_dev_scoo_sort_cols) */
} mfp_device_build_options;
int mfp_matrix_create_device(int format, int value_type, uint32_t rows, uint32_t cols, uint32_t nnz,
                             const uint32_t *row_ptr, const uint32_t *columns, const void *data,
                             const mfp_device_build_options *options, mfp_matrix **out);
int mfp_matrix_destroy(mfp_matrix *m);

typedef struct mfp_matrix_info {
  int format;
  int value_type;
  uint32_t rows, cols;
  uint64_t nnz;                /* stored non-zeros of the source matrix */
  uint64_t format_bytes;       /* bytes one SpMV must move in this layout */
  uint64_t algorithmic_bytes;  /* nnz*(val+4) + (rows+1)*4 + cols*val + rows*val */
  uint64_t device_bytes;       /* device memory held by the handle */
  uint32_t kernel_launches;    /* kernels one mfp_matrix_spmv enqueues */
} mfp_matrix_info;
int mfp_matrix_get_info(const mfp_matrix *m, mfp_matrix_info *out);

/* y = A*x with device x and y (value type of the matrix), enqueued on stream. */
int mfp_matrix_spmv(const mfp_matrix *m, const void *x, void *y, void *stream);
/* y = A*x with HOST x and y: copies x in, runs the kernel, copies y out, and
 * waits for the copy.  Page-locked host buffers give full PCIe bandwidth.
 * When host_y is page-locked and device-addressable and the format's kernel
 * stores each row of y once in row order (CSR scalar / adaptive, CSR vector
 * with lanes per row, ELL, SCOO, the reduced-precision layouts), the kernel
 * stores y straight into host_y, so the copy-out overlaps the kernel.
 * The host-buffer calls stage through buffers owned by the handle: one such
 * call at a time per handle. */
int mfp_matrix_spmv_host(mfp_matrix *m, const void *host_x, void *host_y, void *stream);
/* count independent products host_y[i] = A*host_x[i] with HOST vectors,
 * pipelined: x_{i+1} is copied in while SpMV i runs and y_{i-1} is copied
 * out (two device staging pairs, two copy streams of the handle, made on
 * the first call).  The kernels run in order on `stream`; the call returns
 * when every y is in host memory.  Page-locked host vectors give the copies
 * full PCIe bandwidth and let them overlap.  Engine extension: the serving
 * form of mfp_matrix_spmv_host. */
int mfp_matrix_spmv_host_batch(mfp_matrix *m, uint32_t count, const void *const *host_x, void *const *host_y,
                               void *stream);

/* ------------------------------------------------------------------------- */
/* Measurement records — measurement_class (common/measurement_class.h:11-58) */
/* and compare_results (:60-89).                                              */
/* ------------------------------------------------------------------------- */
typedef struct mfp_measurement {
  char format[64];
  double elapsed;                  /* seconds */
  double effective_bandwidth;      /* load_store_bytes / (elapsed * 1e9) */
  double computational_throughput; /* operations_count / (elapsed * 1e9) */
} mfp_measurement;
int mfp_measurement_make(const char *format, double elapsed, double load_store_bytes,
                         double operations_count, mfp_measurement *out);
/* Relative squared L2 error sum((a-b)^2) / sum(b^2), accumulated in T as the
 * reference does.  *first_bad = first i with |a-b| > 1e-8 when error > 1e-9,
 * else UINT32_MAX.  Does not print. */
int mfp_compare_results_f32(uint32_t n, const float *a, const float *b, double *error,
                            uint32_t *first_bad);
int mfp_compare_results_f64(uint32_t n, const double *a, const double *b, double *error,
                            uint32_t *first_bad);

/* Times `reps` launches of mfp_matrix_spmv with CUDA events on `stream`,
 * writing over an L2-sized buffer between launches when flush_l2 != 0.
 * Returns the mean seconds per launch and the median. */
int mfp_matrix_time(const mfp_matrix *m, const void *x, void *y, uint32_t reps, int flush_l2,
                    void *stream, double *mean_seconds, double *median_seconds);

/* ------------------------------------------------------------------------- */
/* Seeded synthetic matrices (stand-ins for the SuiteSparse inputs).          */
/* Output is CSR with sorted columns and double values; call with NULL       */
/* arrays first to get rows and nnz.                                          */
/* ------------------------------------------------------------------------- */
typedef enum mfp_synth_kind {
  MFP_SYNTH_LAPLACIAN_2D = 0, /* n x n grid, 5-point, 4 / -1 */
  MFP_SYNTH_POWER_LAW = 1,    /* Zipf(alpha) row lengths clipped to [1, max_row] */
  MFP_SYNTH_STENCIL_27 = 2,   /* n^3 grid, 27-point, values U[-1,1] */
  MFP_SYNTH_BANDED = 3,       /* n rows, half bandwidth b, k distinct columns per row */
  MFP_SYNTH_UNIFORM = 4,      /* k_lo..k_hi uniform row lengths, uniform columns */
  MFP_SYNTH_TRIDIAGONAL = 5,
  MFP_SYNTH_BLOCK_DIAGONAL = 6 /* dense b x b blocks on the diagonal */
} mfp_synth_kind;
typedef struct mfp_synth_params {
  int kind;
  uint64_t seed;
  uint32_t n;       /* grid side (laplacian, stencil) or rows (others) */
  uint32_t cols;    /* columns (power law, uniform); 0 = n */
  double alpha;     /* Zipf exponent */
  uint32_t k_lo, k_hi; /* row length bounds (power-law clip [k_lo, k_hi]; uniform) */
  uint32_t band;    /* half bandwidth (banded) or block size (block diagonal) */
} mfp_synth_params;
int mfp_synth_csr(const mfp_synth_params *p, uint32_t *rows, uint32_t *cols, uint64_t *nnz,
                  uint32_t *row_ptr, uint32_t *columns, double *values);
/* Seeded uniform[lo, hi) vectors (x of every configuration). */
int mfp_synth_vector_f64(uint64_t seed, uint64_t n, double lo, double hi, double *out);

#ifdef __cplusplus
}
#endif

#endif /* MFP_SPMV_H */
