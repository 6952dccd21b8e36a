// The reference's GPU operators (gpu/gpu_matrix_multiplier.h:15-152,
// gpu/csr_adaptive_spmv.h:13-23, gpu/scoo_spmv.h:12-23) with the same names,
// arguments and behaviour, running the engine's sm_100a kernels through the
// C ABI:
//   * the matrix arrays are copied into the caller's resizable_gpu_memory
//     buffers (reused across calls), x := 1 on the device, y in `y`;
//   * one launch on the default stream is timed with CUDA events;
//   * y is copied into `reusable_vector` and compared with `reference_y`
//     (compare_results: an error above 1e-9 is reported on stderr);
//   * the result is a measurement_class with the reference's label.
// Temporaries the reference allocates per call (CSR-Adaptive row blocks, SCOO
// slices_ptr) are per call here too: the CSR plan, the COO workspace (the
// warp tiles' partial sums), the SCOO slice pointers and x windows.  A failing CUDA or engine
// call throws std::runtime_error (the reference ignored CUDA status codes).
// Bytes in measurement_class: the reference's per-format counts where it has
// them (CSR, CSR vector, ELL, COO); where it reports 0 (CSR-Adaptive, SCOO,
// hybrid) the algorithmic model nnz*(sizeof(T)+4) + (rows+1)*4 + cols*sizeof(T)
// + rows*sizeof(T); model_bandwidth() is the algorithmic model for all.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "matrix_converter.h"
#include "measurement_class.h"
#include "resizable_gpu_memory.h"
#include "scoo_matrix_class.h"

namespace mfp_host {

inline void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
void upload(resizable_gpu_memory<T> &buf, const T *host, size_t n) {
  buf.resize(std::max<size_t>(n, 1));
  if (n) cuda_check(cudaMemcpy(buf.get(), host, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
}

inline int fill(size_t n, float *v, double value) { return mfp_fill_f32(n, v, (float)value, nullptr); }
inline int fill(size_t n, double *v, double value) { return mfp_fill_f64(n, v, value, nullptr); }

// x := 1, y sized; times launch() between two events on the default stream.
template <typename T, typename Launch>
measurement_class timed_spmv(const char *label, const matrix_market::matrix_class::matrix_meta &meta,
                             resizable_gpu_memory<T> &x, resizable_gpu_memory<T> &y, T *reusable_vector,
                             const T *reference_y, bool compare, double bytes, double ops, Launch launch) {
  x.resize(std::max<size_t>(meta.cols_count, 1));
  y.resize(std::max<size_t>(meta.rows_count, 1));
  check(fill(meta.cols_count, x.get(), 1.0), "fill_vector");
  cudaEvent_t start, stop;
  cuda_check(cudaEventCreate(&start), "cudaEventCreate");
  cuda_check(cudaEventCreate(&stop), "cudaEventCreate");
  cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  cudaEventRecord(start);
  const int st = launch();
  cudaEventRecord(stop);
  const cudaError_t e = cudaEventSynchronize(stop);
  float ms = 0;
  cudaEventElapsedTime(&ms, start, stop);
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  check(st, label);
  cuda_check(e, label);
  if (meta.rows_count)
    cuda_check(cudaMemcpy(reusable_vector, y.get(), meta.rows_count * sizeof(T), cudaMemcpyDeviceToHost),
               "cudaMemcpy D2H");
  double err = 0.0;
  if (compare && meta.rows_count) err = compare_results(meta.rows_count, reusable_vector, reference_y);
  measurement_class m(label, ms / 1000.0, bytes, ops, model_bytes<T>(meta));
  m.error = err;
  return m;
}

inline int csr_spmv(const mfp_csr_plan *p, const float *a, const uint32_t *c, const uint32_t *rp, const float *x,
                    float *y) {
  return mfp_csr_spmv_f32(p, a, c, rp, x, y, nullptr);
}
inline int csr_spmv(const mfp_csr_plan *p, const double *a, const uint32_t *c, const uint32_t *rp,
                    const double *x, double *y) {
  return mfp_csr_spmv_f64(p, a, c, rp, x, y, nullptr);
}

template <typename T>
measurement_class csr_family(int algo, const char *label, bool reference_bytes, const csr_matrix_class<T> &matrix,
                             resizable_gpu_memory<T> &A, resizable_gpu_memory<unsigned int> &col_ids,
                             resizable_gpu_memory<unsigned int> &row_ptr, resizable_gpu_memory<T> &x,
                             resizable_gpu_memory<T> &y, T *reusable_vector, const T *reference_y) {
  const auto &meta = matrix.meta;
  const size_t nnz = meta.non_zero_count;
  upload(A, matrix.data.get(), nnz);
  upload(col_ids, matrix.columns.get(), nnz);
  upload(row_ptr, matrix.row_ptr.get(), (size_t)meta.rows_count + 1);
  mfp_csr_plan *plan = nullptr;
  check(mfp_csr_plan_create(meta.rows_count, meta.cols_count, meta.non_zero_count, matrix.row_ptr.get(), algo,
                            nullptr, &plan),
        label);
  const double bytes = reference_bytes ? (double)nnz * (2 * sizeof(T) + 4) + 2.0 * meta.rows_count * 4 +
                                             (double)meta.rows_count * sizeof(T)
                                       : model_bytes<T>(meta);
  try {
    auto m = timed_spmv<T>(label, meta, x, y, reusable_vector, reference_y, true, bytes, 2.0 * nnz,
                           [&] { return csr_spmv(plan, A.get(), col_ids.get(), row_ptr.get(), x.get(), y.get()); });
    mfp_csr_plan_destroy(plan);
    return m;
  } catch (...) {
    mfp_csr_plan_destroy(plan);
    throw;
  }
}

// device temporary freed on scope exit
struct dev_temp {
  void *p = nullptr;
  explicit dev_temp(size_t bytes) {
    if (bytes) cuda_check(cudaMalloc(&p, bytes), "cudaMalloc");
  }
  ~dev_temp() {
    if (p) cudaFree(p);
  }
  template <typename U>
  U *as() const { return static_cast<U *>(p); }
};

}  // namespace mfp_host

/// y = A*x, one thread per row (csr_spmv_kernel's role): "GPU CSR".
template <typename data_type>
measurement_class gpu_csr_spmv(const csr_matrix_class<data_type> &matrix, resizable_gpu_memory<data_type> &A,
                               resizable_gpu_memory<unsigned int> &col_ids,
                               resizable_gpu_memory<unsigned int> &row_ptr, resizable_gpu_memory<data_type> &x,
                               resizable_gpu_memory<data_type> &y, data_type *reusable_vector,
                               const data_type *reference_y) {
  return mfp_host::csr_family(MFP_CSR_SCALAR, "GPU CSR", true, matrix, A, col_ids, row_ptr, x, y, reusable_vector,
                              reference_y);
}

/// A lane group per row (csr_spmv_vector_kernel's role): "GPU CSR (vector)".
template <typename data_type>
measurement_class gpu_csr_vector_spmv(const csr_matrix_class<data_type> &matrix, resizable_gpu_memory<data_type> &A,
                                      resizable_gpu_memory<unsigned int> &col_ids,
                                      resizable_gpu_memory<unsigned int> &row_ptr,
                                      resizable_gpu_memory<data_type> &x, resizable_gpu_memory<data_type> &y,
                                      data_type *reusable_vector, const data_type *reference_y) {
  return mfp_host::csr_family(MFP_CSR_VECTOR, "GPU CSR (vector)", true, matrix, A, col_ids, row_ptr, x, y,
                              reusable_vector, reference_y);
}

/// Row bins (csr_adaptive_spmv_kernel's role): "GPU CSR-Adaptive".
template <typename data_type>
measurement_class gpu_csr_adaptive_spmv(const csr_matrix_class<data_type> &matrix,
                                        resizable_gpu_memory<data_type> &A,
                                        resizable_gpu_memory<unsigned int> &col_ids,
                                        resizable_gpu_memory<unsigned int> &row_ptr,
                                        resizable_gpu_memory<data_type> &x, resizable_gpu_memory<data_type> &y,
                                        data_type *reusable_vector, const data_type *reference_y) {
  return mfp_host::csr_family(MFP_CSR_ADAPTIVE, "GPU CSR-Adaptive", false, matrix, A, col_ids, row_ptr, x, y,
                              reusable_vector, reference_y);
}

/// Column-major ELL: "GPU ELL".
template <typename data_type>
measurement_class gpu_ell_spmv(const ell_matrix_class<data_type> &matrix, resizable_gpu_memory<data_type> &A,
                               resizable_gpu_memory<unsigned int> &col_ids, resizable_gpu_memory<data_type> &x,
                               resizable_gpu_memory<data_type> &y, data_type *reusable_vector,
                               const data_type *reference_y) {
  const auto &meta = matrix.meta;
  const size_t n = matrix.get_matrix_size();
  mfp_host::upload(A, matrix.data.get(), n);
  mfp_host::upload(col_ids, matrix.columns.get(), n);
  const double bytes = (double)n * (2 * sizeof(data_type) + 4) + (double)meta.rows_count * sizeof(data_type);
  return mfp_host::timed_spmv<data_type>(
      "GPU ELL", meta, x, y, reusable_vector, reference_y, true, bytes, 2.0 * n, [&] {
        return sizeof(data_type) == 4
                   ? mfp_ell_spmv_f32(meta.rows_count, meta.cols_count, matrix.elements_in_rows,
                                      (const float *)A.get(), col_ids.get(), (const float *)x.get(),
                                      (float *)y.get(), nullptr)
                   : mfp_ell_spmv_f64(meta.rows_count, meta.cols_count, matrix.elements_in_rows,
                                      (const double *)A.get(), col_ids.get(), (const double *)x.get(),
                                      (double *)y.get(), nullptr);
      });
}

/// Row-major COO, tile-based segmented reduction (no atomics): "GPU COO".
template <typename data_type>
measurement_class gpu_coo_spmv(const coo_matrix_class<data_type> &matrix, resizable_gpu_memory<data_type> &A,
                               resizable_gpu_memory<unsigned int> &col_ids,
                               resizable_gpu_memory<unsigned int> &row_ids, resizable_gpu_memory<data_type> &x,
                               resizable_gpu_memory<data_type> &y, data_type *reusable_vector,
                               const data_type *reference_y) {
  const auto &meta = matrix.meta;
  const size_t nnz = matrix.get_matrix_size();
  mfp_host::upload(A, matrix.data.get(), nnz);
  mfp_host::upload(col_ids, matrix.cols.get(), nnz);
  mfp_host::upload(row_ids, matrix.rows.get(), nnz);
  size_t wsb = 0;
  mfp_host::check(mfp_coo_workspace_bytes(meta.rows_count, (uint32_t)nnz, &wsb), "GPU COO");
  mfp_host::dev_temp ws(wsb);
  if (wsb) mfp_host::cuda_check(cudaMemset(ws.p, 0, wsb), "cudaMemset");
  const double bytes = (double)nnz * (3 * sizeof(data_type) + 8);
  return mfp_host::timed_spmv<data_type>(
      "GPU COO", meta, x, y, reusable_vector, reference_y, true, bytes, 2.0 * nnz, [&] {
        return sizeof(data_type) == 4
                   ? mfp_coo_spmv_f32(meta.rows_count, meta.cols_count, (uint32_t)nnz, (const float *)A.get(),
                                      col_ids.get(), row_ids.get(), (const float *)x.get(), (float *)y.get(), ws.p,
                                      wsb, nullptr)
                   : mfp_coo_spmv_f64(meta.rows_count, meta.cols_count, (uint32_t)nnz, (const double *)A.get(),
                                      col_ids.get(), row_ids.get(), (const double *)x.get(), (double *)y.get(),
                                      ws.p, wsb, nullptr);
      });
}

/// Sliced COO, one CTA per slice: "GPU SCOO".  As in the reference, the result
/// is compared with reference_y only when print_diff is set.
template <typename data_type>
measurement_class gpu_scoo_spmv(bool print_diff, const scoo_matrix_class<data_type> &matrix,
                                resizable_gpu_memory<data_type> &A, resizable_gpu_memory<unsigned int> &r_index,
                                resizable_gpu_memory<unsigned int> &c_index, resizable_gpu_memory<data_type> &x,
                                resizable_gpu_memory<data_type> &y, data_type *reusable_vector,
                                const data_type *reference_y) {
  const auto &meta = matrix.meta;
  const size_t nnz = matrix.get_matrix_size();
  mfp_host::upload(A, matrix.values.get(), nnz);
  mfp_host::upload(r_index, matrix.r_index.get(), nnz);
  mfp_host::upload(c_index, matrix.c_index.get(), nnz);
  const uint32_t slices = matrix.slices_count;
  mfp_host::dev_temp sp(((size_t)slices + 1) * 4);
  mfp_host::cuda_check(
      cudaMemcpy(sp.p, matrix.slices_ptr.get(), ((size_t)slices + 1) * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
  // x windows: stage a slice's x range in shared memory when 90% of them fit
  std::vector<uint32_t> win(2 * (size_t)slices);
  mfp_host::check(mfp_scoo_x_windows((uint32_t)nnz, matrix.c_index.get(), matrix.slices_ptr.get(), slices,
                                     win.data()),
                  "GPU SCOO");
  std::vector<uint32_t> widths;
  for (uint32_t s = 0; s < slices; ++s)
    if (win[2 * s + 1] > win[2 * s]) widths.push_back(win[2 * s + 1] - win[2 * s]);
  const uint32_t cap = (uint32_t)((sizeof(data_type) == 8 ? 48u : 96u) * 1024u / sizeof(data_type));
  uint32_t max_window = 0;
  if (!widths.empty()) {
    std::sort(widths.begin(), widths.end());
    if (widths[(widths.size() * 9) / 10] <= cap) max_window = (std::min(cap, widths.back()) + 3u) & ~3u;
  }
  // slices heaviest first (shortens the tail when a few slices are heavy)
  std::vector<uint32_t> order(slices);
  mfp_host::check(mfp_scoo_slice_order(slices, matrix.slices_ptr.get(), order.data()), "GPU SCOO");
  mfp_host::dev_temp dord((size_t)slices * 4);
  if (slices)
    mfp_host::cuda_check(cudaMemcpy(dord.p, order.data(), (size_t)slices * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
  mfp_host::dev_temp dwin(max_window ? win.size() * 4 : 0);
  if (max_window)
    mfp_host::cuda_check(cudaMemcpy(dwin.p, win.data(), win.size() * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
  return mfp_host::timed_spmv<data_type>(
      "GPU SCOO", meta, x, y, reusable_vector, reference_y, print_diff, mfp_host::model_bytes<data_type>(meta),
      2.0 * nnz, [&] {
        // the sort_cols layout has rows in any order within a slice
        auto f32 = matrix.cols_sorted ? mfp_scoo_spmv_unsorted_f32 : mfp_scoo_spmv_f32;
        auto f64 = matrix.cols_sorted ? mfp_scoo_spmv_unsorted_f64 : mfp_scoo_spmv_f64;
        return sizeof(data_type) == 4
                   ? f32(meta.rows_count, meta.cols_count, slices, matrix.slice_size, (const float *)A.get(),
                         c_index.get(), r_index.get(), sp.as<uint32_t>(), dwin.as<uint32_t>(), max_window,
                         dord.as<uint32_t>(), (const float *)x.get(), (float *)y.get(), nullptr)
                   : f64(meta.rows_count, meta.cols_count, slices, matrix.slice_size, (const double *)A.get(),
                         c_index.get(), r_index.get(), sp.as<uint32_t>(), dwin.as<uint32_t>(), max_window,
                         dord.as<uint32_t>(), (const double *)x.get(), (double *)y.get(), nullptr);
      });
}

namespace mfp_host {
template <typename data_type>
measurement_class hybrid(const char *label, const hybrid_matrix_class<data_type> &matrix,
                         resizable_gpu_memory<data_type> &A_ell, resizable_gpu_memory<data_type> &A_coo,
                         resizable_gpu_memory<unsigned int> &ell_col_ids,
                         resizable_gpu_memory<unsigned int> &coo_col_ids,
                         resizable_gpu_memory<unsigned int> &coo_row_ids, resizable_gpu_memory<data_type> &x,
                         resizable_gpu_memory<data_type> &y, data_type *reusable_vector, const data_type *reference_y) {
  if (!matrix.ell_matrix || !matrix.coo_matrix) throw std::runtime_error(std::string(label) + ": allocate() first");
  const auto &meta = matrix.meta;
  const auto &E = *matrix.ell_matrix;
  const auto &Cm = *matrix.coo_matrix;
  const size_t ne = E.get_matrix_size(), nc = Cm.get_matrix_size();
  upload(A_ell, E.data.get(), ne);
  upload(ell_col_ids, E.columns.get(), ne);
  upload(A_coo, Cm.data.get(), nc);
  upload(coo_col_ids, Cm.cols.get(), nc);
  upload(coo_row_ids, Cm.rows.get(), nc);
  size_t wsb = 0;
  check(mfp_hybrid_workspace_bytes(meta.rows_count, (uint32_t)nc, &wsb), label);
  dev_temp ws(wsb);
  if (wsb) cuda_check(cudaMemset(ws.p, 0, wsb), "cudaMemset");
  return timed_spmv<data_type>(label, meta, x, y, reusable_vector, reference_y, true, model_bytes<data_type>(meta),
                               2.0 * meta.non_zero_count, [&] {
                                 return sizeof(data_type) == 4
                                            ? mfp_hybrid_spmv_f32(meta.rows_count, meta.cols_count,
                                                                  E.elements_in_rows, (const float *)A_ell.get(),
                                                                  ell_col_ids.get(), (uint32_t)nc,
                                                                  (const float *)A_coo.get(), coo_col_ids.get(),
                                                                  coo_row_ids.get(), (const float *)x.get(),
                                                                  (float *)y.get(), ws.p, wsb, nullptr)
                                            : mfp_hybrid_spmv_f64(meta.rows_count, meta.cols_count,
                                                                  E.elements_in_rows, (const double *)A_ell.get(),
                                                                  ell_col_ids.get(), (uint32_t)nc,
                                                                  (const double *)A_coo.get(), coo_col_ids.get(),
                                                                  coo_row_ids.get(), (const double *)x.get(),
                                                                  (double *)y.get(), ws.p, wsb, nullptr);
                               });
}
}  // namespace mfp_host

/// Hybrid ELL + COO tail: "GPU Hybrid (TODO)" in the reference's labels.
template <typename data_type>
measurement_class gpu_hybrid_spmv(const hybrid_matrix_class<data_type> &matrix,
                                  resizable_gpu_memory<data_type> &A_ell, resizable_gpu_memory<data_type> &A_coo,
                                  resizable_gpu_memory<unsigned int> &ell_col_ids,
                                  resizable_gpu_memory<unsigned int> &coo_col_ids,
                                  resizable_gpu_memory<unsigned int> &coo_row_ids,
                                  resizable_gpu_memory<data_type> &x, resizable_gpu_memory<data_type> &y,
                                  data_type *reusable_vector, const data_type *reference_y) {
  return mfp_host::hybrid("GPU Hybrid (TODO)", matrix, A_ell, A_coo, ell_col_ids, coo_col_ids, coo_row_ids, x, y,
                          reusable_vector, reference_y);
}

/// The same engine path under the reference's second hybrid label
/// (the reference's variant used atomics on y; the engine has none).
template <typename data_type>
measurement_class gpu_hybrid_atomic_spmv(const hybrid_matrix_class<data_type> &matrix,
                                         resizable_gpu_memory<data_type> &A_ell,
                                         resizable_gpu_memory<data_type> &A_coo,
                                         resizable_gpu_memory<unsigned int> &ell_col_ids,
                                         resizable_gpu_memory<unsigned int> &coo_col_ids,
                                         resizable_gpu_memory<unsigned int> &coo_row_ids,
                                         resizable_gpu_memory<data_type> &x, resizable_gpu_memory<data_type> &y,
                                         data_type *reusable_vector, const data_type *reference_y) {
  return mfp_host::hybrid("GPU Hybrid (atomic)", matrix, A_ell, A_coo, ell_col_ids, coo_col_ids, coo_row_ids, x, y,
                          reusable_vector, reference_y);
}
