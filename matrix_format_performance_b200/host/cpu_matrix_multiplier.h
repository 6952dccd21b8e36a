// CPU CSR SpMV with the reference's driver-facing interface
// (cpu/cpu_matrix_multiplier.h): each call sets x := 1, writes y and returns a
// timed measurement_class.  The driver uses them for its "CPU CSR" columns and
// for the reference answers the GPU operators are compared against.
//   cpu_csr_spmv_single_thread_naive           "CPU CSR": a row loop in CSR order
//   cpu_csr_spmv_single_thread_naive_with_reduce_order
//                                              "CPU CSR Reduce order": 32 lane
//                                              partial sums and a halving tree
//                                              (the warp order of a 32-lane
//                                              vector kernel)
//   cpu_csr_spmv_multi_thread_naive            "CPU CSR Parallel": contiguous row
//                                              ranges over all hardware threads,
//                                              elapsed = slowest thread
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <thread>
#include <vector>

#include "matrix_converter.h"
#include "measurement_class.h"

namespace mfp_host {
template <typename T>
double csr_reference_bytes(const matrix_market::matrix_class::matrix_meta &m) {
  return (double)m.non_zero_count * (2 * sizeof(T) + 4) + 2.0 * m.rows_count * 4 + (double)m.rows_count * sizeof(T);
}
template <typename T>
void csr_rows(const csr_matrix_class<T> &A, const T *x, T *y, unsigned r0, unsigned r1) {
  const unsigned *rp = A.row_ptr.get(), *ci = A.columns.get();
  const T *a = A.data.get();
  for (unsigned r = r0; r < r1; ++r) {
    T dot = 0;
    for (unsigned e = rp[r]; e < rp[r + 1]; ++e) dot += a[e] * x[ci[e]];
    y[r] = dot;
  }
}
}  // namespace mfp_host

template <typename data_type>
measurement_class cpu_csr_spmv_single_thread_naive(const csr_matrix_class<data_type> &matrix, data_type *x,
                                                   data_type *y) {
  std::fill_n(x, matrix.meta.cols_count, data_type(1));
  const auto t0 = std::chrono::steady_clock::now();
  mfp_host::csr_rows(matrix, x, y, 0, matrix.meta.rows_count);
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return measurement_class("CPU CSR", s, mfp_host::csr_reference_bytes<data_type>(matrix.meta),
                           2.0 * matrix.meta.non_zero_count, mfp_host::model_bytes<data_type>(matrix.meta));
}

template <typename data_type>
measurement_class cpu_csr_spmv_single_thread_naive_with_reduce_order(const csr_matrix_class<data_type> &matrix,
                                                                     data_type *x, data_type *y) {
  std::fill_n(x, matrix.meta.cols_count, data_type(1));
  const unsigned *rp = matrix.row_ptr.get(), *ci = matrix.columns.get();
  const data_type *a = matrix.data.get();
  const auto t0 = std::chrono::steady_clock::now();
  std::array<data_type, 32> part{};
  for (unsigned r = 0; r < matrix.meta.rows_count; ++r) {
    for (unsigned l = 0; l < 32; ++l) {
      part[l] = 0;
      for (unsigned e = rp[r] + l; e < rp[r + 1]; e += 32) part[l] += a[e] * x[ci[e]];
    }
    for (unsigned half = 16; half > 0; half /= 2)
      for (unsigned l = 0; l < half; ++l) part[l] += part[l + half];
    y[r] = part[0];
  }
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return measurement_class("CPU CSR Reduce order", s, mfp_host::csr_reference_bytes<data_type>(matrix.meta),
                           2.0 * matrix.meta.non_zero_count, mfp_host::model_bytes<data_type>(matrix.meta));
}

template <typename data_type>
measurement_class cpu_csr_spmv_multi_thread_naive(const csr_matrix_class<data_type> &matrix, data_type *x,
                                                  data_type *y) {
  std::fill_n(x, matrix.meta.cols_count, data_type(1));
  const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
  const unsigned rows = matrix.meta.rows_count;
  std::vector<double> el(threads, 0.0);
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      const unsigned r0 = (unsigned)((uint64_t)rows * t / threads), r1 = (unsigned)((uint64_t)rows * (t + 1) / threads);
      const auto t0 = std::chrono::steady_clock::now();
      mfp_host::csr_rows(matrix, x, y, r0, r1);
      el[t] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
  for (auto &p : pool) p.join();
  const double s = *std::max_element(el.begin(), el.end());
  return measurement_class("CPU CSR Parallel", s, mfp_host::csr_reference_bytes<data_type>(matrix.meta),
                           2.0 * matrix.meta.non_zero_count, mfp_host::model_bytes<data_type>(matrix.meta));
}
