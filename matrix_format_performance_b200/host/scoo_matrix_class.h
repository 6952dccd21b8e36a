// Sliced COO with the reference's interface (common/scoo_matrix_class.h:11-39):
// the slice parameters from (sm_count, shared memory per block, sizeof(T)) and
// the arrays values / c_index / r_index / slices_ptr, built by the engine's
// library (mfp_scoo_params_compute, mfp_scoo_from_csr_*), bit-exact with the
// reference's construction.
#pragma once

#include <memory>

#include "matrix_converter.h"

template <typename data_type>
class scoo_matrix_class {
 public:
  scoo_matrix_class() = delete;
  // sort_cols: the reference's disabled option (scoo_matrix_class.cpp:102-138),
  // each slice in column order (stable sort; the reference's is not stable)
  explicit scoo_matrix_class(unsigned int sm_count, size_t shared_mem_size, csr_matrix_class<data_type> &matrix,
                             bool sort_cols = false)
      : meta(matrix.meta), cols_sorted(sort_cols) {
    mfp_scoo_params p{};
    mfp_host::check(mfp_scoo_params_compute(meta.rows_count, sm_count, shared_mem_size,
                                            mfp_host::vt<data_type>::value, &p),
                    "scoo_matrix_class");
    slices_count = p.slices_count;
    slice_size = p.slice_size;
    lane_size = p.lane_size;
    elements_count = meta.non_zero_count;
    const size_t n = elements_count ? elements_count : 1;
    values.reset(new data_type[n]);
    c_index.reset(new unsigned int[n]);
    r_index.reset(new unsigned int[n]);
    slices_ptr.reset(new unsigned int[slices_count + 1]);
    int st = sizeof(data_type) == 4
                 ? mfp_scoo_from_csr_f32(meta.rows_count, matrix.row_ptr.get(), matrix.columns.get(),
                                         (const float *)matrix.data.get(), &p, (float *)values.get(), c_index.get(),
                                         r_index.get(), slices_ptr.get())
                 : mfp_scoo_from_csr_f64(meta.rows_count, matrix.row_ptr.get(), matrix.columns.get(),
                                         (const double *)matrix.data.get(), &p, (double *)values.get(),
                                         c_index.get(), r_index.get(), slices_ptr.get());
    mfp_host::check(st, "scoo_matrix_class");
    if (sort_cols) {
      st = sizeof(data_type) == 4 ? mfp_scoo_sort_cols_f32(slices_count, slices_ptr.get(), (float *)values.get(),
                                                           c_index.get(), r_index.get())
                                  : mfp_scoo_sort_cols_f64(slices_count, slices_ptr.get(), (double *)values.get(),
                                                           c_index.get(), r_index.get());
      mfp_host::check(st, "scoo_matrix_class sort_cols");
    }
  }

  const matrix_market::matrix_class::matrix_meta meta;
  const bool cols_sorted;  // engine extension: true for the sort_cols layout

 public:
  unsigned int slices_count{};
  unsigned int slice_size{};
  unsigned int lane_size{};

  std::unique_ptr<data_type[]> values;
  std::unique_ptr<unsigned int[]> c_index;
  std::unique_ptr<unsigned int[]> r_index;
  std::unique_ptr<unsigned int[]> slices_ptr;

  size_t get_matrix_size() const { return elements_count; }

 private:
  size_t elements_count{};
};
