// The reference's cuSPARSE comparator, gpu_csr_cusparse_spmv
// (gpu/gpu_matrix_multiplier.h, gpu_matrix_multiplier.cu:135-257: "GPU CSR
// (cuSparse)"), on cuSPARSE's generic SpMV through libmfp_yardstick.so (the
// legacy cusparse?csrmv the reference called no longer exists).  Same
// arguments and behaviour as the engine's gpu_csr_spmv: x := 1, one timed
// launch, y into reusable_vector, compared with reference_y.  Library code,
// a yardstick beside the engine's operators.
#pragma once

#include "gpu_matrix_multiplier.h"
#include "mfp_yardstick.h"

template <typename data_type>
measurement_class gpu_csr_cusparse_spmv(const csr_matrix_class<data_type> &matrix,
                                        resizable_gpu_memory<data_type> &A,
                                        resizable_gpu_memory<unsigned int> &col_ids,
                                        resizable_gpu_memory<unsigned int> &row_ptr,
                                        resizable_gpu_memory<data_type> &x, resizable_gpu_memory<data_type> &y,
                                        data_type *reusable_vector, const data_type *reference_y) {
  const auto &meta = matrix.meta;
  const size_t nnz = meta.non_zero_count;
  mfp_host::upload(A, matrix.data.get(), nnz);
  mfp_host::upload(col_ids, matrix.columns.get(), nnz);
  mfp_host::upload(row_ptr, matrix.row_ptr.get(), (size_t)meta.rows_count + 1);
  const double bytes = (double)nnz * (2 * sizeof(data_type) + 4) + 2.0 * meta.rows_count * 4 +
                       (double)meta.rows_count * sizeof(data_type);
  auto m = mfp_host::timed_spmv<data_type>(
      "GPU CSR (cuSparse)", meta, x, y, reusable_vector, reference_y, true, bytes, 2.0 * nnz, [&] {
        const int st = mfp_cusparse_spmv(0, 0, sizeof(data_type) == 8 ? 1 : 0, meta.rows_count, meta.cols_count,
                                         (uint32_t)nnz, row_ptr.get(), col_ids.get(), A.get(), x.get(), y.get(), 0,
                                         0, nullptr, nullptr);
        return st ? (int)MFP_ERROR_CUDA : (int)MFP_SUCCESS;
      });
  return m;
}
