// Host matrix classes with the reference's interface
// (common/matrix_converter.h:12-96): csr_matrix_class, ell_matrix_class,
// coo_matrix_class, hybrid_matrix_class and get_rows_statistics, with the same
// member names and meanings.  The conversions run in the engine's library
// (mfp_csr_from_coo_*, mfp_ell_from_csr_*, mfp_coo_from_csr_*,
// mfp_hybrid_width), which reproduces the reference's arrays bit for bit.
// A conversion error throws std::runtime_error with the library's message.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>

#include "matrix_market_reader.h"
#include "mfp_spmv.h"

namespace mfp_host {
inline void check(int status, const char *what) {
  if (status != MFP_SUCCESS) {
    const char *msg = mfp_last_error();
    throw std::runtime_error(std::string(what) + ": " + (msg ? msg : mfp_status_string(status)));
  }
}
template <typename T> struct vt;
template <> struct vt<float> { static constexpr int value = MFP_F32; };
template <> struct vt<double> { static constexpr int value = MFP_F64; };

inline int csr_from_coo(uint32_t r, uint32_t c, uint32_t n, int s, const uint32_t *ri, const uint32_t *ci,
                        const double *v, uint32_t *rp, uint32_t *cols, float *d) {
  return mfp_csr_from_coo_f32(r, c, n, s, ri, ci, v, rp, cols, d);
}
inline int csr_from_coo(uint32_t r, uint32_t c, uint32_t n, int s, const uint32_t *ri, const uint32_t *ci,
                        const double *v, uint32_t *rp, uint32_t *cols, double *d) {
  return mfp_csr_from_coo_f64(r, c, n, s, ri, ci, v, rp, cols, d);
}
inline int ell_from_csr(uint32_t r, const uint32_t *rp, const uint32_t *c, const float *d, uint32_t w, float *ed,
                        uint32_t *ec) {
  return mfp_ell_from_csr_f32(r, rp, c, d, w, ed, ec);
}
inline int ell_from_csr(uint32_t r, const uint32_t *rp, const uint32_t *c, const double *d, uint32_t w, double *ed,
                        uint32_t *ec) {
  return mfp_ell_from_csr_f64(r, rp, c, d, w, ed, ec);
}
inline int coo_from_csr(uint32_t r, const uint32_t *rp, const uint32_t *c, const float *d, uint32_t k, float *cd,
                        uint32_t *cc, uint32_t *cr) {
  return mfp_coo_from_csr_f32(r, rp, c, d, k, cd, cc, cr);
}
inline int coo_from_csr(uint32_t r, const uint32_t *rp, const uint32_t *c, const double *d, uint32_t k, double *cd,
                        uint32_t *cc, uint32_t *cr) {
  return mfp_coo_from_csr_f64(r, rp, c, d, k, cd, cc, cr);
}
// The algorithmic bytes of one SpMV: nnz*(sizeof(T)+4) + (rows+1)*4 +
// cols*sizeof(T) + rows*sizeof(T).
template <typename T>
double model_bytes(const matrix_market::matrix_class::matrix_meta &m) {
  return (double)m.non_zero_count * (sizeof(T) + 4) + ((double)m.rows_count + 1) * 4 +
         (double)m.cols_count * sizeof(T) + (double)m.rows_count * sizeof(T);
}
}  // namespace mfp_host

struct matrix_rows_statistic {
  unsigned int min_elements_in_rows{};
  unsigned int max_elements_in_rows{};
  unsigned int avg_elements_in_rows{};
  double elements_in_rows_std_deviation{};
};

inline matrix_rows_statistic get_rows_statistics(const matrix_market::matrix_class::matrix_meta &meta,
                                                 const unsigned int *row_ptr) {
  mfp_rows_statistic s{};
  mfp_host::check(mfp_get_rows_statistics(meta.rows_count, row_ptr, &s), "get_rows_statistics");
  return {s.min_elements_in_rows, s.max_elements_in_rows, s.avg_elements_in_rows, s.elements_in_rows_std_deviation};
}

template <typename data_type>
class csr_matrix_class {
 public:
  csr_matrix_class() = delete;
  explicit csr_matrix_class(const matrix_market::matrix_class &matrix, bool row_ptr_only = false)
      : meta(matrix.meta) {
    const unsigned nnz = meta.non_zero_count;
    row_ptr.reset(new unsigned int[meta.rows_count + 1]);
    columns.reset(new unsigned int[nnz ? nnz : 1]);
    data.reset(new data_type[nnz ? nnz : 1]);
    mfp_host::check(mfp_host::csr_from_coo(meta.rows_count, meta.cols_count, nnz,
                                           (int)meta.matrix_storage_scheme, matrix.get_row_ids(),
                                           matrix.get_col_ids(), matrix.get_dbl_data(), row_ptr.get(),
                                           columns.get(), data.get()),
                    "csr_matrix_class");
    if (row_ptr_only) {
      columns.reset();
      data.reset();
    }
  }

  const matrix_market::matrix_class::matrix_meta meta;

  size_t get_matrix_size() const { return meta.non_zero_count; }

 public:
  std::unique_ptr<data_type[]> data;
  std::unique_ptr<unsigned int[]> columns;
  std::unique_ptr<unsigned int[]> row_ptr;
};

template <typename data_type>
class ell_matrix_class {
 public:
  ell_matrix_class() = delete;
  explicit ell_matrix_class(csr_matrix_class<data_type> &matrix) : meta(matrix.meta) {
    unsigned w = 0;
    mfp_host::check(mfp_ell_width(meta.rows_count, matrix.row_ptr.get(), &w), "ell_matrix_class");
    build(matrix, w);
  }
  ell_matrix_class(csr_matrix_class<data_type> &matrix, unsigned int elements_in_row_arg) : meta(matrix.meta) {
    build(matrix, elements_in_row_arg);
  }

  static size_t estimate_size(csr_matrix_class<data_type> &matrix) {
    unsigned w = 0;
    mfp_host::check(mfp_ell_width(matrix.meta.rows_count, matrix.row_ptr.get(), &w), "ell_matrix_class");
    return (size_t)w * matrix.meta.rows_count;
  }

  const matrix_market::matrix_class::matrix_meta meta;

  size_t get_matrix_size() const { return (size_t)elements_in_rows * meta.rows_count; }

 public:
  std::unique_ptr<data_type[]> data;
  std::unique_ptr<unsigned int[]> columns;

  unsigned int elements_in_rows = 0;

 private:
  void build(csr_matrix_class<data_type> &matrix, unsigned w) {
    elements_in_rows = w;
    const size_t n = (size_t)w * meta.rows_count;
    data.reset(new data_type[n ? n : 1]);
    columns.reset(new unsigned int[n ? n : 1]);
    mfp_host::check(mfp_host::ell_from_csr(meta.rows_count, matrix.row_ptr.get(), matrix.columns.get(),
                                           matrix.data.get(), w, data.get(), columns.get()),
                    "ell_matrix_class");
  }
};

template <typename data_type>
class coo_matrix_class {
 public:
  coo_matrix_class() = delete;
  explicit coo_matrix_class(csr_matrix_class<data_type> &matrix) : coo_matrix_class(matrix, 0u) {}
  coo_matrix_class(csr_matrix_class<data_type> &matrix, unsigned int element_start) : meta(matrix.meta) {
    unsigned n = 0;
    mfp_host::check(mfp_coo_count(meta.rows_count, matrix.row_ptr.get(), element_start, &n), "coo_matrix_class");
    elements_count = n;
    data.reset(new data_type[n ? n : 1]);
    cols.reset(new unsigned int[n ? n : 1]);
    rows.reset(new unsigned int[n ? n : 1]);
    mfp_host::check(mfp_host::coo_from_csr(meta.rows_count, matrix.row_ptr.get(), matrix.columns.get(),
                                           matrix.data.get(), element_start, data.get(), cols.get(), rows.get()),
                    "coo_matrix_class");
  }

  const matrix_market::matrix_class::matrix_meta meta;

  size_t get_matrix_size() const { return elements_count; }

 public:
  std::unique_ptr<data_type[]> data;
  std::unique_ptr<unsigned int[]> cols;
  std::unique_ptr<unsigned int[]> rows;

 private:
  size_t elements_count{};
};

template <typename data_type>
class hybrid_matrix_class {
 public:
  hybrid_matrix_class() = delete;
  explicit hybrid_matrix_class(csr_matrix_class<data_type> &matrix) : meta(matrix.meta) {}

  // ELL width = avg + (max - avg) * percent (integer average), the rest in COO
  void allocate(csr_matrix_class<data_type> &matrix, double percent) {
    unsigned w = 0;
    mfp_host::check(mfp_hybrid_width(meta.rows_count, matrix.row_ptr.get(), percent, &w), "hybrid_matrix_class");
    allocate_width(matrix, w);
  }
  // engine extension: an explicit ELL width (e.g. a row-length quantile)
  void allocate_width(csr_matrix_class<data_type> &matrix, unsigned int width) {
    ell_matrix.reset(new ell_matrix_class<data_type>(matrix, width));
    coo_matrix.reset(new coo_matrix_class<data_type>(matrix, width));
  }

  const matrix_market::matrix_class::matrix_meta meta;

  std::unique_ptr<ell_matrix_class<data_type>> ell_matrix;
  std::unique_ptr<coo_matrix_class<data_type>> coo_matrix;
};
