// C entry points over the reference's own classes and CPU multipliers,
// compiled from the unmodified reference sources by oracle/Makefile into
// oracle/_ref/libmfp_ref.so.  Test infrastructure only: it exists to pin the
// oracle restatement (oracle/oracle.c) and the engine's converters to the
// reference, and to time the reference's CPU loop as a baseline.
//
// Every function takes the matrix as COO triplets with double values (the
// reference's matrix_market::matrix_class input) and runs the reference
// constructor chain on it.
#include "cpu_matrix_multiplier.h"
#include "matrix_converter.h"
#include "measurement_class.h"
#include "scoo_matrix_class.h"
#include "mkl.h"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

// Defined in gpu/csr_adaptive_spmv.cu (compiled with nvcc into the same .so).
unsigned int fill_row_blocks(bool fill, unsigned int rows_count, const unsigned int *row_ptr,
                             unsigned int *row_blocks);

// MKL is not installed; the MKL path of cpu_matrix_multiplier.cpp is never
// called by the oracle.  These definitions only satisfy the linker.
extern "C" {
int mkl_enable_instructions(int) { std::abort(); }
sparse_status_t mkl_sparse_s_create_csr(sparse_matrix_t *, sparse_index_base_t, int, int, int *, int *, int *, float *) { std::abort(); }
sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *, sparse_index_base_t, int, int, int *, int *, int *, double *) { std::abort(); }
sparse_status_t mkl_sparse_optimize(sparse_matrix_t) { std::abort(); }
sparse_status_t mkl_sparse_s_mv(sparse_operation_t, float, sparse_matrix_t, struct matrix_descr, const float *, float, float *) { std::abort(); }
sparse_status_t mkl_sparse_d_mv(sparse_operation_t, double, sparse_matrix_t, struct matrix_descr, const double *, double, double *) { std::abort(); }
}

namespace {

matrix_market::matrix_class make(unsigned rows, unsigned cols, unsigned nnz, const unsigned *ri,
                                 const unsigned *ci, const double *v) {
  matrix_market::matrix_class m;
  m.meta.rows_count = rows;
  m.meta.cols_count = cols;
  m.meta.non_zero_count = nnz;
  m.meta.matrix_storage_scheme = matrix_market::matrix_class::storage_scheme::general;
  m.row_ids.assign(ri, ri + nnz);
  m.col_ids.assign(ci, ci + nnz);
  m.values.assign(v, v + nnz);
  return m;
}

template <typename T>
int csr(unsigned rows, unsigned cols, unsigned nnz, const unsigned *ri, const unsigned *ci, const double *v,
        unsigned *rp, unsigned *co, T *d) {
  auto m = make(rows, cols, nnz, ri, ci, v);
  csr_matrix_class<T> c(m);
  std::copy_n(c.row_ptr.get(), rows + 1, rp);
  std::copy_n(c.columns.get(), nnz, co);
  std::copy_n(c.data.get(), nnz, d);
  return 0;
}

// width < 0: the max-width constructor; else the fixed-width one.
template <typename T>
unsigned ell(unsigned rows, unsigned cols, unsigned nnz, const unsigned *ri, const unsigned *ci, const double *v,
             long long width, T *d, unsigned *co) {
  auto m = make(rows, cols, nnz, ri, ci, v);
  csr_matrix_class<T> c(m);
  std::unique_ptr<ell_matrix_class<T>> e;
  if (width < 0)
    e.reset(new ell_matrix_class<T>(c));
  else
    e.reset(new ell_matrix_class<T>(c, (unsigned)width));
  if (d) {
    std::copy_n(e->data.get(), e->get_matrix_size(), d);
    std::copy_n(e->columns.get(), e->get_matrix_size(), co);
  }
  return e->elements_in_rows;
}

template <typename T>
unsigned coo(unsigned rows, unsigned cols, unsigned nnz, const unsigned *ri, const unsigned *ci, const double *v,
             long long start, T *d, unsigned *co, unsigned *ro) {
  auto m = make(rows, cols, nnz, ri, ci, v);
  csr_matrix_class<T> c(m);
  std::unique_ptr<coo_matrix_class<T>> o;
  if (start < 0)
    o.reset(new coo_matrix_class<T>(c));
  else
    o.reset(new coo_matrix_class<T>(c, (unsigned)start));
  const size_t n = o->get_matrix_size();
  if (d) {
    std::copy_n(o->data.get(), n, d);
    std::copy_n(o->cols.get(), n, co);
    std::copy_n(o->rows.get(), n, ro);
  }
  return (unsigned)n;
}

template <typename T>
void hybrid(unsigned rows, unsigned cols, unsigned nnz, const unsigned *ri, const unsigned *ci, const double *v,
            double percent, unsigned *width, unsigned *coo_count, T *ed, unsigned *ec, T *cd, unsigned *cc,
            unsigned *cr) {
  auto m = make(rows, cols, nnz, ri, ci, v);
  csr_matrix_class<T> c(m);
  hybrid_matrix_class<T> h(c);
  h.allocate(c, percent);
  *width = h.ell_matrix->elements_in_rows;
  *coo_count = (unsigned)h.coo_matrix->get_matrix_size();
  if (ed) {
    std::copy_n(h.ell_matrix->data.get(), h.ell_matrix->get_matrix_size(), ed);
    std::copy_n(h.ell_matrix->columns.get(), h.ell_matrix->get_matrix_size(), ec);
    std::copy_n(h.coo_matrix->data.get(), *coo_count, cd);
    std::copy_n(h.coo_matrix->cols.get(), *coo_count, cc);
    std::copy_n(h.coo_matrix->rows.get(), *coo_count, cr);
  }
}

template <typename T>
void scoo(unsigned rows, unsigned cols, unsigned nnz, const unsigned *ri, const unsigned *ci, const double *v,
          unsigned sm, size_t smem, unsigned *params, T *vals, unsigned *c_index, unsigned *r_index,
          unsigned *slices_ptr) {
  auto m = make(rows, cols, nnz, ri, ci, v);
  csr_matrix_class<T> c(m);
  scoo_matrix_class<T> s(sm, smem, c);
  params[0] = s.slices_count;
  params[1] = s.slice_size;
  params[2] = s.lane_size;
  if (vals) {
    std::copy_n(s.values.get(), nnz, vals);
    std::copy_n(s.c_index.get(), nnz, c_index);
    std::copy_n(s.r_index.get(), nnz, r_index);
    std::copy_n(s.slices_ptr.get(), s.slices_count + 1, slices_ptr);
  }
}

template <typename T>
void spmv(unsigned rows, unsigned cols, unsigned nnz, const unsigned *ri, const unsigned *ci, const double *v,
          int reduce_order, T *y) {
  auto m = make(rows, cols, nnz, ri, ci, v);
  csr_matrix_class<T> c(m);
  std::vector<T> x(std::max(rows, cols));
  if (reduce_order)
    cpu_csr_spmv_single_thread_naive_with_reduce_order(c, x.data(), y);
  else
    cpu_csr_spmv_single_thread_naive(c, x.data(), y);
}

// Timing harness: the reference's single-thread CSR loop run concurrently on
// `threads` contiguous row ranges (the split of cpu_matrix_multiplier.cpp:
// 277-279), each range its own csr_matrix_class built by the reference
// constructor.  Elapsed = the slowest range, as the reference's parallel
// variant reports it (:295-299).
struct bench {
  int f64 = 0;
  unsigned rows = 0;
  std::vector<std::unique_ptr<csr_matrix_class<float>>> sf;
  std::vector<std::unique_ptr<csr_matrix_class<double>>> sd;
  std::vector<unsigned> begin;
  std::vector<std::vector<float>> xf;
  std::vector<std::vector<double>> xd;
};

}  // namespace

extern "C" {

int ref_csr_f32(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                unsigned *rp, unsigned *co, float *d) {
  return csr<float>(r, c, n, ri, ci, v, rp, co, d);
}
int ref_csr_f64(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                unsigned *rp, unsigned *co, double *d) {
  return csr<double>(r, c, n, ri, ci, v, rp, co, d);
}
void ref_rows_statistics(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                         unsigned *out, double *sd) {
  auto m = make(r, c, n, ri, ci, v);
  csr_matrix_class<float> cm(m);
  const auto s = get_rows_statistics(cm.meta, cm.row_ptr.get());
  out[0] = s.min_elements_in_rows;
  out[1] = s.max_elements_in_rows;
  out[2] = s.avg_elements_in_rows;
  *sd = s.elements_in_rows_std_deviation;
}
unsigned ref_ell_f32(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                     long long w, float *d, unsigned *co) {
  return ell<float>(r, c, n, ri, ci, v, w, d, co);
}
unsigned ref_ell_f64(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                     long long w, double *d, unsigned *co) {
  return ell<double>(r, c, n, ri, ci, v, w, d, co);
}
unsigned ref_coo_f32(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                     long long start, float *d, unsigned *co, unsigned *ro) {
  return coo<float>(r, c, n, ri, ci, v, start, d, co, ro);
}
unsigned ref_coo_f64(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                     long long start, double *d, unsigned *co, unsigned *ro) {
  return coo<double>(r, c, n, ri, ci, v, start, d, co, ro);
}
void ref_hybrid_f32(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                    double p, unsigned *w, unsigned *cn, float *ed, unsigned *ec, float *cd, unsigned *cc,
                    unsigned *cr) {
  hybrid<float>(r, c, n, ri, ci, v, p, w, cn, ed, ec, cd, cc, cr);
}
void ref_hybrid_f64(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                    double p, unsigned *w, unsigned *cn, double *ed, unsigned *ec, double *cd, unsigned *cc,
                    unsigned *cr) {
  hybrid<double>(r, c, n, ri, ci, v, p, w, cn, ed, ec, cd, cc, cr);
}
void ref_scoo_f32(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                  unsigned sm, size_t smem, unsigned *prm, float *vals, unsigned *cx, unsigned *rx, unsigned *sp) {
  scoo<float>(r, c, n, ri, ci, v, sm, smem, prm, vals, cx, rx, sp);
}
void ref_scoo_f64(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                  unsigned sm, size_t smem, unsigned *prm, double *vals, unsigned *cx, unsigned *rx, unsigned *sp) {
  scoo<double>(r, c, n, ri, ci, v, sm, smem, prm, vals, cx, rx, sp);
}
void ref_spmv_f32(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                  int reduce_order, float *y) {
  spmv<float>(r, c, n, ri, ci, v, reduce_order, y);
}
void ref_spmv_f64(unsigned r, unsigned c, unsigned n, const unsigned *ri, const unsigned *ci, const double *v,
                  int reduce_order, double *y) {
  spmv<double>(r, c, n, ri, ci, v, reduce_order, y);
}
unsigned ref_fill_row_blocks(int fill, unsigned rows, const unsigned *rp, unsigned *blocks) {
  return fill_row_blocks(fill != 0, rows, rp, blocks);
}
void ref_measurement(const char *fmt, double elapsed, double bytes, double ops, double *out) {
  measurement_class m(fmt, elapsed, bytes, ops);
  out[0] = m.get_elapsed();
  out[1] = m.get_effective_bandwidth();
  out[2] = m.get_computational_throughput();
}

// CSR input (row_ptr, columns, values as double) -> per-thread reference CSR objects.
void *ref_bench_create(int f64, unsigned threads, unsigned rows, unsigned cols, const unsigned *rp,
                       const unsigned *ci, const double *v) {
  auto *b = new bench();
  b->f64 = f64;
  b->rows = rows;
  threads = std::max(1u, std::min(threads, std::max(1u, rows)));
  const unsigned per = rows / threads;
  std::vector<std::thread> th;
  b->sf.resize(threads);
  b->sd.resize(threads);
  b->begin.resize(threads + 1);
  for (unsigned t = 0; t < threads; ++t) {
    b->begin[t] = per * t;
    b->begin[t + 1] = t == threads - 1 ? rows : (t + 1) * per;
  }
  if (f64)
    b->xd.assign(threads, std::vector<double>(std::max(rows, cols)));
  else
    b->xf.assign(threads, std::vector<float>(std::max(rows, cols)));
  for (unsigned t = 0; t < threads; ++t)
    th.emplace_back([=] {
      const unsigned r0 = b->begin[t], r1 = b->begin[t + 1];
      const unsigned e0 = rp[r0], e1 = rp[r1];
      matrix_market::matrix_class m;
      m.meta.rows_count = r1 - r0;
      m.meta.cols_count = cols;
      m.meta.non_zero_count = e1 - e0;
      m.row_ids.resize(e1 - e0);
      for (unsigned r = r0; r < r1; ++r)
        for (unsigned e = rp[r]; e < rp[r + 1]; ++e) m.row_ids[e - e0] = r - r0;
      m.col_ids.assign(ci + e0, ci + e1);
      m.values.assign(v + e0, v + e1);
      if (b->f64)
        b->sd[t].reset(new csr_matrix_class<double>(m));
      else
        b->sf[t].reset(new csr_matrix_class<float>(m));
    });
  for (auto &t : th) t.join();
  return b;
}

// One timed pass; y receives A*1 (the reference fixes x = 1).  Returns the
// slowest thread's elapsed seconds as the reference measures it.
double ref_bench_run(void *h, void *y) {
  auto *b = static_cast<bench *>(h);
  const unsigned threads = (unsigned)b->begin.size() - 1;
  std::vector<double> el(threads, 0.0);
  std::atomic<unsigned> ready{0};
  std::vector<std::thread> th;
  for (unsigned t = 0; t < threads; ++t)
    th.emplace_back([&, t] {
      ready.fetch_add(1);
      while (ready.load() < threads) {
      }
      if (b->f64)
        el[t] = cpu_csr_spmv_single_thread_naive(*b->sd[t], b->xd[t].data(),
                                                 static_cast<double *>(y) + b->begin[t]).get_elapsed();
      else
        el[t] = cpu_csr_spmv_single_thread_naive(*b->sf[t], b->xf[t].data(),
                                                 static_cast<float *>(y) + b->begin[t]).get_elapsed();
    });
  for (auto &t : th) t.join();
  return *std::max_element(el.begin(), el.end());
}

void ref_bench_destroy(void *h) { delete static_cast<bench *>(h); }

}  // extern "C"
