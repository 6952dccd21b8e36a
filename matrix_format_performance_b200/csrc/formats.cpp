// Host-side format construction with the reference's exact layouts, plus
// the measurement record and the result comparison.
//
// Layout rules follow common/matrix_converter.cpp and
// common/scoo_matrix_class.cpp of the reference; each function cites the
// lines it reproduces.  The arrays produced here are compared element for
// element with the reference's own converters in the test suite.
#include "host_common.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

using namespace mfp;

namespace {

// CSR from COO triplets (matrix_converter.cpp:15-87): count elements per
// row, exclusive scan into row_ptr, place elements in input order, then
// order each row by column.  The per-row order is a stable sort on the column
// (identical to the reference for any matrix without repeated (row, col)
// entries; repeated entries keep their input order).
template <typename T>
int csr_from_coo(uint32_t rows, uint32_t cols, uint32_t nnz, int scheme, const uint32_t *ri,
                 const uint32_t *ci, const double *v, uint32_t *row_ptr, uint32_t *columns, T *data) {
  if (scheme != 0)
    return fail(MFP_ERROR_NOT_SUPPORTED, "Only general matrices are supported");
  if (!row_ptr || (nnz && (!ri || !ci || !v || !columns || !data)))
    return fail(MFP_ERROR_INVALID_VALUE, "null array");
  std::fill_n(row_ptr, (size_t)rows + 1, 0u);
  for (uint32_t i = 0; i < nnz; ++i) {
    if (ri[i] >= rows) return fail(MFP_ERROR_INVALID_VALUE, "row id %u >= rows %u", ri[i], rows);
    if (ci[i] >= cols) return fail(MFP_ERROR_INVALID_VALUE, "col id %u >= cols %u", ci[i], cols);
    row_ptr[ri[i]]++;
  }
  uint32_t acc = 0;
  for (uint32_t r = 0; r <= rows; ++r) {
    const uint32_t c = row_ptr[r];
    row_ptr[r] = acc;
    acc += c;
  }
  std::vector<uint32_t> fill(rows, 0u);
  for (uint32_t i = 0; i < nnz; ++i) {
    const uint32_t at = row_ptr[ri[i]] + fill[ri[i]]++;
    data[at] = static_cast<T>(v[i]);
    columns[at] = ci[i];
  }
  std::vector<uint32_t> perm;
  std::vector<uint32_t> tc;
  std::vector<T> tv;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t b = row_ptr[r], e = row_ptr[r + 1];
    bool sorted = true;
    for (uint32_t k = b + 1; k < e && sorted; ++k) sorted = columns[k - 1] <= columns[k];
    if (sorted) continue;
    const uint32_t n = e - b;
    perm.resize(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::stable_sort(perm.begin(), perm.end(),
                     [&](uint32_t l, uint32_t q) { return columns[b + l] < columns[b + q]; });
    tc.assign(columns + b, columns + e);
    tv.assign(data + b, data + e);
    for (uint32_t k = 0; k < n; ++k) {
      columns[b + k] = tc[perm[k]];
      data[b + k] = tv[perm[k]];
    }
  }
  return ok();
}

template <typename T>
int ell_from_csr(uint32_t rows, const uint32_t *rp, const uint32_t *columns, const T *data,
                 uint32_t width, T *ed, uint32_t *ec) {
  const size_t n = (size_t)rows * width;
  if (!rp || (n && (!ed || !ec))) return fail(MFP_ERROR_INVALID_VALUE, "null array");
  std::fill_n(ed, n, T(0));
  std::fill_n(ec, n, 0u);
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t b = rp[r], e = std::min(rp[r + 1], rp[r] + width);
    for (uint32_t k = b; k < e; ++k) {
      ed[(size_t)(k - b) * rows + r] = data[k];
      ec[(size_t)(k - b) * rows + r] = columns[k];
    }
  }
  return ok();
}

template <typename T>
int coo_from_csr(uint32_t rows, const uint32_t *rp, const uint32_t *columns, const T *data,
                 uint32_t start, T *cd, uint32_t *cc, uint32_t *cr) {
  if (!rp) return fail(MFP_ERROR_INVALID_VALUE, "null row_ptr");
  uint32_t id = 0;
  for (uint32_t r = 0; r < rows; ++r)
    for (uint32_t k = rp[r]; k < rp[r + 1]; ++k)
      if (k - rp[r] >= start) {
        cd[id] = data[k];
        cc[id] = columns[k];
        cr[id] = r;
        ++id;
      }
  return ok();
}

// next_pow_2 / prev_pow_2 (scoo_matrix_class.cpp:13-28), 32-bit unsigned.
uint32_t next_pow2(uint32_t x) {
  --x;
  x |= x >> 1u;
  x |= x >> 2u;
  x |= x >> 4u;
  x |= x >> 8u;
  x |= x >> 16u;
  return ++x;
}
uint32_t prev_pow2(uint32_t x) {
  const uint32_t n = next_pow2(x);
  return n > x ? n / 2 : n;
}

template <typename T>
int scoo_from_csr(uint32_t rows, const uint32_t *rp, const uint32_t *columns, const T *data,
                  const mfp_scoo_params *prm, T *values, uint32_t *ci, uint32_t *ri, uint32_t *sp) {
  if (!rp || !prm || !sp) return fail(MFP_ERROR_INVALID_VALUE, "null array");
  if (prm->slice_size == 0 && rows) return fail(MFP_ERROR_INVALID_VALUE, "slice_size 0");
  std::fill_n(sp, (size_t)prm->slices_count + 1, 0u);
  // scoo_matrix_class.cpp:69-93: a new slice every slice_size rows, the
  // trailing slices_ptr entries stay zero.
  uint32_t offset = 0, slice = 0, last = 0;
  for (uint32_t r = 0; r < rows; ++r) {
    if (r - last >= prm->slice_size || slice == 0) {
      if (slice > prm->slices_count) return fail(MFP_ERROR_INVALID_VALUE, "too many slices");
      sp[slice++] = offset;
      last = r;
    }
    for (uint32_t k = rp[r]; k < rp[r + 1]; ++k) {
      values[offset] = data[k];
      ci[offset] = columns[k];
      ri[offset] = r;
      ++offset;
    }
  }
  if (slice > prm->slices_count) return fail(MFP_ERROR_INVALID_VALUE, "too many slices");
  sp[slice] = offset;
  return ok();
}

// The reference's disabled sort_cols block (scoo_matrix_class.cpp:102-138):
// each slice's elements ordered by column.  The reference sorts a permutation
// with std::sort, which is not stable, so its order between equal columns is
// unspecified; this restatement sorts stably (equal columns keep CSR order).
template <typename T>
int scoo_sort_cols(uint32_t slices, const uint32_t *sp, T *values, uint32_t *ci, uint32_t *ri) {
  if (!sp) return fail(MFP_ERROR_INVALID_VALUE, "null slices_ptr");
  std::vector<uint32_t> perm, tc, tr;
  std::vector<T> tv;
  for (uint32_t s = 0; s < slices; ++s) {
    const uint32_t b = sp[s], e = sp[s + 1];
    if (b >= e) continue;
    if (!values || !ci || !ri) return fail(MFP_ERROR_INVALID_VALUE, "null array");
    const uint32_t n = e - b;
    perm.resize(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t l, uint32_t r) { return ci[b + l] < ci[b + r]; });
    tv.assign(values + b, values + e);
    tc.assign(ci + b, ci + e);
    tr.assign(ri + b, ri + e);
    for (uint32_t k = 0; k < n; ++k) {
      values[b + k] = tv[perm[k]];
      ci[b + k] = tc[perm[k]];
      ri[b + k] = tr[perm[k]];
    }
  }
  return ok();
}

template <typename T>
int compare(uint32_t n, const T *a, const T *b, double *error, uint32_t *first_bad) {
  if (!a || !b || !error) return fail(MFP_ERROR_INVALID_VALUE, "null array");
  T num = 0, den = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const T d = a[i] - b[i];
    num += d * d;
    den += b[i] * b[i];
  }
  const T err = num / den;
  *error = (double)err;
  if (first_bad) {
    *first_bad = UINT32_MAX;
    if (err > 1e-9)
      for (uint32_t i = 0; i < n; ++i)
        if (std::abs(a[i] - b[i]) > 1e-8) {
          *first_bad = i;
          break;
        }
  }
  return ok();
}

}  // namespace

extern "C" {

int mfp_csr_from_coo_f32(uint32_t rows, uint32_t cols, uint32_t nnz, int scheme, const uint32_t *ri,
                         const uint32_t *ci, const double *v, uint32_t *rp, uint32_t *c, float *d) {
  return csr_from_coo<float>(rows, cols, nnz, scheme, ri, ci, v, rp, c, d);
}
int mfp_csr_from_coo_f64(uint32_t rows, uint32_t cols, uint32_t nnz, int scheme, const uint32_t *ri,
                         const uint32_t *ci, const double *v, uint32_t *rp, uint32_t *c, double *d) {
  return csr_from_coo<double>(rows, cols, nnz, scheme, ri, ci, v, rp, c, d);
}

// get_rows_statistics — matrix_converter.cpp:95-127.
int mfp_get_rows_statistics(uint32_t rows, const uint32_t *rp, mfp_rows_statistic *out) {
  if (!rp || !out) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  if (rows == 0) return fail(MFP_ERROR_INVALID_VALUE, "rows == 0");
  mfp_rows_statistic s{};
  s.min_elements_in_rows = std::numeric_limits<unsigned int>::max() - 1;
  uint32_t sum = 0;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t n = rp[r + 1] - rp[r];
    if (n > s.max_elements_in_rows) s.max_elements_in_rows = n;
    if (n < s.min_elements_in_rows) s.min_elements_in_rows = n;
    sum += n;
  }
  s.avg_elements_in_rows = sum / rows;
  double acc = 0.0;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t n = rp[r + 1] - rp[r];
    acc += std::pow(static_cast<double>(n) - s.avg_elements_in_rows, 2);
  }
  s.elements_in_rows_std_deviation = std::sqrt(acc / rows);
  *out = s;
  return ok();
}

int mfp_ell_width(uint32_t rows, const uint32_t *rp, uint32_t *width) {
  if (!rp || !width) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  uint32_t w = 0;
  for (uint32_t r = 0; r < rows; ++r) w = std::max(w, rp[r + 1] - rp[r]);
  *width = w;
  return ok();
}

int mfp_ell_from_csr_f32(uint32_t rows, const uint32_t *rp, const uint32_t *c, const float *d,
                         uint32_t width, float *ed, uint32_t *ec) {
  return ell_from_csr<float>(rows, rp, c, d, width, ed, ec);
}
int mfp_ell_from_csr_f64(uint32_t rows, const uint32_t *rp, const uint32_t *c, const double *d,
                         uint32_t width, double *ed, uint32_t *ec) {
  return ell_from_csr<double>(rows, rp, c, d, width, ed, ec);
}

int mfp_coo_count(uint32_t rows, const uint32_t *rp, uint32_t start, uint32_t *count) {
  if (!rp || !count) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  uint64_t n = 0;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t len = rp[r + 1] - rp[r];
    if (len > start) n += len - start;
  }
  *count = (uint32_t)n;
  return ok();
}

int mfp_coo_from_csr_f32(uint32_t rows, const uint32_t *rp, const uint32_t *c, const float *d,
                         uint32_t start, float *cd, uint32_t *cc, uint32_t *cr) {
  return coo_from_csr<float>(rows, rp, c, d, start, cd, cc, cr);
}
int mfp_coo_from_csr_f64(uint32_t rows, const uint32_t *rp, const uint32_t *c, const double *d,
                         uint32_t start, double *cd, uint32_t *cc, uint32_t *cr) {
  return coo_from_csr<double>(rows, rp, c, d, start, cd, cc, cr);
}

// hybrid_matrix_class<T>::allocate — matrix_converter.cpp:288-310.
int mfp_hybrid_width(uint32_t rows, const uint32_t *rp, double percent, uint32_t *width) {
  if (!width) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  mfp_rows_statistic s;
  const int st = mfp_get_rows_statistics(rows, rp, &s);
  if (st) return st;
  const unsigned int w = s.avg_elements_in_rows + (s.max_elements_in_rows - s.avg_elements_in_rows) * percent;
  *width = w;
  return ok();
}

int mfp_row_length_quantile(uint32_t rows, const uint32_t *rp, double q, uint32_t *width) {
  if (!rp || !width) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  if (rows == 0 || !(q >= 0.0 && q <= 1.0)) return fail(MFP_ERROR_INVALID_VALUE, "bad rows or q");
  std::vector<uint32_t> len(rows);
  for (uint32_t r = 0; r < rows; ++r) len[r] = rp[r + 1] - rp[r];
  // smallest length L with at least q*rows rows of length <= L
  uint64_t k = (uint64_t)std::ceil(q * (double)rows);
  if (k == 0) k = 1;
  std::nth_element(len.begin(), len.begin() + (k - 1), len.end());
  *width = len[k - 1];
  return ok();
}

// calculate_slices_count / calculate_lane_size and the constructor's
// initialisers — scoo_matrix_class.cpp:30-66.
int mfp_scoo_params_compute(uint32_t rows, uint32_t sm_count, uint64_t smem, int value_type,
                            mfp_scoo_params *out) {
  if (!out || sm_count == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad argument");
  if (value_type != MFP_F32 && value_type != MFP_F64) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  const unsigned long vs = value_type == MFP_F64 ? 8ul : 4ul;
  const unsigned int max_rows_per_block = std::min(512ul, (unsigned long)(smem / vs));
  unsigned int mult = 1;
  while (max_rows_per_block < (rows / (sm_count * mult))) mult++;
  const unsigned int slices = sm_count * mult;
  const unsigned int slice_size = (rows + slices - 1) / slices;
  unsigned int lane = 0;
  if (slice_size) {
    lane = prev_pow2(std::min(slices, prev_pow2((unsigned int)(smem / (slice_size * vs)))));
    while (slice_size * lane > 1024) lane /= 2;
  }
  out->slices_count = slices;
  out->slice_size = slice_size;
  out->lane_size = lane ? lane : 1;
  return ok();
}

int mfp_scoo_from_csr_f32(uint32_t rows, const uint32_t *rp, const uint32_t *c, const float *d,
                          const mfp_scoo_params *p, float *v, uint32_t *ci, uint32_t *ri, uint32_t *sp) {
  return scoo_from_csr<float>(rows, rp, c, d, p, v, ci, ri, sp);
}
int mfp_scoo_from_csr_f64(uint32_t rows, const uint32_t *rp, const uint32_t *c, const double *d,
                          const mfp_scoo_params *p, double *v, uint32_t *ci, uint32_t *ri, uint32_t *sp) {
  return scoo_from_csr<double>(rows, rp, c, d, p, v, ci, ri, sp);
}

int mfp_scoo_sort_cols_f32(uint32_t slices, const uint32_t *sp, float *v, uint32_t *ci, uint32_t *ri) {
  return scoo_sort_cols<float>(slices, sp, v, ci, ri);
}
int mfp_scoo_sort_cols_f64(uint32_t slices, const uint32_t *sp, double *v, uint32_t *ci, uint32_t *ri) {
  return scoo_sort_cols<double>(slices, sp, v, ci, ri);
}

// fill_row_blocks — csr_adaptive_spmv.cu:180-240: close a bin when its
// elements reach nnz_per_wg exactly; on overflow step back one row unless the
// bin holds a single row; cap a bin at nnz_per_wg rows.
int mfp_csr_adaptive_row_blocks(uint32_t rows, const uint32_t *rp, uint32_t per_wg, uint32_t *blocks,
                                uint32_t *count) {
  if (!rp || !count || per_wg == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad argument");
  if (blocks) blocks[0] = 0;
  int64_t last = 0;
  uint32_t wg = 1;
  uint32_t sum = 0;
  for (int64_t i = 1; i <= (int64_t)rows; ++i) {
    sum += rp[i] - rp[i - 1];
    if (sum == per_wg) {
      last = i;
      if (blocks) blocks[wg] = (uint32_t)i;
      ++wg;
      sum = 0;
    } else if (sum > per_wg) {
      if (i - last > 1) {
        if (blocks) blocks[wg] = (uint32_t)(i - 1);
        ++wg;
        --i;
      } else {
        if (blocks) blocks[wg] = (uint32_t)i;
        ++wg;
      }
      last = i;
      sum = 0;
    } else if ((uint64_t)(i - last) > per_wg) {
      last = i;
      if (blocks) blocks[wg] = (uint32_t)i;
      ++wg;
      sum = 0;
    }
  }
  if (blocks) blocks[wg] = rows;
  *count = wg;
  return ok();
}

// measurement_class::measurement_class — measurement_class.cpp:7-16.
int mfp_measurement_make(const char *format, double elapsed, double bytes, double ops,
                         mfp_measurement *out) {
  if (!format || !out) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  std::memset(out, 0, sizeof(*out));
  std::strncpy(out->format, format, sizeof(out->format) - 1);
  const size_t giga = 1E+9;
  out->elapsed = elapsed;
  out->effective_bandwidth = bytes / (elapsed * giga);
  out->computational_throughput = ops / (elapsed * giga);
  return ok();
}

// compare_results — measurement_class.h:60-89 (without the printing).
int mfp_compare_results_f32(uint32_t n, const float *a, const float *b, double *e, uint32_t *fb) {
  return compare<float>(n, a, b, e, fb);
}
int mfp_compare_results_f64(uint32_t n, const double *a, const double *b, double *e, uint32_t *fb) {
  return compare<double>(n, a, b, e, fb);
}

// ---- reduced-precision CSR (engine extension) ------------------------------
static uint16_t to_bf16_rne(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}
static uint16_t to_fp16(float f) {
  const _Float16 h = (_Float16)f;  // round-to-nearest-even
  uint16_t u;
  std::memcpy(&u, &h, 2);
  return u;
}

int mfp_lowp_quantize(int vt, uint32_t rows, const uint32_t *rp, const double *v, uint16_t *q, float *scale) {
  if (vt != MFP_BF16 && vt != MFP_F16) return fail(MFP_ERROR_INVALID_VALUE, "value type must be BF16 or F16");
  if (!rp || !scale) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const uint32_t nnz = rp[rows];
  if (nnz && (!v || !q)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  for (uint32_t r = 0; r < rows; ++r) {
    double mx = 0.0;
    for (uint32_t e = rp[r]; e < rp[r + 1]; ++e) mx = std::max(mx, std::fabs(v[e]));
    const float s = mx > 0.0 ? (float)mx : 1.0f;
    scale[r] = s;
    for (uint32_t e = rp[r]; e < rp[r + 1]; ++e) {
      const float f = (float)(v[e] / (double)s);
      q[e] = vt == MFP_BF16 ? to_bf16_rne(f) : to_fp16(f);
    }
  }
  return ok();
}

int mfp_lowp_deltas(uint32_t nnz, const uint32_t *c, uint16_t *delta, uint32_t *base) {
  if (nnz && (!c || !delta || !base)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const uint32_t chunks = (uint32_t)(((uint64_t)nnz + MFP_LOWP_DELTA_CHUNK - 1) / MFP_LOWP_DELTA_CHUNK);
  for (uint32_t k = 0; k < chunks; ++k) {
    const uint32_t b = k * MFP_LOWP_DELTA_CHUNK, e = (uint32_t)std::min<uint64_t>(nnz, (uint64_t)b + MFP_LOWP_DELTA_CHUNK);
    uint32_t lo = UINT32_MAX, hi = 0;
    for (uint32_t i = b; i < e; ++i) {
      lo = std::min(lo, c[i]);
      hi = std::max(hi, c[i]);
    }
    if (hi - lo > 65535u)
      return fail(MFP_ERROR_NOT_SUPPORTED, "16-bit deltas: columns of chunk %u span %u > 65535", k, hi - lo);
    base[k] = lo;
    for (uint32_t i = b; i < e; ++i) delta[i] = (uint16_t)(c[i] - lo);
  }
  return ok();
}

int mfp_lowp_ell_from_csr(int vt, int index16, uint32_t rows, uint32_t cols, const uint32_t *rp, const uint32_t *ci,
                          const double *v, uint32_t width, uint16_t *q, void *idx, float *scale) {
  if (vt != MFP_BF16 && vt != MFP_F16) return fail(MFP_ERROR_INVALID_VALUE, "value type must be BF16 or F16");
  if (!rp || !scale || ((uint64_t)width * rows != 0 && (!q || !idx))) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const uint32_t nnz = rp[rows];
  if (nnz && (!ci || !v)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  for (uint32_t r = 0; r < rows; ++r)
    if (rp[r + 1] - rp[r] > width) return fail(MFP_ERROR_INVALID_VALUE, "row %u longer than the width %u", r, width);
  std::vector<uint16_t> qc(nnz);
  int st = mfp_lowp_quantize(vt, rows, rp, v, qc.data(), scale);
  if (st) return st;
  uint16_t *off = static_cast<uint16_t *>(idx);
  uint32_t *c32 = static_cast<uint32_t *>(idx);
  const size_t stride = rows;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t b = rp[r], len = rp[r + 1] - b;
    // a padding slot gathers a column its row already reads (or the diagonal)
    const uint32_t pad_col = len ? ci[b + len - 1] : (r < cols ? r : 0u);
    for (uint32_t k = 0; k < width; ++k) {
      const size_t o = (size_t)k * stride + r;
      const uint32_t c = k < len ? ci[b + k] : pad_col;
      q[o] = k < len ? qc[b + k] : uint16_t(0);
      if (index16) {
        const int64_t d = (int64_t)c - (int64_t)r;
        if (d < -32768 || d > 32767)
          return fail(MFP_ERROR_NOT_SUPPORTED, "16-bit column offsets: row %u column %u is %lld away", r, c,
                      (long long)d);
        off[o] = (uint16_t)(d + 32768);
      } else {
        c32[o] = c;
      }
    }
  }
  return ok();
}

// ---- selector features (engine extension) ---------------------------------
int mfp_selector_features(uint32_t rows, uint32_t cols, const uint32_t *rp, const uint32_t *ci, float *f) {
  if (!rp || !f) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const uint32_t nnz = rp[rows];
  if (nnz && !ci) return fail(MFP_ERROR_INVALID_VALUE, "null columns");
  std::vector<uint32_t> len(rows);
  double sum = 0, sq = 0;
  uint32_t mx = 0, empty = 0;
  uint64_t band = 0, near = 0, diag = 0, long_nnz = 0;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t l = rp[r + 1] - rp[r];
    len[r] = l;
    sum += l;
    sq += (double)l * l;
    mx = std::max(mx, l);
    empty += l == 0;
    if (l > 4096) long_nnz += l;
    for (uint32_t e = rp[r]; e < rp[r + 1]; ++e) {
      const uint64_t d = ci[e] > r ? (uint64_t)ci[e] - r : (uint64_t)r - ci[e];
      band = std::max(band, d);
      near += d <= 64;
      diag += d == 0;
    }
  }
  const double mean = rows ? sum / rows : 0.0;
  const double var = rows ? std::max(0.0, sq / rows - mean * mean) : 0.0;
  // Gini coefficient of the row lengths: sum_i (2i - n - 1) x_(i) / (n sum x)
  double gini = 0.0;
  if (rows && sum > 0) {
    std::sort(len.begin(), len.end());
    double acc = 0.0;
    for (uint32_t i = 0; i < rows; ++i) acc += (2.0 * (i + 1) - rows - 1.0) * len[i];
    gini = acc / ((double)rows * sum);
  }
  const double dim = std::max<double>(1.0, std::max(rows, cols));
  f[0] = (float)std::log10(std::max(1u, rows));
  f[1] = (float)std::log10(std::max(1u, cols));
  f[2] = (float)std::log10((double)nnz + 1.0);
  f[3] = (float)std::log2(1.0 + mean);
  f[4] = (float)std::log2(1.0 + std::sqrt(var));
  f[5] = (float)std::log2(1.0 + mx);
  f[6] = (float)gini;
  f[7] = (float)(band / dim);
  f[8] = nnz ? (float)((double)near / nnz) : 0.f;
  f[9] = (float)((double)diag / std::max(1u, std::min(rows, cols)));
  f[10] = rows ? (float)((double)empty / rows) : 0.f;
  f[11] = nnz ? (float)((double)long_nnz / nnz) : 0.f;
  return ok();
}

int mfp_scoo_x_windows(uint32_t nnz, const uint32_t *ci, const uint32_t *sp, uint32_t slices,
                       uint32_t *win) {
  if (!sp || !win || (nnz && !ci)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  for (uint32_t s = 0; s < slices; ++s) {
    const uint32_t b = sp[s], e = sp[s + 1];
    uint32_t lo = 0, hi = 0;
    if (b < e && e <= nnz) {
      lo = UINT32_MAX;
      for (uint32_t k = b; k < e; ++k) {
        lo = std::min(lo, ci[k]);
        hi = std::max(hi, ci[k] + 1u);
      }
    }
    win[2 * s] = lo;
    win[2 * s + 1] = hi;
  }
  return ok();
}

}  // extern "C"
