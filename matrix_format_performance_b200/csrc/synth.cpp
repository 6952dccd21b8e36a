// Seeded synthetic sparse matrices in CSR (sorted columns, double values).
//
// These stand in for the SuiteSparse matrices the reference benchmarks
// (its inputs are not shipped).  Every random draw is a counter-based hash of
// (seed, stream, index), so a matrix is a pure function of its parameters and
// does not depend on the number of host threads used to build it.
#include "host_common.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

using namespace mfp;

namespace {

inline uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t i) {
  return splitmix(splitmix(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ (i * 0x9E3779B97F4A7C15ull));
}
// uniform in [0, 1)
inline double unit(uint64_t seed, uint64_t stream, uint64_t i) {
  return (double)(hash3(seed, stream, i) >> 11) * (1.0 / 9007199254740992.0);
}
inline double sym(uint64_t seed, uint64_t stream, uint64_t i) { return 2.0 * unit(seed, stream, i) - 1.0; }
inline uint64_t below(uint64_t seed, uint64_t stream, uint64_t i, uint64_t n) {
  // multiply-shift range reduction of a 64-bit hash
  return (uint64_t)(((__uint128_t)hash3(seed, stream, i) * n) >> 64);
}

enum : uint64_t { kLen = 1, kCol = 2, kVal = 3, kVec = 4, kColRetry = 5 };

template <typename F>
void parallel_rows(uint32_t rows, F f) {
  unsigned nt = std::max(1u, std::thread::hardware_concurrency());
  nt = std::min<unsigned>(nt, 64u);
  if (rows < 4096 || nt == 1) {
    f(0u, rows);
    return;
  }
  std::vector<std::thread> th;
  const uint32_t step = (rows + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const uint32_t b = std::min<uint64_t>((uint64_t)t * step, rows), e = std::min<uint64_t>((uint64_t)(t + 1) * step, rows);
    if (b < e) th.emplace_back(f, b, e);
  }
  for (auto &t : th) t.join();
}

// k distinct sorted integers from [lo, lo + w): Floyd's sampling.
void sample_distinct(uint64_t seed, uint64_t key, uint32_t lo, uint32_t w, uint32_t k,
                     std::vector<uint32_t> &out) {
  out.clear();
  if (k >= w) {
    for (uint32_t i = 0; i < w; ++i) out.push_back(lo + i);
    return;
  }
  if ((uint64_t)k * 16 < w) {
    // sparse case: draw, sort, redraw duplicates with fresh counters
    uint64_t ctr = 0;
    while (out.size() < k) {
      while (out.size() < k) out.push_back(lo + (uint32_t)below(seed, kColRetry, key * 4294967296ull + ctr++, w));
      std::sort(out.begin(), out.end());
      out.erase(std::unique(out.begin(), out.end()), out.end());
    }
    return;
  }
  std::vector<uint64_t> bits((w + 63) / 64, 0);
  for (uint32_t j = w - k; j < w; ++j) {
    const uint32_t t = (uint32_t)below(seed, kCol, key * 4294967296ull + j, (uint64_t)j + 1);
    if (bits[t >> 6] >> (t & 63) & 1ull)
      bits[j >> 6] |= 1ull << (j & 63);
    else
      bits[t >> 6] |= 1ull << (t & 63);
  }
  for (uint32_t i = 0; i < w; ++i)
    if (bits[i >> 6] >> (i & 63) & 1ull) out.push_back(lo + i);
}

double zeta(double a) {
  // sum to 1e6 plus the Euler-Maclaurin tail
  double s = 0.0;
  const double N = 1e6;
  for (double k = N; k >= 1.0; k -= 1.0) s += std::pow(k, -a);
  s += std::pow(N, 1.0 - a) / (a - 1.0) - 0.5 * std::pow(N, -a);
  return s;
}

struct builder {
  uint32_t rows = 0, cols = 0;
  std::vector<uint32_t> len;  // per row
};

int finish(const builder &b, uint32_t *rows, uint32_t *cols, uint64_t *nnz, uint32_t *rp) {
  uint64_t n = 0;
  for (uint32_t r = 0; r < b.rows; ++r) n += b.len[r];
  if (n > 0xffffffffull) return fail(MFP_ERROR_TOO_LARGE, "nnz %llu exceeds 32-bit indexing", (unsigned long long)n);
  *rows = b.rows;
  *cols = b.cols;
  *nnz = n;
  if (rp) {
    uint32_t acc = 0;
    for (uint32_t r = 0; r < b.rows; ++r) {
      rp[r] = acc;
      acc += b.len[r];
    }
    rp[b.rows] = acc;
  }
  return MFP_SUCCESS;
}

}  // namespace

extern "C" int mfp_synth_csr(const mfp_synth_params *p, uint32_t *rows, uint32_t *cols, uint64_t *nnz,
                             uint32_t *rp, uint32_t *ci, double *vals) {
  if (!p || !rows || !cols || !nnz) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const bool fill = rp != nullptr;
  if (fill && (!ci || !vals)) return fail(MFP_ERROR_INVALID_VALUE, "row_ptr given without columns/values");
  const uint64_t seed = p->seed;
  builder b;
  switch (p->kind) {
    case MFP_SYNTH_LAPLACIAN_2D: {
      const uint64_t n = p->n;
      if (n == 0 || n * n > 0xffffffffull) return fail(MFP_ERROR_INVALID_VALUE, "bad grid size");
      b.rows = b.cols = (uint32_t)(n * n);
      b.len.resize(b.rows);
      for (uint64_t i = 0; i < n; ++i)
        for (uint64_t j = 0; j < n; ++j) b.len[i * n + j] = 1 + (i > 0) + (i + 1 < n) + (j > 0) + (j + 1 < n);
      int st = finish(b, rows, cols, nnz, rp);
      if (st || !fill) return st;
      parallel_rows(b.rows, [&](uint32_t r0, uint32_t r1) {
        for (uint32_t r = r0; r < r1; ++r) {
          const uint64_t i = r / n, j = r % n;
          uint32_t k = rp[r];
          if (i > 0) { ci[k] = r - (uint32_t)n; vals[k++] = -1.0; }
          if (j > 0) { ci[k] = r - 1; vals[k++] = -1.0; }
          ci[k] = r; vals[k++] = 4.0;
          if (j + 1 < n) { ci[k] = r + 1; vals[k++] = -1.0; }
          if (i + 1 < n) { ci[k] = r + (uint32_t)n; vals[k++] = -1.0; }
        }
      });
      return ok();
    }
    case MFP_SYNTH_STENCIL_27: {
      const uint64_t n = p->n;
      if (n == 0 || n * n * n > 0xffffffffull) return fail(MFP_ERROR_INVALID_VALUE, "bad grid size");
      b.rows = b.cols = (uint32_t)(n * n * n);
      b.len.resize(b.rows);
      for (uint64_t r = 0; r < b.rows; ++r) {
        const uint64_t i = r / (n * n), j = (r / n) % n, k = r % n;
        const uint32_t a = 1 + (i > 0) + (i + 1 < n), c = 1 + (j > 0) + (j + 1 < n), d = 1 + (k > 0) + (k + 1 < n);
        b.len[r] = a * c * d;
      }
      int st = finish(b, rows, cols, nnz, rp);
      if (st || !fill) return st;
      parallel_rows(b.rows, [&](uint32_t r0, uint32_t r1) {
        for (uint32_t r = r0; r < r1; ++r) {
          const int64_t i = r / (n * n), j = (r / n) % n, k = r % n;
          uint32_t at = rp[r], local = 0;
          for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
              for (int dk = -1; dk <= 1; ++dk) {
                const int64_t ii = i + di, jj = j + dj, kk = k + dk;
                if (ii < 0 || jj < 0 || kk < 0 || ii >= (int64_t)n || jj >= (int64_t)n || kk >= (int64_t)n) continue;
                ci[at] = (uint32_t)((ii * (int64_t)n + jj) * (int64_t)n + kk);
                vals[at++] = sym(seed, kVal, (uint64_t)r * 32 + local++);
              }
        }
      });
      return ok();
    }
    case MFP_SYNTH_BANDED: {
      const uint32_t n = p->n, bw = p->band, k = p->k_lo;
      if (n == 0 || k == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad banded parameters");
      b.rows = b.cols = n;
      b.len.resize(n);
      for (uint32_t r = 0; r < n; ++r) {
        const uint32_t lo = r > bw ? r - bw : 0, hi = (uint64_t)r + bw < n ? r + bw : n - 1;
        b.len[r] = std::min(k, hi - lo + 1);
      }
      int st = finish(b, rows, cols, nnz, rp);
      if (st || !fill) return st;
      parallel_rows(n, [&](uint32_t r0, uint32_t r1) {
        std::vector<uint32_t> tmp;
        for (uint32_t r = r0; r < r1; ++r) {
          const uint32_t lo = r > bw ? r - bw : 0, hi = (uint64_t)r + bw < n ? r + bw : n - 1;
          sample_distinct(seed, r, lo, hi - lo + 1, k, tmp);
          uint32_t at = rp[r];
          for (uint32_t q = 0; q < tmp.size(); ++q) {
            ci[at] = tmp[q];
            vals[at++] = sym(seed, kVal, (uint64_t)r * 65536 + q);
          }
        }
      });
      return ok();
    }
    case MFP_SYNTH_POWER_LAW:
    case MFP_SYNTH_UNIFORM: {
      const uint32_t n = p->n, c = p->cols ? p->cols : p->n;
      const uint32_t klo = std::max(1u, p->k_lo), khi = std::max(klo, p->k_hi);
      if (n == 0 || c == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad size");
      b.rows = n;
      b.cols = c;
      b.len.resize(n);
      if (p->kind == MFP_SYNTH_POWER_LAW) {
        // Zipf(alpha) on k >= 1 (P(k) = k^-alpha / zeta(alpha)), clipped to [klo, khi].
        if (!(p->alpha > 1.0)) return fail(MFP_ERROR_INVALID_VALUE, "alpha must exceed 1");
        const double z = zeta(p->alpha);
        std::vector<double> cdf(khi);
        double acc = 0.0;
        for (uint32_t k = 1; k <= khi; ++k) {
          acc += std::pow((double)k, -p->alpha) / z;
          cdf[k - 1] = acc;
        }
        parallel_rows(n, [&](uint32_t r0, uint32_t r1) {
          for (uint32_t r = r0; r < r1; ++r) {
            const double u = unit(seed, kLen, r);
            const uint32_t k = (uint32_t)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) + 1;  // khi+1 past the table
            b.len[r] = std::min(std::max(k, klo), std::min(khi, c));
          }
        });
      } else {
        parallel_rows(n, [&](uint32_t r0, uint32_t r1) {
          for (uint32_t r = r0; r < r1; ++r)
            b.len[r] = std::min<uint32_t>(c, klo + (uint32_t)below(seed, kLen, r, (uint64_t)(khi - klo + 1)));
        });
      }
      int st = finish(b, rows, cols, nnz, rp);
      if (st || !fill) return st;
      parallel_rows(n, [&](uint32_t r0, uint32_t r1) {
        std::vector<uint32_t> tmp;
        for (uint32_t r = r0; r < r1; ++r) {
          sample_distinct(seed, r, 0, c, b.len[r], tmp);
          uint32_t at = rp[r];
          for (uint32_t q = 0; q < tmp.size(); ++q) {
            ci[at] = tmp[q];
            vals[at++] = sym(seed, kVal, (uint64_t)r * 65536 + q);
          }
        }
      });
      return ok();
    }
    case MFP_SYNTH_TRIDIAGONAL: {
      const uint32_t n = p->n;
      if (n == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad size");
      b.rows = b.cols = n;
      b.len.resize(n);
      for (uint32_t r = 0; r < n; ++r) b.len[r] = 1 + (r > 0) + (r + 1 < n);
      int st = finish(b, rows, cols, nnz, rp);
      if (st || !fill) return st;
      for (uint32_t r = 0; r < n; ++r) {
        uint32_t at = rp[r], q = 0;
        for (int d = -1; d <= 1; ++d) {
          const int64_t cc = (int64_t)r + d;
          if (cc < 0 || cc >= n) continue;
          ci[at] = (uint32_t)cc;
          vals[at++] = sym(seed, kVal, (uint64_t)r * 65536 + q++);
        }
      }
      return ok();
    }
    case MFP_SYNTH_BLOCK_DIAGONAL: {
      const uint32_t n = p->n, bs = std::max(1u, p->band);
      if (n == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad size");
      b.rows = b.cols = n;
      b.len.resize(n);
      for (uint32_t r = 0; r < n; ++r) {
        const uint32_t q0 = (r / bs) * bs;
        b.len[r] = std::min(n, q0 + bs) - q0;
      }
      int st = finish(b, rows, cols, nnz, rp);
      if (st || !fill) return st;
      parallel_rows(n, [&](uint32_t r0, uint32_t r1) {
        for (uint32_t r = r0; r < r1; ++r) {
          const uint32_t q0 = (r / bs) * bs, q1 = std::min(n, q0 + bs);
          uint32_t at = rp[r];
          for (uint32_t cc = q0; cc < q1; ++cc) {
            ci[at] = cc;
            vals[at++] = sym(seed, kVal, (uint64_t)r * 65536 + (cc - q0));
          }
        }
      });
      return ok();
    }
    default:
      return fail(MFP_ERROR_INVALID_VALUE, "unknown synthetic kind %d", p->kind);
  }
}

extern "C" int mfp_synth_vector_f64(uint64_t seed, uint64_t n, double lo, double hi, double *out) {
  if (!out && n) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  for (uint64_t i = 0; i < n; ++i) out[i] = lo + (hi - lo) * unit(seed, kVec, i);
  return ok();
}
