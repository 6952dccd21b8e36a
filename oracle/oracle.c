/*
 * ORACLE — test infrastructure only.  Nothing in the engine links or calls
 * this file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it, as the checker.
 *
 * A plain-C restatement of the reference's CPU SpMV path and of its format
 * converters (gevtushenko/matrix_format_performance), each function citing the
 * lines it follows.  It is pinned against the reference itself: the tests
 * compare it element for element with the reference's own sources compiled
 * into oracle/_ref/ (recipe: oracle/Makefile) and with the fixtures in
 * tests/golden/ that those sources produced.
 *
 * Build with -ffp-contract=off: products and sums are rounded separately, as
 * in the reference loop compiled without contraction.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ---- SpMV -------------------------------------------------------------- */

/* cpu_csr_spmv_single_thread_naive — cpu/cpu_matrix_multiplier.cpp:20-61,
 * with an explicit x instead of x := 1 (the reference fills x with 1.0). */
void oracle_csr_spmv_f32(uint32_t rows, const uint32_t *rp, const uint32_t *ci, const float *a,
                         const float *x, float *y) {
  for (uint32_t r = 0; r < rows; ++r) {
    float dot = 0;
    for (uint32_t e = rp[r]; e < rp[r + 1]; ++e) dot += a[e] * x[ci[e]];
    y[r] = dot;
  }
}
void oracle_csr_spmv_f64(uint32_t rows, const uint32_t *rp, const uint32_t *ci, const double *a,
                         const double *x, double *y) {
  for (uint32_t r = 0; r < rows; ++r) {
    double dot = 0;
    for (uint32_t e = rp[r]; e < rp[r + 1]; ++e) dot += a[e] * x[ci[e]];
    y[r] = dot;
  }
}

/* cpu_csr_spmv_single_thread_naive_with_reduce_order —
 * cpu_matrix_multiplier.cpp:170-227: 32 lane-strided partial sums, then the
 * shuffle-down tree 16, 8, 4, 2, 1 of lane 0. */
#define REDUCE_ORDER(T, NAME)                                                                  \
  void NAME(uint32_t rows, const uint32_t *rp, const uint32_t *ci, const T *a, const T *x, T *y) { \
    T dots[32];                                                                                \
    for (uint32_t r = 0; r < rows; ++r) {                                                      \
      for (uint32_t lane = 0; lane < 32; ++lane) {                                             \
        dots[lane] = 0;                                                                        \
        for (uint32_t e = rp[r] + lane; e < rp[r + 1]; e += 32) dots[lane] += a[e] * x[ci[e]]; \
      }                                                                                        \
      for (int off = 16; off > 0; off /= 2)                                                    \
        for (uint32_t lane = 0; lane < 16; ++lane) dots[lane] += dots[lane + off];             \
      y[r] = dots[0];                                                                          \
    }                                                                                          \
  }
REDUCE_ORDER(float, oracle_csr_spmv_reduce_order_f32)
REDUCE_ORDER(double, oracle_csr_spmv_reduce_order_f64)

/* ELL loop — cpu_matrix_multiplier.cpp:310-331 (and the GPU kernel
 * gpu_matrix_multiplier.cu:450-471): slots 0..width-1 in order. */
void oracle_ell_spmv_f32(uint32_t rows, uint32_t width, const float *a, const uint32_t *ci, const float *x,
                         float *y) {
  for (uint32_t r = 0; r < rows; ++r) {
    float dot = 0;
    for (uint32_t k = 0; k < width; ++k) dot += a[(size_t)k * rows + r] * x[ci[(size_t)k * rows + r]];
    y[r] = dot;
  }
}
void oracle_ell_spmv_f64(uint32_t rows, uint32_t width, const double *a, const uint32_t *ci, const double *x,
                         double *y) {
  for (uint32_t r = 0; r < rows; ++r) {
    double dot = 0;
    for (uint32_t k = 0; k < width; ++k) dot += a[(size_t)k * rows + r] * x[ci[(size_t)k * rows + r]];
    y[r] = dot;
  }
}

/* Extended-precision reference used for tolerances: y[r] in long double and
 * absrow[r] = sum |a_re * x_c|, the scale a per-row error is measured in. */
void oracle_csr_spmv_ld(uint32_t rows, const uint32_t *rp, const uint32_t *ci, const double *a, const double *x,
                        double *y, double *absrow) {
  for (uint32_t r = 0; r < rows; ++r) {
    long double s = 0, t = 0;
    for (uint32_t e = rp[r]; e < rp[r + 1]; ++e) {
      const long double p = (long double)a[e] * (long double)x[ci[e]];
      s += p;
      t += p < 0 ? -p : p;
    }
    y[r] = (double)s;
    if (absrow) absrow[r] = (double)t;
  }
}

/* cpu_csr_spmv_multi_thread_naive — cpu_matrix_multiplier.cpp:229-308,
 * restated: the same contiguous row split (rows / threads per thread, the
 * last takes the rest), threads released together, elapsed = the slowest
 * thread.  (The reference helper at :229-249 lacks its return statement and
 * cannot be called safely.) */
struct par_job {
  uint32_t b, e;
  const uint32_t *rp, *ci;
  const void *a, *x;
  void *y;
  int f64;
  volatile int *go;
  double seconds;
};
static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
static void *par_worker(void *p) {
  struct par_job *j = (struct par_job *)p;
  while (!*j->go) {
  }
  const double t0 = now_s();
  if (j->f64) {
    const double *a = (const double *)j->a, *x = (const double *)j->x;
    double *y = (double *)j->y;
    for (uint32_t r = j->b; r < j->e; ++r) {
      double dot = 0;
      for (uint32_t k = j->rp[r]; k < j->rp[r + 1]; ++k) dot += a[k] * x[j->ci[k]];
      y[r] = dot;
    }
  } else {
    const float *a = (const float *)j->a, *x = (const float *)j->x;
    float *y = (float *)j->y;
    for (uint32_t r = j->b; r < j->e; ++r) {
      float dot = 0;
      for (uint32_t k = j->rp[r]; k < j->rp[r + 1]; ++k) dot += a[k] * x[j->ci[k]];
      y[r] = dot;
    }
  }
  j->seconds = now_s() - t0;
  return NULL;
}
double oracle_csr_spmv_parallel(uint32_t threads, int f64, uint32_t rows, const uint32_t *rp, const uint32_t *ci,
                                const void *a, const void *x, void *y) {
  if (threads == 0) threads = 1;
  struct par_job *jobs = (struct par_job *)calloc(threads, sizeof(struct par_job));
  pthread_t *th = (pthread_t *)calloc(threads, sizeof(pthread_t));
  volatile int go = 0;
  const uint32_t per = rows / threads;
  for (uint32_t t = 0; t < threads; ++t) {
    jobs[t].b = per * t;
    jobs[t].e = t == threads - 1 ? rows : (t + 1) * per;
    jobs[t].rp = rp;
    jobs[t].ci = ci;
    jobs[t].a = a;
    jobs[t].x = x;
    jobs[t].y = y;
    jobs[t].f64 = f64;
    jobs[t].go = &go;
    pthread_create(&th[t], NULL, par_worker, &jobs[t]);
  }
  __sync_synchronize();
  go = 1;
  double mx = 0;
  for (uint32_t t = 0; t < threads; ++t) {
    pthread_join(th[t], NULL);
    if (jobs[t].seconds > mx) mx = jobs[t].seconds;
  }
  free(jobs);
  free(th);
  return mx;
}

/* ---- format converters ------------------------------------------------- */

struct colpos {
  uint32_t col, pos;
};
static int colpos_cmp(const void *l, const void *r) {
  const struct colpos *a = (const struct colpos *)l, *b = (const struct colpos *)r;
  if (a->col != b->col) return a->col < b->col ? -1 : 1;
  return a->pos < b->pos ? -1 : (a->pos > b->pos);
}

/* csr_matrix_class<T>(matrix_class) — common/matrix_converter.cpp:15-87. */
#define CSR_FROM_COO(T, NAME)                                                                           \
  int NAME(uint32_t rows, uint32_t nnz, const uint32_t *ri, const uint32_t *ci, const double *v, uint32_t *rp, \
           uint32_t *cols, T *data) {                                                                   \
    memset(rp, 0, sizeof(uint32_t) * ((size_t)rows + 1));                                               \
    for (uint32_t i = 0; i < nnz; ++i) rp[ri[i]]++;                                                     \
    uint32_t acc = 0;                                                                                   \
    for (uint32_t r = 0; r <= rows; ++r) {                                                              \
      const uint32_t c = rp[r];                                                                         \
      rp[r] = acc;                                                                                      \
      acc += c;                                                                                         \
    }                                                                                                   \
    uint32_t *fill = (uint32_t *)calloc(rows ? rows : 1, sizeof(uint32_t));                             \
    for (uint32_t i = 0; i < nnz; ++i) {                                                                \
      const uint32_t at = rp[ri[i]] + fill[ri[i]]++;                                                    \
      data[at] = (T)v[i];                                                                               \
      cols[at] = ci[i];                                                                                 \
    }                                                                                                   \
    free(fill);                                                                                         \
    for (uint32_t r = 0; r < rows; ++r) {                                                               \
      const uint32_t b = rp[r], n = rp[r + 1] - rp[r];                                                  \
      if (n < 2) continue;                                                                              \
      struct colpos *cp = (struct colpos *)malloc(sizeof(struct colpos) * n);                           \
      T *tv = (T *)malloc(sizeof(T) * n);                                                               \
      for (uint32_t k = 0; k < n; ++k) {                                                                \
        cp[k].col = cols[b + k];                                                                        \
        cp[k].pos = k;                                                                                  \
        tv[k] = data[b + k];                                                                            \
      }                                                                                                 \
      qsort(cp, n, sizeof(struct colpos), colpos_cmp);                                                  \
      for (uint32_t k = 0; k < n; ++k) {                                                                \
        cols[b + k] = cp[k].col;                                                                        \
        data[b + k] = tv[cp[k].pos];                                                                    \
      }                                                                                                 \
      free(cp);                                                                                         \
      free(tv);                                                                                         \
    }                                                                                                   \
    return 0;                                                                                           \
  }
CSR_FROM_COO(float, oracle_csr_from_coo_f32)
CSR_FROM_COO(double, oracle_csr_from_coo_f64)

/* get_rows_statistics — matrix_converter.cpp:95-127. out = {min, max, avg}. */
void oracle_rows_statistics(uint32_t rows, const uint32_t *rp, uint32_t *out, double *std_dev) {
  uint32_t mn = 0xffffffffu - 1u, mx = 0, sum = 0;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t n = rp[r + 1] - rp[r];
    if (n > mx) mx = n;
    if (n < mn) mn = n;
    sum += n;
  }
  const uint32_t avg = sum / rows;
  double acc = 0.0;
  for (uint32_t r = 0; r < rows; ++r) acc += pow((double)(rp[r + 1] - rp[r]) - avg, 2);
  out[0] = mn;
  out[1] = mx;
  out[2] = avg;
  *std_dev = sqrt(acc / rows);
}

/* ell_matrix_class — matrix_converter.cpp:139-203 (width given). */
#define ELL_FROM_CSR(T, NAME)                                                                              \
  void NAME(uint32_t rows, const uint32_t *rp, const uint32_t *cols, const T *data, uint32_t width, T *ed,  \
            uint32_t *ec) {                                                                                \
    const size_t n = (size_t)rows * width;                                                                 \
    for (size_t i = 0; i < n; ++i) {                                                                       \
      ed[i] = 0;                                                                                           \
      ec[i] = 0;                                                                                           \
    }                                                                                                      \
    for (uint32_t r = 0; r < rows; ++r)                                                                    \
      for (uint32_t k = rp[r]; k < rp[r + 1] && k - rp[r] < width; ++k) {                                 \
        ed[(size_t)(k - rp[r]) * rows + r] = data[k];                                                      \
        ec[(size_t)(k - rp[r]) * rows + r] = cols[k];                                                      \
      }                                                                                                    \
  }
ELL_FROM_CSR(float, oracle_ell_from_csr_f32)
ELL_FROM_CSR(double, oracle_ell_from_csr_f64)

/* coo_matrix_class — matrix_converter.cpp:211-280; returns the element count. */
#define COO_FROM_CSR(T, NAME)                                                                              \
  uint32_t NAME(uint32_t rows, const uint32_t *rp, const uint32_t *cols, const T *data, uint32_t start,     \
                T *cd, uint32_t *cc, uint32_t *cr) {                                                       \
    uint32_t id = 0;                                                                                       \
    for (uint32_t r = 0; r < rows; ++r)                                                                    \
      for (uint32_t k = rp[r]; k < rp[r + 1]; ++k)                                                         \
        if (k - rp[r] >= start) {                                                                          \
          if (cd) {                                                                                        \
            cd[id] = data[k];                                                                              \
            cc[id] = cols[k];                                                                              \
            cr[id] = r;                                                                                    \
          }                                                                                                \
          ++id;                                                                                            \
        }                                                                                                  \
    return id;                                                                                             \
  }
COO_FROM_CSR(float, oracle_coo_from_csr_f32)
COO_FROM_CSR(double, oracle_coo_from_csr_f64)

/* hybrid_matrix_class::allocate width — matrix_converter.cpp:296-302. */
uint32_t oracle_hybrid_width(uint32_t rows, const uint32_t *rp, double percent) {
  uint32_t s[3];
  double sd;
  oracle_rows_statistics(rows, rp, s, &sd);
  const unsigned int w = s[2] + (s[1] - s[2]) * percent;
  return w;
}

/* next_pow_2 / prev_pow_2 / calculate_slices_count / calculate_lane_size —
 * common/scoo_matrix_class.cpp:13-56.  out = {slices_count, slice_size, lane_size}. */
static uint32_t np2(uint32_t x) {
  --x;
  x |= x >> 1u;
  x |= x >> 2u;
  x |= x >> 4u;
  x |= x >> 8u;
  x |= x >> 16u;
  return ++x;
}
static uint32_t pp2(uint32_t x) {
  const uint32_t n = np2(x);
  return n > x ? n / 2 : n;
}
void oracle_scoo_params(uint32_t rows, uint32_t sm_count, uint64_t smem, uint32_t value_size, uint32_t *out) {
  const uint64_t q = smem / value_size;
  const uint32_t max_rows = (uint32_t)(q < 512 ? q : 512);
  uint32_t mult = 1;
  while (max_rows < rows / (sm_count * mult)) mult++;
  const uint32_t slices = sm_count * mult;
  const uint32_t slice = (rows + slices - 1) / slices;
  uint32_t lane = 0;
  if (slice) {
    const uint32_t a = pp2((uint32_t)(smem / ((uint64_t)slice * value_size)));
    lane = pp2(slices < a ? slices : a);
    while (slice * lane > 1024) lane /= 2;
  }
  out[0] = slices;
  out[1] = slice;
  out[2] = lane ? lane : 1;
}

/* scoo_matrix_class constructor body — scoo_matrix_class.cpp:58-101. */
#define SCOO_FROM_CSR(T, NAME)                                                                              \
  void NAME(uint32_t rows, const uint32_t *rp, const uint32_t *cols, const T *data, uint32_t slices,         \
            uint32_t slice_size, T *v, uint32_t *ci, uint32_t *ri, uint32_t *sp) {                          \
    memset(sp, 0, sizeof(uint32_t) * ((size_t)slices + 1));                                                 \
    uint32_t off = 0, s = 0, last = 0;                                                                      \
    for (uint32_t r = 0; r < rows; ++r) {                                                                   \
      if (r - last >= slice_size || s == 0) {                                                               \
        sp[s++] = off;                                                                                      \
        last = r;                                                                                           \
      }                                                                                                     \
      for (uint32_t k = rp[r]; k < rp[r + 1]; ++k) {                                                        \
        v[off] = data[k];                                                                                   \
        ci[off] = cols[k];                                                                                  \
        ri[off] = r;                                                                                        \
        ++off;                                                                                              \
      }                                                                                                     \
    }                                                                                                       \
    sp[s] = off;                                                                                            \
  }
SCOO_FROM_CSR(float, oracle_scoo_from_csr_f32)
SCOO_FROM_CSR(double, oracle_scoo_from_csr_f64)

/* fill_row_blocks — gpu/csr_adaptive_spmv.cu:180-240. Returns the bin count. */
uint32_t oracle_fill_row_blocks(int fill, uint32_t rows, const uint32_t *rp, uint32_t per_wg, uint32_t *blocks) {
  if (fill) blocks[0] = 0;
  long long last = 0, i;
  uint32_t wg = 1, sum = 0;
  for (i = 1; i <= (long long)rows; i++) {
    sum += rp[i] - rp[i - 1];
    if (sum == per_wg) {
      last = i;
      if (fill) blocks[wg] = (uint32_t)i;
      wg++;
      sum = 0;
    } else if (sum > per_wg) {
      if (i - last > 1) {
        if (fill) blocks[wg] = (uint32_t)(i - 1);
        wg++;
        i--;
      } else {
        if (fill) blocks[wg] = (uint32_t)i;
        wg++;
      }
      last = i;
      sum = 0;
    } else if ((unsigned long long)(i - last) > per_wg) {
      last = i;
      if (fill) blocks[wg] = (uint32_t)i;
      wg++;
      sum = 0;
    }
  }
  if (fill) blocks[wg] = rows;
  return wg;
}
