// On-device format conversion: the reference's host converters
// (common/matrix_converter.cpp, common/scoo_matrix_class.cpp) as CUDA kernels
// over device arrays.  Every output array is identical, element for element,
// to the host converters in formats.cpp (and so to the reference's).
//
// Building blocks:
//   - an exclusive scan of a per-item count (row lengths, tail lengths, radix
//     histograms): block sums, one CTA over the block sums, block-local scans;
//   - a row expansion for COO-shaped outputs: a 2048-element output tile marks
//     the first position of every row that starts inside it with the row id,
//     then an inclusive max-scan over the tile gives each position its row
//     (empty rows never mark a position, long rows span tiles);
//   - a stable LSD radix sort (8-bit digits, per-tile histograms in
//     digit-major order, stable in-tile ranking by warp match) for COO
//     triplets -> CSR on the composite key (row, column).
#include "host_common.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

using namespace mfp;

namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kWarps = kThreads / 32;
constexpr uint32_t kItems = 8;
constexpr uint32_t kTile = kThreads * kItems;  // items per CTA in scans and expansions
constexpr uint32_t kRadixRounds = 16;
constexpr uint32_t kRadixTile = kThreads * kRadixRounds;  // keys per CTA in a radix pass

int cuda_fail(cudaError_t e, const char *what) {
  return fail(MFP_ERROR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
#define CV_TRY(expr, what)                               \
  do {                                                   \
    cudaError_t _e = (expr);                             \
    if (_e != cudaSuccess) return cuda_fail(_e, what);   \
  } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }
inline uint32_t blocks_for(uint64_t n, uint64_t per) { return (uint32_t)((n + per - 1) / per); }
inline uint32_t bits_for(uint32_t x) { return x ? 32u - (uint32_t)__builtin_clz(x) : 0u; }

// shared-memory index with one pad word per 32 (conflict-free strided reads)
__device__ __forceinline__ uint32_t pad(uint32_t i) { return i + (i >> 5); }

__device__ __forceinline__ uint32_t warp_incl_sum(uint32_t v) {
  const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
  for (uint32_t o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ uint32_t warp_incl_max(uint32_t v) {
  const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
  for (uint32_t o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = max(v, t);
  }
  return v;
}

// Exclusive block prefix (sum or max) of one value per thread; *total gets the
// block's reduction.  s holds kWarps words.
template <bool MAX>
__device__ __forceinline__ uint32_t block_excl(uint32_t v, uint32_t *s, uint32_t *total) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint32_t inc = MAX ? warp_incl_max(v) : warp_incl_sum(v);
  if (lane == 31) s[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t t = lane < kWarps ? s[lane] : 0u;
    t = MAX ? warp_incl_max(t) : warp_incl_sum(t);
    if (lane < kWarps) s[lane] = t;
  }
  __syncthreads();
  const uint32_t before = w ? s[w - 1] : 0u;
  if (total) *total = s[kWarps - 1];
  __syncthreads();
  if (MAX) {
    const uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
    return max(before, lane ? ex : 0u);
  }
  return before + inc - v;
}

// ---------------------------------------------------------------------------
// Exclusive scan of f(i), i in [0, n): out[0..n], out[n] = the total.
// ---------------------------------------------------------------------------
struct f_counts {
  const uint32_t *c;
  __device__ uint32_t operator()(uint32_t i) const { return c[i]; }
};
// in-row positions >= start of row i (coo_matrix_class tail, matrix_converter.cpp:242-257)
struct f_tail {
  const uint32_t *rp;
  uint32_t start;
  __device__ uint32_t operator()(uint32_t i) const {
    const uint32_t len = rp[i + 1] - rp[i];
    return len > start ? len - start : 0u;
  }
};

template <typename F>
__global__ void __launch_bounds__(kThreads) scan_reduce_kernel(uint32_t n, F f, uint32_t *sums) {
  __shared__ uint32_t s[kWarps];
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  uint32_t acc = 0;
#pragma unroll
  for (uint32_t j = 0; j < kItems; ++j) {
    const uint64_t i = base + j * kThreads + threadIdx.x;
    if (i < n) acc += f((uint32_t)i);
  }
  uint32_t total;
  block_excl<false>(acc, s, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One CTA: sums[0..nb) -> exclusive offsets in place; *grand = the total.
__global__ void __launch_bounds__(kThreads) scan_sums_kernel(uint32_t nb, uint32_t *sums, uint32_t *grand) {
  __shared__ uint32_t s[kWarps];
  uint32_t carry = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += kThreads) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t v = i < nb ? sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_excl<false>(v, s, &total);
    if (i < nb) sums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *grand = carry;
}

template <typename F>
__global__ void __launch_bounds__(kThreads) scan_apply_kernel(uint32_t n, F f, const uint32_t *offsets,
                                                              uint32_t *out) {
  __shared__ uint32_t tile[kTile + kTile / 32];
  __shared__ uint32_t s[kWarps];
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
#pragma unroll
  for (uint32_t j = 0; j < kItems; ++j) {
    const uint32_t p = j * kThreads + threadIdx.x;
    tile[pad(p)] = base + p < n ? f((uint32_t)(base + p)) : 0u;
  }
  __syncthreads();
  uint32_t v[kItems], acc = 0;
#pragma unroll
  for (uint32_t k = 0; k < kItems; ++k) {
    v[k] = acc;
    acc += tile[pad(threadIdx.x * kItems + k)];
  }
  const uint32_t ex = block_excl<false>(acc, s, nullptr) + offsets[blockIdx.x];
#pragma unroll
  for (uint32_t k = 0; k < kItems; ++k) tile[pad(threadIdx.x * kItems + k)] = ex + v[k];
  __syncthreads();
#pragma unroll
  for (uint32_t j = 0; j < kItems; ++j) {
    const uint32_t p = j * kThreads + threadIdx.x;
    if (base + p < n) out[base + p] = tile[pad(p)];
  }
}

// Scratch comes from a per-device memory pool private to the converters.  Its
// release threshold is unlimited, so freed scratch stays mapped for the next
// conversion (the device's default pool would hand it back to the driver at
// every synchronisation and map it again on the next call, which costs
// milliseconds per GB); mfp_dev_scratch_release returns it.
std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;

int scratch_pool(cudaMemPool_t *out) {
  int dev = 0;
  CV_TRY(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(dev);
  if (it != g_pools.end()) {
    *out = it->second;
    return MFP_SUCCESS;
  }
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool;
  CV_TRY(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
  uint64_t keep = UINT64_MAX;
  CV_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
  g_pools[dev] = pool;
  *out = pool;
  return MFP_SUCCESS;
}

// Scratch that lives for one converter call, freed in stream order.
struct scratch {
  cudaStream_t st;
  cudaMemPool_t pool = nullptr;
  std::vector<void *> ptrs;
  explicit scratch(cudaStream_t s) : st(s) {}
  ~scratch() {
    for (void *p : ptrs) cudaFreeAsync(p, st);
  }
  template <typename T>
  int get(T **p, size_t count) {
    *p = nullptr;
    if (!count) return MFP_SUCCESS;
    if (!pool) {
      const int s = scratch_pool(&pool);
      if (s) return s;
    }
    void *q = nullptr;
    CV_TRY(cudaMallocFromPoolAsync(&q, count * sizeof(T), pool, st), "cudaMallocFromPoolAsync");
    ptrs.push_back(q);
    *p = static_cast<T *>(q);
    return MFP_SUCCESS;
  }
};

template <typename F>
int exclusive_scan(uint32_t n, F f, uint32_t *out, scratch &sc) {
  if (n == 0) {
    CV_TRY(cudaMemsetAsync(out, 0, sizeof(uint32_t), sc.st), "cudaMemsetAsync");
    return MFP_SUCCESS;
  }
  const uint32_t nb = blocks_for(n, kTile);
  uint32_t *sums = nullptr;
  int st = sc.get(&sums, nb);
  if (st) return st;
  scan_reduce_kernel<F><<<nb, kThreads, 0, sc.st>>>(n, f, sums);
  scan_sums_kernel<<<1, kThreads, 0, sc.st>>>(nb, sums, out + n);
  scan_apply_kernel<F><<<nb, kThreads, 0, sc.st>>>(n, f, sums, out);
  CV_TRY(cudaGetLastError(), "scan launch");
  return MFP_SUCCESS;
}

// ---------------------------------------------------------------------------
// Row expansion: output element j in [0, total) belongs to the row r with
// tp[r] <= j < tp[r+1] and copies source element rp[r] + start + (j - tp[r]).
// With tp == rp and start == 0 (plain COO / SCOO) the values and columns are
// the CSR arrays themselves, copied whole; only the row ids are written here.
// ---------------------------------------------------------------------------
// tr[i] = the row holding output position i * kTile (i < ntiles) or total - 1
// (i = ntiles): the largest r < rows with tp[r] <= pos.
__global__ void __launch_bounds__(kThreads) tile_rows_kernel(uint32_t rows, uint32_t total, const uint32_t *tp,
                                                             uint32_t ntiles, uint32_t *tr) {
  const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i > ntiles) return;
  const uint32_t pos = i < ntiles ? i * kTile : total - 1u;
  uint32_t lo = 0, hi = rows - 1;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo + 1) / 2;
    if (tp[mid] <= pos) lo = mid; else hi = mid - 1;
  }
  tr[i] = lo;
}

template <typename T, bool COPY>
__global__ void __launch_bounds__(kThreads) expand_kernel(uint32_t total, const uint32_t *tr, const uint32_t *tp,
                                                          const uint32_t *rp, uint32_t start,
                                                          const uint32_t *__restrict__ cols,
                                                          const T *__restrict__ vals, T *__restrict__ od,
                                                          uint32_t *__restrict__ oc, uint32_t *__restrict__ orow) {
  __shared__ uint32_t s_row[kTile + kTile / 32];
  __shared__ uint32_t s[kWarps];
  const uint32_t j0 = blockIdx.x * kTile;
  const uint32_t n = min(kTile, total - j0);
  const uint32_t r0 = tr[blockIdx.x], r1 = tr[blockIdx.x + 1];
  for (uint32_t p = threadIdx.x; p < kTile; p += kThreads) s_row[pad(p)] = 0u;
  __syncthreads();
  // mark the first position of every row starting in this tile (r0 covers
  // position 0; rows up to r1 may start in the next tile and are skipped)
  for (uint32_t r = r0 + threadIdx.x; r <= r1 && r >= r0; r += kThreads) {
    const uint32_t b = tp[r], e = tp[r + 1];
    if (b < e && b < j0 + n) s_row[pad(max(b, j0) - j0)] = r;
  }
  __syncthreads();
  // inclusive max-scan over the tile: each position takes the last row mark
  uint32_t v[kItems], m = 0;
#pragma unroll
  for (uint32_t k = 0; k < kItems; ++k) {
    m = max(m, s_row[pad(threadIdx.x * kItems + k)]);
    v[k] = m;
  }
  const uint32_t before = block_excl<true>(m, s, nullptr);
#pragma unroll
  for (uint32_t k = 0; k < kItems; ++k) s_row[pad(threadIdx.x * kItems + k)] = max(before, v[k]);
  __syncthreads();
  // all loads of a thread are issued before its stores
  uint32_t src[kItems];
#pragma unroll
  for (uint32_t k = 0; k < kItems; ++k) {
    const uint32_t p = k * kThreads + threadIdx.x;
    v[k] = p < n ? s_row[pad(p)] : 0u;
    if (COPY) src[k] = p < n ? rp[v[k]] + start + (j0 + p - tp[v[k]]) : 0u;
  }
  if (COPY) {
    T dv[kItems];
    uint32_t dc[kItems];
#pragma unroll
    for (uint32_t k = 0; k < kItems; ++k)
      if (k * kThreads + threadIdx.x < n) {
        dv[k] = vals[src[k]];
        dc[k] = cols[src[k]];
      }
#pragma unroll
    for (uint32_t k = 0; k < kItems; ++k)
      if (k * kThreads + threadIdx.x < n) {
        od[j0 + k * kThreads + threadIdx.x] = dv[k];
        oc[j0 + k * kThreads + threadIdx.x] = dc[k];
      }
  }
#pragma unroll
  for (uint32_t k = 0; k < kItems; ++k) {
    const uint32_t p = k * kThreads + threadIdx.x;
    if (p < n) orow[j0 + p] = v[k];
  }
}

// ELL: thread per row, slots in order, column-major stores (coalesced across
// the warp).  When a CTA's CSR segment fits kEllCap elements and is not much
// longer than the slots it fills, it is first staged in shared memory with
// coalesced loads (one pad word per 32: conflict-free for rows of 32).
constexpr uint32_t kEllCap = 8192;
template <typename T>
constexpr size_t ell_smem_bytes() {
  return (size_t)(kEllCap + kEllCap / 32) * (sizeof(T) + sizeof(uint32_t));
}

template <typename T>
__global__ void __launch_bounds__(kThreads) ell_kernel(uint32_t rows, uint32_t width, const uint32_t *__restrict__ rp,
                                                       const uint32_t *__restrict__ cols,
                                                       const T *__restrict__ vals, T *__restrict__ ed,
                                                       uint32_t *__restrict__ ec) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sv = reinterpret_cast<T *>(smem_raw);
  uint32_t *sc = reinterpret_cast<uint32_t *>(sv + kEllCap + kEllCap / 32);
  const uint32_t r0 = blockIdx.x * kThreads;
  const uint32_t nr = min(kThreads, rows - r0);
  const uint32_t seg0 = rp[r0], seg1 = rp[r0 + nr];
  const uint32_t r = r0 + threadIdx.x;
  const bool has = r < rows;
  const uint32_t b = has ? rp[r] : 0u;
  const uint32_t len = has ? min(rp[r + 1] - b, width) : 0u;
  const bool staged = seg1 - seg0 <= kEllCap && (uint64_t)(seg1 - seg0) <= 2ull * nr * width;
  if (staged) {
    // 8 loads in flight per thread before their shared-memory stores
    for (uint32_t e0 = seg0 + threadIdx.x; e0 < seg1; e0 += 8u * kThreads) {
      T vv[8];
      uint32_t cc[8];
#pragma unroll
      for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t e = e0 + k * kThreads;
        if (e < seg1) {
          vv[k] = vals[e];
          cc[k] = cols[e];
        }
      }
#pragma unroll
      for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t e = e0 + k * kThreads;
        if (e < seg1) {
          sv[pad(e - seg0)] = vv[k];
          sc[pad(e - seg0)] = cc[k];
        }
      }
    }
    __syncthreads();
  }
  if (!has) return;
  for (uint32_t s = 0; s < width; ++s) {
    const size_t o = (size_t)s * rows + r;
    if (s < len) {
      ed[o] = staged ? sv[pad(b - seg0 + s)] : vals[b + s];
      ec[o] = staged ? sc[pad(b - seg0 + s)] : cols[b + s];
    } else {
      ed[o] = T(0);
      ec[o] = 0u;
    }
  }
}

// slices_ptr: a slice starts every slice_size rows (scoo_matrix_class.cpp:76-100);
// entries after the last real slice stay 0.
__global__ void __launch_bounds__(kThreads) scoo_slices_kernel(uint32_t nnz, const uint32_t *rp, uint32_t slice_size,
                                                               uint32_t count, uint32_t real, uint32_t *sp) {
  const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i > count) return;
  sp[i] = i < real ? rp[(size_t)i * slice_size] : (i == real ? nnz : 0u);
}

// ---------------------------------------------------------------------------
// Row statistics: min / max / sum of row lengths, then the sum of squared
// deviations from the integer average as an exact 64-bit integer.
// ---------------------------------------------------------------------------
// Grid-stride over rows, then one atomic per block and quantity (same-address
// atomics from every warp would serialise in L2).
constexpr uint32_t kStatBlocks = 148 * 4;

template <typename T>
__device__ __forceinline__ T block_reduce_op(T v, T *s, int op) {  // op 0 sum, 1 min, 2 max, 3 or
  for (uint32_t o = 16; o; o >>= 1) {
    const T u = __shfl_xor_sync(0xffffffffu, v, o);
    v = op == 0 ? v + u : op == 1 ? min(v, u) : op == 2 ? max(v, u) : (v | u);
  }
  if ((threadIdx.x & 31u) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0)
    for (uint32_t w = 1; w < kWarps; ++w) v = op == 0 ? v + s[w] : op == 1 ? min(v, s[w]) : op == 2 ? max(v, s[w]) : (v | s[w]);
  __syncthreads();
  return v;  // valid in thread 0
}

__global__ void __launch_bounds__(kThreads) row_minmax_kernel(uint32_t rows, const uint32_t *rp,
                                                              unsigned long long *acc) {
  __shared__ unsigned long long s[kWarps];
  unsigned long long mn = 0xffffffffull, mx = 0ull, sm = 0ull;
  for (uint64_t r = (uint64_t)blockIdx.x * kThreads + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * kThreads) {
    const unsigned long long n = rp[r + 1] - rp[r];
    mn = min(mn, n);
    mx = max(mx, n);
    sm += n;
  }
  mn = block_reduce_op(mn, s, 1);
  mx = block_reduce_op(mx, s, 2);
  sm = block_reduce_op(sm, s, 0);
  if (threadIdx.x == 0) {
    atomicMin(&acc[0], mn);
    atomicMax(&acc[1], mx);
    atomicAdd(&acc[2], sm);
  }
}
// acc[3] += (n - avg)^2; acc[4] flags a deviation >= 2^26 (its square may not
// be exact in double, so the exact-sum shortcut does not apply)
__global__ void __launch_bounds__(kThreads) row_sqdev_kernel(uint32_t rows, const uint32_t *rp, uint32_t avg,
                                                             unsigned long long *acc) {
  __shared__ unsigned long long s[kWarps];
  unsigned long long q = 0, big = 0;
  for (uint64_t r = (uint64_t)blockIdx.x * kThreads + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * kThreads) {
    const uint32_t n = rp[r + 1] - rp[r];
    const unsigned long long d = n > avg ? n - avg : avg - n;
    q += d * d;
    big |= d >= (1ull << 26);
  }
  q = block_reduce_op(q, s, 0);
  big = block_reduce_op(big, s, 3);
  if (threadIdx.x == 0) {
    atomicAdd(&acc[3], q);
    if (big) atomicOr(&acc[4], 1ull);
  }
}
// acc[0] += sum over rows of max(0, len - start)
__global__ void __launch_bounds__(kThreads) tail_count_kernel(uint32_t rows, const uint32_t *rp, uint32_t start,
                                                              unsigned long long *acc) {
  __shared__ unsigned long long s[kWarps];
  unsigned long long c = 0;
  for (uint64_t r = (uint64_t)blockIdx.x * kThreads + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * kThreads) {
    const uint32_t n = rp[r + 1] - rp[r];
    c += n > start ? n - start : 0u;
  }
  c = block_reduce_op(c, s, 0);
  if (threadIdx.x == 0) atomicAdd(acc, c);
}

// Checks a device CSR: row_ptr[0] = 0, non-decreasing, row_ptr[rows] = nnz,
// columns < cols.  err[0] |= 1 (row_ptr) / 2 (column), err[1] = min bad index.
__global__ void __launch_bounds__(kThreads) check_csr_kernel(uint32_t rows, uint32_t nnz, uint32_t cols,
                                                             const uint32_t *rp, const uint32_t *ci, uint32_t *err) {
  const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  if (i <= rows) {
    const uint32_t a = rp[i];
    const bool bad = (i == 0 && a != 0) || (i == rows && a != nnz) || (i < rows && rp[i + 1] < a);
    if (bad) {
      atomicOr(&err[0], 1u);
      atomicMin(&err[1], (uint32_t)i);
    }
  }
  if (i < nnz && ci[i] >= cols && !(cols == 0 && ci[i] == 0)) {
    atomicOr(&err[0], 2u);
    atomicMin(&err[2], (uint32_t)i);
  }
}

// Per-slice column window [min, max + 1) (mfp_scoo_x_windows on the device).
__global__ void __launch_bounds__(kThreads) scoo_windows_kernel(uint32_t nnz, const uint32_t *ci, const uint32_t *sp,
                                                                uint32_t *win) {
  __shared__ uint32_t s_lo[kWarps], s_hi[kWarps];
  const uint32_t sl = blockIdx.x;
  const uint32_t b = sp[sl], e = sp[sl + 1];
  uint32_t lo = 0xffffffffu, hi = 0u;
  const bool any = b < e && e <= nnz;
  if (any)
    for (uint32_t k = b + threadIdx.x; k < e; k += kThreads) {
      lo = min(lo, ci[k]);
      hi = max(hi, ci[k] + 1u);
    }
  for (uint32_t o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31u) == 0) {
    s_lo[threadIdx.x >> 5] = lo;
    s_hi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t w = 1; w < kWarps; ++w) {
      lo = min(lo, s_lo[w]);
      hi = max(hi, s_hi[w]);
    }
    win[2 * sl] = any ? lo : 0u;
    win[2 * sl + 1] = any ? hi : 0u;
  }
}

// ---------------------------------------------------------------------------
// COO triplets -> CSR: keys (row << cb | col) with the value converted to T as
// payload, a stable LSD radix sort when the input is not already in CSR
// order, then row_ptr from the row boundaries of the sorted keys.
// ---------------------------------------------------------------------------
constexpr uint32_t kKeyBlocks = 148 * 8;

// err[0] |= 1 (row id) / 2 (col id), err[1] = first bad element; err[2] = 1
// when some key is smaller than its predecessor (input not in CSR order)
template <typename T>
__global__ void __launch_bounds__(kThreads) make_keys_kernel(uint32_t nnz, uint32_t rows, uint32_t cols,
                                                             const uint32_t *__restrict__ ri,
                                                             const uint32_t *__restrict__ ci,
                                                             const double *__restrict__ v, uint32_t cb,
                                                             unsigned long long *__restrict__ keys,
                                                             T *__restrict__ pay, uint32_t *err) {
  bool unsorted = false;
  for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < nnz; i += (uint64_t)gridDim.x * kThreads) {
    const uint32_t r = ri[i], c = ci[i];
    if (r >= rows || c >= cols) {
      atomicOr(&err[0], r >= rows ? 1u : 2u);
      atomicMin(&err[1], (uint32_t)i);
    }
    const unsigned long long k = ((unsigned long long)r << cb) | c;
    keys[i] = k;
    pay[i] = static_cast<T>(v[i]);
    if (i && (((unsigned long long)ri[i - 1] << cb) | ci[i - 1]) > k) unsorted = true;
  }
  if (__syncthreads_or(unsorted) && threadIdx.x == 0) err[2] = 1u;
}

__global__ void __launch_bounds__(kThreads) radix_hist_kernel(uint32_t n, const unsigned long long *keys,
                                                              uint32_t shift, uint32_t tiles, uint32_t *counts) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0u;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
#pragma unroll 4
  for (uint32_t j = 0; j < kRadixRounds; ++j) {
    const uint64_t i = base + j * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[(size_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one 4096-key tile: keys go, in tile order, after every key
// of a smaller digit and after the same digit's keys of earlier tiles
// (offsets = exclusive scan of the digit-major tile histograms).  Warp w ranks
// its contiguous 512 keys with a warp-private digit histogram (warp match for
// equal digits), the warps' counts are scanned per digit, the tile is placed
// in shared memory in digit order and written out as contiguous digit runs.
template <typename P>
struct radix_smem {
  unsigned long long key[kRadixTile];
  P pay[kRadixTile];
  uint32_t wh[kWarps][256];
  uint32_t gbase[256], start[256];
  uint32_t red[kWarps];
};

template <typename P>
__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(uint32_t n, const unsigned long long *keys,
                                                                 const P *pay, uint32_t shift, uint32_t tiles,
                                                                 const uint32_t *offsets,
                                                                 unsigned long long *keys_out, P *pay_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  radix_smem<P> &S = *reinterpret_cast<radix_smem<P> *>(smem_raw);
  constexpr uint32_t kPerWarp = kRadixTile / kWarps;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
  const uint32_t tn = (uint32_t)min((uint64_t)kRadixTile, n - base);
  const uint32_t wbase = warp * kPerWarp;
  unsigned long long k[kRadixRounds];
  P v[kRadixRounds];
#pragma unroll
  for (uint32_t j = 0; j < kRadixRounds; ++j) {
    const uint32_t p = wbase + j * 32u + lane;
    k[j] = p < tn ? keys[base + p] : 0ull;
    v[j] = p < tn ? pay[base + p] : P(0);
  }
#pragma unroll
  for (uint32_t w = 0; w < kWarps; ++w) S.wh[w][t] = 0u;
  S.gbase[t] = offsets[(size_t)t * tiles + blockIdx.x];
  __syncthreads();
  uint32_t rk[kRadixRounds];
#pragma unroll
  for (uint32_t j = 0; j < kRadixRounds; ++j) {
    const bool valid = wbase + j * 32u + lane < tn;
    const uint32_t d = valid ? (uint32_t)(k[j] >> shift) & 255u : 256u;  // 256: never a digit
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t before = valid ? S.wh[warp][d] : 0u;
    __syncwarp();
    if (valid && lane == (uint32_t)(__ffs(peers) - 1)) S.wh[warp][d] = before + __popc(peers);
    __syncwarp();
    rk[j] = before + __popc(peers & ((1u << lane) - 1u));
  }
  __syncthreads();
  uint32_t tot = 0;  // thread t: digit t
#pragma unroll
  for (uint32_t w = 0; w < kWarps; ++w) {
    const uint32_t c = S.wh[w][t];
    S.wh[w][t] = tot;
    tot += c;
  }
  S.start[t] = block_excl<false>(tot, S.red, nullptr);
  __syncthreads();
#pragma unroll
  for (uint32_t j = 0; j < kRadixRounds; ++j) {
    if (wbase + j * 32u + lane < tn) {
      const uint32_t d = (uint32_t)(k[j] >> shift) & 255u;
      const uint32_t lp = S.start[d] + S.wh[warp][d] + rk[j];
      S.key[lp] = k[j];
      S.pay[lp] = v[j];
    }
  }
  __syncthreads();
  for (uint32_t p = t; p < tn; p += kThreads) {
    const unsigned long long kk = S.key[p];
    const uint32_t d = (uint32_t)(kk >> shift) & 255u;
    const uint32_t g = S.gbase[d] + (p - S.start[d]);
    keys_out[g] = kk;
    pay_out[g] = S.pay[p];
  }
}

// row_ptr from sorted keys: position p starts the rows (row(p-1), row(p)]
// (p = nnz closes the rows after the last element's row).
__global__ void __launch_bounds__(kThreads) rowptr_from_keys_kernel(uint32_t nnz, uint32_t rows,
                                                                    const unsigned long long *keys, uint32_t cb,
                                                                    uint32_t *rp) {
  const uint64_t p = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  if (p > nnz) return;
  const int64_t cur = p < nnz ? (int64_t)(keys[p] >> cb) : (int64_t)rows;
  const int64_t prev = p ? (int64_t)(keys[p - 1] >> cb) : -1;
  for (int64_t q = prev + 1; q <= cur; ++q) rp[q] = (uint32_t)p;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) csr_split_kernel(uint32_t nnz, const unsigned long long *__restrict__ keys,
                                                             const T *__restrict__ pay, unsigned long long cmask,
                                                             uint32_t *__restrict__ cols_out, T *__restrict__ data_out) {
  const uint32_t p = blockIdx.x * kThreads + threadIdx.x;
  if (p >= nnz) return;
  cols_out[p] = (uint32_t)(keys[p] & cmask);
  data_out[p] = pay[p];
}

bool valid_vt(int vt) { return vt == MFP_F32 || vt == MFP_F64; }

template <typename T>
int coo_from_csr_t(uint32_t rows, const uint32_t *rp, const uint32_t *ci, const T *vals, uint32_t start, T *od,
                   uint32_t *oc, uint32_t *orow, void *stream) {
  cudaStream_t st = as_stream(stream);
  scratch sc(st);
  if (rows == 0) return ok();
  const uint32_t *tp = rp;
  uint32_t *tpw = nullptr;
  int s;
  if (start) {
    if ((s = sc.get(&tpw, (size_t)rows + 1))) return s;
    if ((s = exclusive_scan(rows, f_tail{rp, start}, tpw, sc))) return s;
    tp = tpw;
  }
  uint32_t total = 0;
  CV_TRY(cudaMemcpyAsync(&total, tp + rows, sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (total == 0) return ok();
  if (!od || !oc || !orow) return fail(MFP_ERROR_INVALID_VALUE, "null output array");
  const uint32_t ntiles = blocks_for(total, kTile);
  uint32_t *tr = nullptr;
  if ((s = sc.get(&tr, (size_t)ntiles + 1))) return s;
  tile_rows_kernel<<<blocks_for((uint64_t)ntiles + 1, kThreads), kThreads, 0, st>>>(rows, total, tp, ntiles, tr);
  if (start) {
    expand_kernel<T, true><<<ntiles, kThreads, 0, st>>>(total, tr, tp, rp, start, ci, vals, od, oc, orow);
  } else {
    CV_TRY(cudaMemcpyAsync(od, vals, (size_t)total * sizeof(T), cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
    CV_TRY(cudaMemcpyAsync(oc, ci, (size_t)total * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
    expand_kernel<T, false><<<ntiles, kThreads, 0, st>>>(total, tr, tp, rp, 0u, ci, vals, od, oc, orow);
  }
  CV_TRY(cudaGetLastError(), "expand_kernel");
  return ok();
}

// Stable LSD radix sort of n (key, payload) pairs on the low `bits` key bits;
// k0 / p0 hold the input and, on return, the sorted pairs (buffers swap).
template <typename P>
int radix_sort_pairs(uint32_t n, uint32_t bits, unsigned long long *&k0, P *&p0, scratch &sc) {
  if (n == 0 || bits == 0) return MFP_SUCCESS;
  const uint32_t tiles = blocks_for(n, kRadixTile);
  const uint64_t ncount = 256ull * tiles;
  if (ncount > 0xffffffffull) return fail(MFP_ERROR_TOO_LARGE, "too many radix tiles");
  unsigned long long *k1 = nullptr;
  P *p1 = nullptr;
  uint32_t *hist = nullptr, *hoff = nullptr;
  int s;
  if ((s = sc.get(&k1, n)) || (s = sc.get(&p1, n)) || (s = sc.get(&hist, ncount)) || (s = sc.get(&hoff, ncount + 1)))
    return s;
  const size_t smem = sizeof(radix_smem<P>);
  CV_TRY(cudaFuncSetAttribute(radix_scatter_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
         "cudaFuncSetAttribute");
  for (uint32_t shift = 0; shift < bits; shift += 8) {
    radix_hist_kernel<<<tiles, kThreads, 0, sc.st>>>(n, k0, shift, tiles, hist);
    if ((s = exclusive_scan((uint32_t)ncount, f_counts{hist}, hoff, sc))) return s;
    radix_scatter_kernel<P><<<tiles, kThreads, smem, sc.st>>>(n, k0, p0, shift, tiles, hoff, k1, p1);
    CV_TRY(cudaGetLastError(), "radix pass");
    std::swap(k0, k1);
    std::swap(p0, p1);
  }
  return MFP_SUCCESS;
}

template <typename T>
int csr_from_coo_t(uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *ri, const uint32_t *ci,
                   const double *v, uint32_t *rp, uint32_t *co, T *data, void *stream) {
  cudaStream_t st = as_stream(stream);
  scratch sc(st);
  if (!rp) return fail(MFP_ERROR_INVALID_VALUE, "null row_ptr");
  if (nnz && (!ri || !ci || !v || !co || !data)) return fail(MFP_ERROR_INVALID_VALUE, "null array");
  if (nnz == 0) {
    CV_TRY(cudaMemsetAsync(rp, 0, ((size_t)rows + 1) * sizeof(uint32_t), st), "cudaMemsetAsync");
    CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    return ok();
  }
  const uint32_t rb = rows > 1 ? bits_for(rows - 1) : 0u, cb = cols > 1 ? bits_for(cols - 1) : 0u;
  uint32_t *err = nullptr;
  unsigned long long *k0 = nullptr;
  T *p0 = nullptr;
  int s;
  if ((s = sc.get(&err, 4)) || (s = sc.get(&k0, nnz)) || (s = sc.get(&p0, nnz))) return s;
  const uint32_t err_init[4] = {0u, 0xffffffffu, 0u, 0u};
  CV_TRY(cudaMemcpyAsync(err, err_init, sizeof(err_init), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
  make_keys_kernel<T><<<std::min(kKeyBlocks, blocks_for(nnz, kThreads)), kThreads, 0, st>>>(nnz, rows, cols, ri, ci,
                                                                                           v, cb, k0, p0, err);
  CV_TRY(cudaGetLastError(), "make_keys_kernel");
  uint32_t h_err[4];
  CV_TRY(cudaMemcpyAsync(h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (h_err[0] & 1u) return fail(MFP_ERROR_INVALID_VALUE, "row id >= rows %u at element %u", rows, h_err[1]);
  if (h_err[0] & 2u) return fail(MFP_ERROR_INVALID_VALUE, "col id >= cols %u at element %u", cols, h_err[1]);
  // not in CSR order: stable sort on (row, col); in order already, a stable sort would keep it
  if (h_err[2] && (s = radix_sort_pairs<T>(nnz, rb + cb, k0, p0, sc))) return s;
  rowptr_from_keys_kernel<<<blocks_for((uint64_t)nnz + 1, kThreads), kThreads, 0, st>>>(nnz, rows, k0, cb, rp);
  csr_split_kernel<T><<<blocks_for(nnz, kThreads), kThreads, 0, st>>>(nnz, k0, p0, (1ull << cb) - 1ull, co, data);
  CV_TRY(cudaGetLastError(), "csr_split_kernel");
  CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return ok();
}

// SCOO sort_cols: keys (slice << cb | col) with the element index as payload;
// after the stable sort, values and rows are gathered by index.
__global__ void __launch_bounds__(kThreads) slice_keys_kernel(uint32_t nnz, const uint32_t *__restrict__ ri,
                                                              const uint32_t *__restrict__ ci, uint32_t slice_size,
                                                              uint32_t cb, unsigned long long *__restrict__ keys,
                                                              uint32_t *__restrict__ idx) {
  const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= nnz) return;
  keys[i] = ((unsigned long long)(ri[i] / slice_size) << cb) | ci[i];
  idx[i] = i;
}
template <typename T>
__global__ void __launch_bounds__(kThreads) slice_gather_kernel(uint32_t nnz, const unsigned long long *__restrict__ keys,
                                                                const uint32_t *__restrict__ idx,
                                                                unsigned long long cmask, const T *__restrict__ v_in,
                                                                const uint32_t *__restrict__ r_in, T *__restrict__ v_out,
                                                                uint32_t *__restrict__ c_out, uint32_t *__restrict__ r_out) {
  const uint32_t p = blockIdx.x * kThreads + threadIdx.x;
  if (p >= nnz) return;
  const uint32_t j = idx[p];
  c_out[p] = (uint32_t)(keys[p] & cmask);
  v_out[p] = v_in[j];
  r_out[p] = r_in[j];
}

template <typename T>
int scoo_sort_cols_t(uint32_t rows, uint32_t cols, uint32_t slice_size, uint32_t nnz, T *v, uint32_t *ci,
                     uint32_t *ri, cudaStream_t st) {
  scratch sc(st);
  if (nnz == 0) return ok();
  if (!v || !ci || !ri) return fail(MFP_ERROR_INVALID_VALUE, "null array");
  if (slice_size == 0) return fail(MFP_ERROR_INVALID_VALUE, "slice_size 0");
  const uint32_t cb = cols > 1 ? bits_for(cols - 1) : 0u;
  const uint32_t sb = rows > slice_size ? bits_for((rows - 1) / slice_size) : 0u;
  unsigned long long *k0 = nullptr;
  uint32_t *p0 = nullptr;
  T *vcopy = nullptr;
  uint32_t *rcopy = nullptr;
  int s;
  if ((s = sc.get(&k0, nnz)) || (s = sc.get(&p0, nnz)) || (s = sc.get(&vcopy, nnz)) || (s = sc.get(&rcopy, nnz)))
    return s;
  CV_TRY(cudaMemcpyAsync(vcopy, v, (size_t)nnz * sizeof(T), cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
  CV_TRY(cudaMemcpyAsync(rcopy, ri, (size_t)nnz * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
  slice_keys_kernel<<<blocks_for(nnz, kThreads), kThreads, 0, st>>>(nnz, ri, ci, slice_size, cb, k0, p0);
  CV_TRY(cudaGetLastError(), "slice_keys_kernel");
  if ((s = radix_sort_pairs<uint32_t>(nnz, sb + cb, k0, p0, sc))) return s;
  slice_gather_kernel<T><<<blocks_for(nnz, kThreads), kThreads, 0, st>>>(nnz, k0, p0, (1ull << cb) - 1ull, vcopy, rcopy,
                                                                         v, ci, ri);
  CV_TRY(cudaGetLastError(), "slice_gather_kernel");
  CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return ok();
}

}  // namespace

extern "C" {

int mfp_dev_rows_statistics(uint32_t rows, const uint32_t *rp, mfp_rows_statistic *out, void *stream) {
  if (!rp || !out) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  if (rows == 0) return fail(MFP_ERROR_INVALID_VALUE, "rows == 0");
  cudaStream_t st = as_stream(stream);
  scratch sc(st);
  unsigned long long *acc = nullptr;
  int s = sc.get(&acc, 5);
  if (s) return s;
  // min starts at UINT_MAX - 1 like the reference (matrix_converter.cpp:100)
  const unsigned long long init[5] = {0xfffffffeull, 0ull, 0ull, 0ull, 0ull};
  CV_TRY(cudaMemcpyAsync(acc, init, sizeof(init), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
  const uint32_t sb = std::min(kStatBlocks, blocks_for(rows, kThreads));
  row_minmax_kernel<<<sb, kThreads, 0, st>>>(rows, rp, acc);
  unsigned long long h[5];
  CV_TRY(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  mfp_rows_statistic r{};
  r.min_elements_in_rows = (uint32_t)h[0];
  r.max_elements_in_rows = (uint32_t)h[1];
  // the reference sums in unsigned int (matrix_converter.cpp:102-116)
  r.avg_elements_in_rows = (uint32_t)h[2] / rows;
  row_sqdev_kernel<<<sb, kThreads, 0, st>>>(rows, rp, r.avg_elements_in_rows, acc);
  CV_TRY(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (h[4] == 0 && h[3] < (1ull << 53)) {
    // every partial sum of the reference's double loop is an integer below
    // 2^53, so that loop is exact and equals this integer sum
    r.elements_in_rows_std_deviation = std::sqrt((double)h[3] / rows);
  } else {
    // outside the exact range: run the reference's sequential loop on the host
    std::vector<uint32_t> hp((size_t)rows + 1);
    CV_TRY(cudaMemcpy(hp.data(), rp, hp.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
    return mfp_get_rows_statistics(rows, hp.data(), out);
  }
  *out = r;
  return ok();
}

int mfp_dev_check_csr(uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *rp, const uint32_t *ci,
                      void *stream) {
  if (!rp || (nnz && !ci)) return fail(MFP_ERROR_INVALID_VALUE, "null array");
  cudaStream_t st = as_stream(stream);
  scratch sc(st);
  uint32_t *err = nullptr;
  int s = sc.get(&err, 3);
  if (s) return s;
  const uint32_t init[3] = {0u, 0xffffffffu, 0xffffffffu};
  CV_TRY(cudaMemcpyAsync(err, init, sizeof(init), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
  const uint64_t n = std::max<uint64_t>((uint64_t)rows + 1, nnz);
  check_csr_kernel<<<blocks_for(n, kThreads), kThreads, 0, st>>>(rows, nnz, cols, rp, ci, err);
  CV_TRY(cudaGetLastError(), "check_csr_kernel");
  uint32_t h[3];
  CV_TRY(cudaMemcpyAsync(h, err, sizeof(h), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (h[0] & 1u) return fail(MFP_ERROR_INVALID_VALUE, "row_ptr is not a CSR row pointer (entry %u)", h[1]);
  if (h[0] & 2u) return fail(MFP_ERROR_INVALID_VALUE, "column id >= cols %u at element %u", cols, h[2]);
  return ok();
}

int mfp_dev_coo_count(uint32_t rows, const uint32_t *rp, uint32_t start, uint32_t *count, void *stream) {
  if (!rp || !count) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  *count = 0;
  if (rows == 0) return ok();
  cudaStream_t st = as_stream(stream);
  if (start == 0) {  // every element: row_ptr[rows] - row_ptr[0]
    uint32_t ends[2];
    CV_TRY(cudaMemcpyAsync(&ends[0], rp, sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CV_TRY(cudaMemcpyAsync(&ends[1], rp + rows, sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    *count = ends[1] - ends[0];
    return ok();
  }
  scratch sc(st);
  unsigned long long *acc = nullptr;
  int s;
  if ((s = sc.get(&acc, 1))) return s;
  CV_TRY(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), st), "cudaMemsetAsync");
  tail_count_kernel<<<std::min(kStatBlocks, blocks_for(rows, kThreads)), kThreads, 0, st>>>(rows, rp, start, acc);
  CV_TRY(cudaGetLastError(), "tail_count_kernel");
  unsigned long long h = 0;
  CV_TRY(cudaMemcpyAsync(&h, acc, sizeof(h), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  CV_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  *count = (uint32_t)h;
  return ok();
}

int mfp_dev_coo_from_csr(int vt, uint32_t rows, const uint32_t *rp, const uint32_t *ci, const void *vals,
                         uint32_t start, void *od, uint32_t *oc, uint32_t *orow, void *stream) {
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  if (!rp) return fail(MFP_ERROR_INVALID_VALUE, "null row_ptr");
  if (vt == MFP_F64)
    return coo_from_csr_t<double>(rows, rp, ci, static_cast<const double *>(vals), start, static_cast<double *>(od),
                                  oc, orow, stream);
  return coo_from_csr_t<float>(rows, rp, ci, static_cast<const float *>(vals), start, static_cast<float *>(od), oc,
                               orow, stream);
}

int mfp_dev_ell_from_csr(int vt, uint32_t rows, const uint32_t *rp, const uint32_t *ci, const void *vals,
                         uint32_t width, void *ed, uint32_t *ec, void *stream) {
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  if (!rp || ((uint64_t)rows * width && (!ed || !ec))) return fail(MFP_ERROR_INVALID_VALUE, "null array");
  if (rows == 0 || width == 0) return ok();
  cudaStream_t st = as_stream(stream);
  if (vt == MFP_F64) {
    CV_TRY(cudaFuncSetAttribute(ell_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ell_smem_bytes<double>()),
           "cudaFuncSetAttribute");
    ell_kernel<double><<<blocks_for(rows, kThreads), kThreads, ell_smem_bytes<double>(), st>>>(
        rows, width, rp, ci, static_cast<const double *>(vals), static_cast<double *>(ed), ec);
  } else {
    CV_TRY(cudaFuncSetAttribute(ell_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ell_smem_bytes<float>()),
           "cudaFuncSetAttribute");
    ell_kernel<float><<<blocks_for(rows, kThreads), kThreads, ell_smem_bytes<float>(), st>>>(
        rows, width, rp, ci, static_cast<const float *>(vals), static_cast<float *>(ed), ec);
  }
  CV_TRY(cudaGetLastError(), "ell_kernel");
  return ok();
}

int mfp_dev_scoo_from_csr(int vt, uint32_t rows, uint32_t nnz, const uint32_t *rp, const uint32_t *ci,
                          const void *vals, const mfp_scoo_params *prm, void *ov, uint32_t *oc, uint32_t *orow,
                          uint32_t *sp, void *stream) {
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  if (!rp || !prm || !sp) return fail(MFP_ERROR_INVALID_VALUE, "null array");
  if (prm->slice_size == 0 && rows) return fail(MFP_ERROR_INVALID_VALUE, "slice_size 0");
  const uint32_t real = rows ? (uint32_t)(((uint64_t)rows + prm->slice_size - 1) / prm->slice_size) : 0u;
  if (real > prm->slices_count) return fail(MFP_ERROR_INVALID_VALUE, "too many slices");
  cudaStream_t st = as_stream(stream);
  scoo_slices_kernel<<<blocks_for((uint64_t)prm->slices_count + 1, kThreads), kThreads, 0, st>>>(
      nnz, rp, prm->slice_size, prm->slices_count, real, sp);
  CV_TRY(cudaGetLastError(), "scoo_slices_kernel");
  // values, c_index and r_index are the CSR arrays in CSR order with row ids
  return mfp_dev_coo_from_csr(vt, rows, rp, ci, vals, 0, ov, oc, orow, stream);
}

int mfp_dev_scoo_sort_cols(int vt, uint32_t rows, uint32_t cols, uint32_t slice_size, uint32_t nnz, void *values,
                           uint32_t *c_index, uint32_t *r_index, void *stream) {
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  if (vt == MFP_F64)
    return scoo_sort_cols_t<double>(rows, cols, slice_size, nnz, static_cast<double *>(values), c_index, r_index,
                                    as_stream(stream));
  return scoo_sort_cols_t<float>(rows, cols, slice_size, nnz, static_cast<float *>(values), c_index, r_index,
                                 as_stream(stream));
}

int mfp_dev_scoo_x_windows(uint32_t nnz, const uint32_t *ci, const uint32_t *sp, uint32_t slices, uint32_t *win,
                           void *stream) {
  if (!sp || !win || (nnz && !ci)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  if (slices == 0) return ok();
  scoo_windows_kernel<<<slices, kThreads, 0, as_stream(stream)>>>(nnz, ci, sp, win);
  CV_TRY(cudaGetLastError(), "scoo_windows_kernel");
  return ok();
}

int mfp_dev_scratch_release(void) {
  cudaMemPool_t pool;
  const int s = scratch_pool(&pool);
  if (s) return s;
  CV_TRY(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  CV_TRY(cudaMemPoolTrimTo(pool, 0), "cudaMemPoolTrimTo");
  return ok();
}

int mfp_dev_scratch_bytes(uint64_t *reserved) {
  if (!reserved) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  cudaMemPool_t pool;
  const int s = scratch_pool(&pool);
  if (s) return s;
  CV_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, reserved), "cudaMemPoolGetAttribute");
  return ok();
}

int mfp_dev_csr_from_coo(int vt, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *ri, const uint32_t *ci,
                         const double *v, uint32_t *rp, uint32_t *co, void *data, void *stream) {
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  if (vt == MFP_F64)
    return csr_from_coo_t<double>(rows, cols, nnz, ri, ci, v, rp, co, static_cast<double *>(data), stream);
  return csr_from_coo_t<float>(rows, cols, nnz, ri, ci, v, rp, co, static_cast<float *>(data), stream);
}

}  // extern "C"
