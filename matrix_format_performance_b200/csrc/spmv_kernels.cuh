// SpMV format kernels for B200 (sm_100a).
//
// Every kernel stages a CTA's share of the matrix through shared memory as
// products p = value * x[col] (16-byte streaming loads, see spmv_device.cuh)
// and then reduces the products by row.  What differs per format is how
// rows are assigned to threads, which mirrors the reference algorithm of the
// same name:
//   CSR scalar    one thread sums one row, in CSR order
//                 (gpu/gpu_matrix_multiplier.cu:22-43)
//   CSR vector    a group of 2..32 lanes per row, lane-strided + shuffle tree
//                 (gpu/gpu_matrix_multiplier.cu:331-362, gpu/reduce.cuh)
//   CSR-Adaptive  host-built row bins; many-row bins reduce from shared
//                 memory, single-row bins by the whole CTA
//                 (gpu/csr_adaptive_spmv.cu:26-178)
//   ELL           one thread per row over column-major slots
//                 (gpu/gpu_matrix_multiplier.cu:450-471)
//   COO           two passes: warp tiles of 256 consecutive elements reduce
//                 their runs (shuffle segmented scan) and write inner rows;
//                 a fix-up pass adds the rows that cross tiles (replaces the
//                 atomics of gpu_matrix_multiplier.cu:622-638).  The
//                 allocation-free entry point keeps a single-pass kernel
//                 whose tiles combine shared rows by look-back.
//   SCOO          one CTA per slice, shared-memory row accumulators and an
//                 optional shared-memory copy of the slice's x window
//                 (gpu/scoo_spmv.cu:46-129); the sort_cols layout adds into
//                 the accumulators with shared-memory atomics
//   HYB           the ELL kernel for the ELL part, then the two COO passes in
//                 accumulate mode for the tail (the reference's
//                 gpu/gpu_matrix_multiplier.cu:969-1002, with the tail's
//                 atomics replaced by the COO reduction)
// Rows longer than a plan threshold (CSR family) are cut into pieces that
// run as extra CTAs of the same launch and meet in a partial-sum buffer.
#pragma once

#include "spmv_device.cuh"

namespace mfp {
namespace dev {

// Tuning knobs (compile-time): CTAs per SM the CSR kernel is register-limited
// to, and whether long-row pieces take the first block indices.  Measured on
// the power-law configuration: 8 CTAs per SM and pieces last are fastest.
#ifndef MFP_CSR_MINBLOCKS
#define MFP_CSR_MINBLOCKS 8
#endif
// CTAs per SM the FP32 CSR vector kernel and the FP64 CSR kernels (scalar;
// vector and adaptive) are register-limited to.  Measured on the power-law,
// stencil and banded matrices in FP64: 5 for scalar (48 registers instead of
// 40 with spills) and 6 for the others are fastest.
#ifndef MFP_CSR_MINBLOCKS_VEC
#define MFP_CSR_MINBLOCKS_VEC 6
#endif
#ifndef MFP_CSR_MINBLOCKS64
#define MFP_CSR_MINBLOCKS64 5
#endif
#ifndef MFP_CSR_MINBLOCKS64_OTHER
#define MFP_CSR_MINBLOCKS64_OTHER 6
#endif
// CTAs per SM the warp-tile kernels (COO warp pass, warp-tile CSR) are
// register-limited to in FP32: 8 (32 registers) measured fastest on the
// power-law matrix (COO 0.169 -> 0.165 ms, CSR vector 0.187 -> 0.181 ms,
// hybrid tail 0.175 -> 0.169 ms against 6) and the stencil; SCOO keeps 6
// (0.195 ms against 0.203 at 8).  FP64: 5 measured faster than 4 and 6.
#ifndef MFP_COO_MINBLOCKS
#define MFP_COO_MINBLOCKS 8
#endif
#ifndef MFP_SCOO_MINBLOCKS
#define MFP_SCOO_MINBLOCKS 6
#endif
#ifndef MFP_COO_MINBLOCKS64
#define MFP_COO_MINBLOCKS64 5
#endif
#ifndef MFP_PIECES_FIRST
#define MFP_PIECES_FIRST 0
#endif

constexpr int kBlock = 256;   // threads per CTA for every kernel
constexpr int kEpt = 8;       // staged elements per thread
constexpr int kChunk = kBlock * kEpt;  // elements staged per phase
constexpr int kChunkPad = kChunk + 64; // room for the alignment offset and swizzle

// Shared-memory swizzle: XOR the low 5 bits of an index with bits 5..9.
// Rows walked one element at a time by consecutive threads (stride = row
// length) and per-thread contiguous ranges (stride 8) both hit 32 banks.
__device__ __forceinline__ uint32_t swz(uint32_t i) { return i ^ ((i >> 5) & 31u); }

// Store elements i..i+3 (i a multiple of 4) of a swizzled array with one
// 16-byte (float) or two 16-byte (double) stores.
template <typename T>
__device__ __forceinline__ void store_group4(T *dst, uint32_t i, const T (&v)[4]);
template <>
__device__ __forceinline__ void store_group4<float>(float *dst, uint32_t i, const float (&v)[4]) {
  const uint32_t s = (i >> 5) & 31u, m = s & 3u;
  const float a0 = (m & 1u) ? v[1] : v[0], a1 = (m & 1u) ? v[0] : v[1];
  const float a2 = (m & 1u) ? v[3] : v[2], a3 = (m & 1u) ? v[2] : v[3];
  float4 w;
  w.x = (m & 2u) ? a2 : a0;
  w.y = (m & 2u) ? a3 : a1;
  w.z = (m & 2u) ? a0 : a2;
  w.w = (m & 2u) ? a1 : a3;
  *reinterpret_cast<float4 *>(dst + (i ^ (s & ~3u))) = w;
}
template <>
__device__ __forceinline__ void store_group4<double>(double *dst, uint32_t i, const double (&v)[4]) {
  const uint32_t s = (i >> 5) & 31u, m = s & 3u;
  const double a0 = (m & 1u) ? v[1] : v[0], a1 = (m & 1u) ? v[0] : v[1];
  const double a2 = (m & 1u) ? v[3] : v[2], a3 = (m & 1u) ? v[2] : v[3];
  double2 w0, w1;
  w0.x = (m & 2u) ? a2 : a0;
  w0.y = (m & 2u) ? a3 : a1;
  w1.x = (m & 2u) ? a0 : a2;
  w1.y = (m & 2u) ? a1 : a3;
  double *g = dst + (i ^ (s & ~3u));
  reinterpret_cast<double2 *>(g)[0] = w0;
  reinterpret_cast<double2 *>(g)[1] = w1;
}
template <typename T>
__device__ __forceinline__ void store_group4_u32(uint32_t *dst, uint32_t i, const uint32_t (&v)[4]) {
  const uint32_t s = (i >> 5) & 31u, m = s & 3u;
  const uint32_t a0 = (m & 1u) ? v[1] : v[0], a1 = (m & 1u) ? v[0] : v[1];
  const uint32_t a2 = (m & 1u) ? v[3] : v[2], a3 = (m & 1u) ? v[2] : v[3];
  uint4 w;
  w.x = (m & 2u) ? a2 : a0;
  w.y = (m & 2u) ? a3 : a1;
  w.z = (m & 2u) ? a0 : a2;
  w.w = (m & 2u) ? a1 : a3;
  *reinterpret_cast<uint4 *>(dst + (i ^ (s & ~3u))) = w;
}

// x source: global memory, or a shared-memory window [lo, lo + n).
template <typename T>
struct x_global {
  const T *__restrict__ x;
  __device__ __forceinline__ T operator()(uint32_t c) const { return ld_x(x + c); }
};
template <typename T>
struct x_window {
  const T *s_x;
  uint32_t lo;
  __device__ __forceinline__ T operator()(uint32_t c) const { return s_x[c - lo]; }
};

// Stage products of elements [a, b) (b - (a & ~3) <= kChunkPad - 32) into
// dst at swizzled local index e - (a & ~3); optionally also their row ids.
template <typename T, bool VEC, bool ROWS, typename XS>
__device__ __forceinline__ void stage(const T *__restrict__ vals, const uint32_t *__restrict__ cols,
                                      const uint32_t *__restrict__ rows, XS xs, uint32_t a,
                                      uint32_t b, T *__restrict__ dst, uint32_t *__restrict__ dst_rows,
                                      uint64_t pol) {
  const uint32_t base = a & ~3u;
  uint32_t s0 = a, s1 = b;  // scalar part(s)
  if (VEC) {
    const uint32_t a4 = (a + 3u) & ~3u, b4 = b & ~3u;
    if (a4 < b4) {
      if (threadIdx.x < a4 - a) {
        const uint32_t e = a + threadIdx.x;
        dst[swz(e - base)] = mul_rn(ld_stream1(vals + e, pol), xs(ld_stream1(cols + e, pol)));
        if (ROWS) dst_rows[swz(e - base)] = ld_stream1(rows + e, pol);
      }
      if (threadIdx.x < b - b4) {
        const uint32_t e = b4 + threadIdx.x;
        dst[swz(e - base)] = mul_rn(ld_stream1(vals + e, pol), xs(ld_stream1(cols + e, pol)));
        if (ROWS) dst_rows[swz(e - base)] = ld_stream1(rows + e, pol);
      }
      const uint32_t ng = (b4 - a4) >> 2;
      uint32_t g = threadIdx.x;
      for (; g + kBlock < ng; g += 2 * kBlock) {
        const uint32_t e0 = a4 + 4u * g, e1 = e0 + 4u * kBlock;
        T v0[4], v1[4];
        uint32_t c0[4], c1[4], r0[4], r1[4];
        ld_stream4(vals + e0, v0, pol);
        ld_stream4(cols + e0, c0, pol);
        ld_stream4(vals + e1, v1, pol);
        ld_stream4(cols + e1, c1, pol);
        if (ROWS) {
          ld_stream4(rows + e0, r0, pol);
          ld_stream4(rows + e1, r1, pol);
        }
        T p0[4], p1[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) p0[k] = mul_rn(v0[k], xs(c0[k]));
#pragma unroll
        for (int k = 0; k < 4; ++k) p1[k] = mul_rn(v1[k], xs(c1[k]));
        store_group4<T>(dst, e0 - base, p0);
        store_group4<T>(dst, e1 - base, p1);
        if (ROWS) {
          store_group4_u32<T>(dst_rows, e0 - base, r0);
          store_group4_u32<T>(dst_rows, e1 - base, r1);
        }
      }
      if (g < ng) {
        const uint32_t e0 = a4 + 4u * g;
        T v0[4];
        uint32_t c0[4], r0[4];
        ld_stream4(vals + e0, v0, pol);
        ld_stream4(cols + e0, c0, pol);
        if (ROWS) ld_stream4(rows + e0, r0, pol);
        T p0[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) p0[k] = mul_rn(v0[k], xs(c0[k]));
        store_group4<T>(dst, e0 - base, p0);
        if (ROWS) store_group4_u32<T>(dst_rows, e0 - base, r0);
      }
      return;
    }
  }
  for (uint32_t e = s0 + threadIdx.x; e < s1; e += kBlock) {
    dst[swz(e - base)] = mul_rn(ld_stream1(vals + e, pol), xs(ld_stream1(cols + e, pol)));
    if (ROWS) dst_rows[swz(e - base)] = ld_stream1(rows + e, pol);
  }
}

// ---------------------------------------------------------------------------
// Block segmented reduction over staged (product, row) pairs.
// Local indices [off, off + n), n <= kChunk, off < 4, rows non-decreasing.
// Thread t owns [off + t*kEpt, off + (t+1)*kEpt).  Calls
//   emit(row, total, is_first_segment, is_last_segment)
// exactly once per row present in the chunk, from one thread, and
//   gap(lo, hi) for every run of absent rows lo..hi-1 strictly between two
// present rows.  Sums are deterministic (fixed order for a given chunking).
// ---------------------------------------------------------------------------
template <typename T>
struct seg_scan_smem {
  T warp_v[kBlock / 32];
  uint32_t warp_f[kBlock / 32];
  T prefix_v[kBlock / 32];
  uint32_t prefix_f[kBlock / 32];
};

template <typename T, typename Emit, typename Gap>
__device__ __forceinline__ void block_segmented_reduce(const T *s_prod, const uint32_t *s_row,
                                                       uint32_t off, uint32_t n, Emit emit, Gap gap,
                                                       seg_scan_smem<T> &sm) {
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t end = off + n;
  const uint32_t i0 = off + t * kEpt;
  const uint32_t i1 = min(i0 + kEpt, end);
  const bool active = i0 < end;
  const uint32_t row_first_chunk = s_row[swz(off)];
  const uint32_t row_last_chunk = s_row[swz(end - 1)];

  uint32_t first_row = 0, last_row = 0;
  T first_sum = T(0), cur = T(0);
  bool multi = false, head_cont = false;
  if (active) {
    first_row = s_row[swz(i0)];
    if (i0 > off) {
      const uint32_t prev = s_row[swz(i0 - 1)];
      head_cont = (prev == first_row);
      if (!head_cont && first_row > prev + 1u) gap(prev + 1u, first_row);
    }
    uint32_t r = first_row;
    cur = s_prod[swz(i0)];
    for (uint32_t i = i0 + 1; i < i1; ++i) {
      const uint32_t ri = s_row[swz(i)];
      const T p = s_prod[swz(i)];
      if (ri != r) {
        if (!multi) {
          first_sum = cur;
          multi = true;
        } else {
          emit(r, cur, false, false);
        }
        if (ri > r + 1u) gap(r + 1u, ri);
        r = ri;
        cur = p;
      } else {
        cur = add_rn(cur, p);
      }
    }
    last_row = r;
  }
  // Segmented inclusive scan of the last-run partials across threads.  A
  // thread continues its left neighbour's chain only if it holds a single run
  // of the row that the neighbour's last run has.
  uint32_t f = (active && !multi && head_cont) ? 0u : 1u;
  T v = active ? cur : T(0);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T ov = __shfl_up_sync(0xffffffffu, v, o);
    const uint32_t of = __shfl_up_sync(0xffffffffu, f, o);
    if (lane >= (uint32_t)o) {
      if (!f) v = add_rn(ov, v);
      f |= of;
    }
  }
  if (lane == 31) {
    sm.warp_v[warp] = v;
    sm.warp_f[warp] = f;
  }
  __syncthreads();
  if (warp == 0) {
    // exclusive prefix over warps (kBlock/32 <= 32 entries)
    const uint32_t nw = kBlock / 32;
    T wv = lane < nw ? sm.warp_v[lane] : T(0);
    uint32_t wf = lane < nw ? sm.warp_f[lane] : 1u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T ov = __shfl_up_sync(0xffffffffu, wv, o);
      const uint32_t of = __shfl_up_sync(0xffffffffu, wf, o);
      if (lane >= (uint32_t)o) {
        if (!wf) wv = add_rn(ov, wv);
        wf |= of;
      }
    }
    // inclusive (wv, wf) at lane w -> exclusive for warp w+1
    const T pv = __shfl_up_sync(0xffffffffu, wv, 1);
    const uint32_t pf = __shfl_up_sync(0xffffffffu, wf, 1);
    if (lane < nw) {
      sm.prefix_v[lane] = lane == 0 ? T(0) : pv;
      sm.prefix_f[lane] = lane == 0 ? 1u : pf;
    }
  }
  __syncthreads();
  if (!f && warp > 0) v = add_rn(sm.prefix_v[warp], v);  // chain reaches into previous warps
  // S_{t-1}
  T left = __shfl_up_sync(0xffffffffu, v, 1);
  if (lane == 0) left = warp > 0 ? sm.prefix_v[warp] : T(0);

  if (!active) return;
  const bool tail_cont = (i1 < end) && (s_row[swz(i1)] == last_row);
  if (multi) {
    if (head_cont)
      emit(first_row, add_rn(left, first_sum), first_row == row_first_chunk, first_row == row_last_chunk);
    else
      emit(first_row, first_sum, first_row == row_first_chunk, first_row == row_last_chunk);
    if (!tail_cont) emit(last_row, cur, false, last_row == row_last_chunk);
  } else if (!tail_cont) {
    emit(last_row, v, last_row == row_first_chunk, last_row == row_last_chunk);
  }
}

// ---------------------------------------------------------------------------
// Register-resident variant for row-sorted element streams (COO tiles, the
// hybrid's COO tail, SCOO slices).  Thread t owns the 8 consecutive elements
// [g, g + 8) of the chunk, g = (c0 & ~7) + 8 t, clipped to [c0, c1): it loads
// them with 16-byte loads straight into registers (consecutive threads,
// consecutive 32-byte pieces: coalesced), issues their 8 x gathers together,
// and runs the same thread-sequential run sums and carry scan as
// block_segmented_reduce, without staging products and row ids through
// shared memory.
// ---------------------------------------------------------------------------
template <typename T, int VEC, typename XS>
__device__ __forceinline__ uint32_t load_run_group(const T *__restrict__ vals, const uint32_t *__restrict__ cols,
                                                   const uint32_t *__restrict__ rows, XS xs, uint32_t g,
                                                   uint32_t c0, uint32_t c1, T (&p)[kEpt], uint32_t (&r)[kEpt],
                                                   uint32_t &i0, uint64_t pol) {
  static_assert(kEpt == 8, "a group is one 8-element vector or two 4-element vectors");
  i0 = max(g, c0);
  const uint32_t i1 = min(g + kEpt, c1);
  if (i0 >= i1) return 0u;
  const uint32_t cnt = i1 - i0;
  if (VEC == 2 && cnt == kEpt) {  // i0 == g, a multiple of 8: 32-byte aligned
    T v[8];
    uint32_t k[8];
    ld_stream8(vals + i0, v, pol);
    ld_stream8(cols + i0, k, pol);
    ld_stream8(rows + i0, r, pol);
    T xv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) xv[j] = xs(k[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j) p[j] = mul_rn(v[j], xv[j]);
  } else if (VEC == 1 && cnt == kEpt) {  // 16-byte aligned: two loads per array
    T v0[4], v1[4];
    uint32_t k0[4], k1[4], q0[4], q1[4];
    ld_stream4(vals + i0, v0, pol);
    ld_stream4(vals + i0 + 4, v1, pol);
    ld_stream4(cols + i0, k0, pol);
    ld_stream4(cols + i0 + 4, k1, pol);
    ld_stream4(rows + i0, q0, pol);
    ld_stream4(rows + i0 + 4, q1, pol);
    T x0[4], x1[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x0[k] = xs(k0[k]);
      x1[k] = xs(k1[k]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      p[k] = mul_rn(v0[k], x0[k]);
      p[4 + k] = mul_rn(v1[k], x1[k]);
      r[k] = q0[k];
      r[4 + k] = q1[k];
    }
  } else {
#pragma unroll
    for (uint32_t k = 0; k < kEpt; ++k) {
      if (k < cnt) {
        const uint32_t e = i0 + k;
        r[k] = ld_stream1(rows + e, pol);
        p[k] = mul_rn(ld_stream1(vals + e, pol), xs(ld_stream1(cols + e, pol)));
      }
    }
  }
  return cnt;
}

// block_segmented_reduce over register-held runs.  cnt: the thread's element
// count (0 = inactive); i0, i1 = i0 + cnt its element range; c0, c1 the
// chunk; row_at(e) the row of element e (read for the neighbours across
// warps and the chunk's first and last rows).
struct rows_u32 {
  const uint32_t *__restrict__ p;
  __device__ __forceinline__ uint32_t operator()(uint32_t e) const { return __ldg(p + e); }
};
template <typename T, typename Emit, typename Gap, typename RowAt>
__device__ __forceinline__ void block_segmented_reduce_regs(const T (&pr)[kEpt], const uint32_t (&rw)[kEpt],
                                                            uint32_t cnt, uint32_t i0, uint32_t c0, uint32_t c1,
                                                            RowAt row_at, Emit emit, Gap gap, seg_scan_smem<T> &sm) {
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const bool active = cnt > 0;
  const uint32_t i1 = i0 + cnt;
  const uint32_t row_first_chunk = row_at(c0);
  const uint32_t row_last_chunk = row_at(c1 - 1u);
  uint32_t first_row = active ? rw[0] : 0u, last_row = 0u;
  T first_sum = T(0), cur = T(0);
  bool multi = false;
  if (active) {
    uint32_t r = first_row;
    cur = pr[0];
#pragma unroll
    for (uint32_t k = 1; k < kEpt; ++k) {
      if (k < cnt) {
        const uint32_t ri = rw[k];
        if (ri != r) {
          if (!multi) {
            first_sum = cur;
            multi = true;
          } else {
            emit(r, cur, false, false);
          }
          if (ri > r + 1u) gap(r + 1u, ri);
          r = ri;
          cur = pr[k];
        } else {
          cur = add_rn(cur, pr[k]);
        }
      }
    }
    last_row = r;
  }
  // neighbours' rows: the previous element (i0 - 1) is the last element of
  // thread t - 1, the next (i1) the first of thread t + 1
  uint32_t prev_row = __shfl_up_sync(0xffffffffu, last_row, 1);
  uint32_t next_row = __shfl_down_sync(0xffffffffu, first_row, 1);
  if (lane == 0) prev_row = (active && i0 > c0) ? row_at(i0 - 1u) : 0u;
  if (lane == 31) next_row = (active && i1 < c1) ? row_at(i1) : 0u;
  const bool has_prev = active && i0 > c0, has_next = active && i1 < c1;
  bool head_cont = false;
  if (has_prev) {
    head_cont = prev_row == first_row;
    if (!head_cont && first_row > prev_row + 1u) gap(prev_row + 1u, first_row);
  }
  uint32_t f = (active && !multi && head_cont) ? 0u : 1u;
  T v = active ? cur : T(0);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T ov = __shfl_up_sync(0xffffffffu, v, o);
    const uint32_t of = __shfl_up_sync(0xffffffffu, f, o);
    if (lane >= (uint32_t)o) {
      if (!f) v = add_rn(ov, v);
      f |= of;
    }
  }
  if (lane == 31) {
    sm.warp_v[warp] = v;
    sm.warp_f[warp] = f;
  }
  __syncthreads();
  if (warp == 0) {
    const uint32_t nw = kBlock / 32;
    T wv = lane < nw ? sm.warp_v[lane] : T(0);
    uint32_t wf = lane < nw ? sm.warp_f[lane] : 1u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T ov = __shfl_up_sync(0xffffffffu, wv, o);
      const uint32_t of = __shfl_up_sync(0xffffffffu, wf, o);
      if (lane >= (uint32_t)o) {
        if (!wf) wv = add_rn(ov, wv);
        wf |= of;
      }
    }
    const T pv = __shfl_up_sync(0xffffffffu, wv, 1);
    const uint32_t pf = __shfl_up_sync(0xffffffffu, wf, 1);
    if (lane < nw) {
      sm.prefix_v[lane] = lane == 0 ? T(0) : pv;
      sm.prefix_f[lane] = lane == 0 ? 1u : pf;
    }
  }
  __syncthreads();
  if (!f && warp > 0) v = add_rn(sm.prefix_v[warp], v);
  T left = __shfl_up_sync(0xffffffffu, v, 1);
  if (lane == 0) left = warp > 0 ? sm.prefix_v[warp] : T(0);
  if (!active) return;
  const bool tail_cont = has_next && next_row == last_row;
  if (multi) {
    if (head_cont)
      emit(first_row, add_rn(left, first_sum), first_row == row_first_chunk, first_row == row_last_chunk);
    else
      emit(first_row, first_sum, first_row == row_first_chunk, first_row == row_last_chunk);
    if (!tail_cont) emit(last_row, cur, false, last_row == row_last_chunk);
  } else if (!tail_cont) {
    emit(last_row, v, last_row == row_first_chunk, last_row == row_last_chunk);
  }
}

// acc + p[lo] + p[lo+1] + ... + p[hi-1] in that order (exact CSR order);
// UNROLL keeps four shared-memory loads in flight per step (faster for long
// segments, costs registers).
template <typename T, bool UNROLL = true>
__device__ __forceinline__ T seq_sum(T acc, const T *prod, uint32_t lo, uint32_t hi) {
  uint32_t i = lo;
  for (; UNROLL && i + 4 <= hi; i += 4) {
    const T a = prod[swz(i)], b = prod[swz(i + 1)], c = prod[swz(i + 2)], d = prod[swz(i + 3)];
    acc = add_rn(acc, a);
    acc = add_rn(acc, b);
    acc = add_rn(acc, c);
    acc = add_rn(acc, d);
  }
  for (; i < hi; ++i) acc = add_rn(acc, prod[swz(i)]);
  return acc;
}

// Lane-strided partial sum over [lo, hi) with stride L starting at lo + lane,
// four loads in flight per step (same order as the one-at-a-time loop).
template <typename T, bool UNROLL = true>
__device__ __forceinline__ T strided_sum(const T *prod, uint32_t lo, uint32_t hi, uint32_t lane, uint32_t L) {
  T acc = T(0);
  uint32_t i = lo + lane;
  for (; UNROLL && i + 3 * L < hi; i += 4 * L) {
    const T a = prod[swz(i)], b = prod[swz(i + L)], c = prod[swz(i + 2 * L)], d = prod[swz(i + 3 * L)];
    acc = add_rn(acc, a);
    acc = add_rn(acc, b);
    acc = add_rn(acc, c);
    acc = add_rn(acc, d);
  }
  for (; i < hi; i += L) acc = add_rn(acc, prod[swz(i)]);
  return acc;
}

// ---------------------------------------------------------------------------
// Long-row pieces (CSR family)
// ---------------------------------------------------------------------------
struct long_piece {
  uint32_t row;
  uint32_t e0, e1;     // element range of this piece
  uint32_t slot_base;  // first partial slot of the row (pieces of a row are consecutive)
  uint32_t piece;      // index of this piece within the row
  uint32_t npieces;
  uint32_t counter;    // arrival counter of the row
  uint32_t fp64;       // 1: accumulate in FP64 (rows longer than 4096)
};

// Whole-CTA dot product of vals[e] * x[cols[e]] over e in [a, b).  Each
// thread takes 8 elements per round (two 4-element groups) and issues all of
// a round's streaming loads before its first x gather, so a round costs one
// DRAM and one L2 round trip.  Acc is T (plain) or comp_sum (FP64).
template <typename T, bool VEC>
struct acc_plain {
  T v = T(0);
  __device__ __forceinline__ void add(T p) { v = add_rn(v, p); }
  __device__ __forceinline__ void add_prod(T a, T xv) { v = add_rn(v, mul_rn(a, xv)); }
};
template <typename T, bool VEC>
struct acc_fp64 {
  comp_sum v;
  __device__ __forceinline__ void add_prod(T a, T xv) { v.add(__dmul_rn((double)a, (double)xv)); }
};

template <typename T, bool VEC, typename ACC>
__device__ __forceinline__ void cta_range_dot(const T *__restrict__ vals, const uint32_t *__restrict__ cols,
                                              const T *__restrict__ x, uint32_t a, uint32_t b, ACC &acc,
                                              uint64_t pol) {
  uint32_t s0 = a, s1 = b;
  if (VEC) {
    const uint32_t a4 = (a + 3u) & ~3u, b4 = b & ~3u;
    if (a4 < b4) {
      const uint32_t ng = (b4 - a4) >> 2;
      uint32_t g = threadIdx.x;
      for (; g + kBlock < ng; g += 2 * kBlock) {
        T v[2][4];
        uint32_t c[2][4];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          ld_stream4(vals + a4 + 4u * (g + u * kBlock), v[u], pol);
          ld_stream4(cols + a4 + 4u * (g + u * kBlock), c[u], pol);
        }
        T xv[2][4];
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int k = 0; k < 4; ++k) xv[u][k] = ld_x(x + c[u][k]);
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int k = 0; k < 4; ++k) acc.add_prod(v[u][k], xv[u][k]);
      }
      for (; g < ng; g += kBlock) {
        T v[4];
        uint32_t c[4];
        ld_stream4(vals + a4 + 4u * g, v, pol);
        ld_stream4(cols + a4 + 4u * g, c, pol);
        T xv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) xv[k] = ld_x(x + c[k]);
#pragma unroll
        for (int k = 0; k < 4; ++k) acc.add_prod(v[k], xv[k]);
      }
      if (threadIdx.x < a4 - a) {
        const uint32_t e = a + threadIdx.x;
        acc.add_prod(ld_stream1(vals + e, pol), ld_x(x + ld_stream1(cols + e, pol)));
      }
      if (threadIdx.x < b - b4) {
        const uint32_t e = b4 + threadIdx.x;
        acc.add_prod(ld_stream1(vals + e, pol), ld_x(x + ld_stream1(cols + e, pol)));
      }
      return;
    }
  }
  uint32_t e = s0 + threadIdx.x;
  for (; e + 3 * kBlock < s1; e += 4 * kBlock) {
    T v[4];
    uint32_t c[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      v[u] = ld_stream1(vals + e + u * kBlock, pol);
      c[u] = ld_stream1(cols + e + u * kBlock, pol);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) acc.add_prod(v[u], ld_x(x + c[u]));
  }
  for (; e < s1; e += kBlock) acc.add_prod(ld_stream1(vals + e, pol), ld_x(x + ld_stream1(cols + e, pol)));
}

template <typename T, bool VEC>
__device__ __forceinline__ void run_piece(const long_piece &pc, const T *__restrict__ vals,
                                          const uint32_t *__restrict__ cols, const T *__restrict__ x,
                                          T *__restrict__ y, double *partials, uint32_t *counters,
                                          double *s_a, double *s_b, uint64_t pol) {
  double result;
  if (pc.fp64) {
    acc_fp64<T, VEC> acc;
    cta_range_dot<T, VEC>(vals, cols, x, pc.e0, pc.e1, acc, pol);
    result = block_reduce_comp<kBlock>(acc.v, s_a, s_b).value();
  } else {
    acc_plain<T, VEC> acc;
    cta_range_dot<T, VEC>(vals, cols, x, pc.e0, pc.e1, acc, pol);
    result = (double)block_reduce<T, kBlock>(acc.v, reinterpret_cast<T *>(s_a));
  }
  if (threadIdx.x != 0) return;
  if (pc.npieces == 1) {
    y[pc.row] = (T)result;
    return;
  }
  partials[pc.slot_base + pc.piece] = result;
  __threadfence();
  const uint32_t arrived = atomicAdd(counters + pc.counter, 1u);
  if (arrived == pc.npieces - 1) {
    __threadfence();
    comp_sum s;
    for (uint32_t k = 0; k < pc.npieces; ++k) s.add(__ldcg(partials + pc.slot_base + k));
    y[pc.row] = (T)s.value();
    counters[pc.counter] = 0u;  // ready for the next launch
  }
}

// ---------------------------------------------------------------------------
// CSR family kernel: blocks [0, n_main) run the algorithm's main part,
// blocks [n_main, n_main + n_pieces) run long-row pieces.
// ---------------------------------------------------------------------------
template <typename T>
struct csr_args {
  uint32_t n_rows;
  const uint32_t *__restrict__ row_ptr;
  const uint32_t *__restrict__ cols;
  const T *__restrict__ vals;
  const T *__restrict__ x;
  T *__restrict__ y;
  uint32_t long_thr;    // rows with more elements are handled by pieces
  uint32_t assist_thr;  // scalar/vector: rows with more elements are reduced by a warp
  uint32_t lanes;       // CSR vector: lanes per row (power of two, 2..32)
  const uint32_t *__restrict__ row_blocks;  // CSR-Adaptive bins (n_main + 1 entries)
  uint32_t n_main;
  uint32_t n_pieces;
  const long_piece *__restrict__ pieces;
  double *partials;
  uint32_t *counters;
  // work item of each block index (w < n_main: row block / bin w, else piece
  // w - n_main), heaviest first; NULL = blocks in index order
  const uint32_t *__restrict__ order;
  // per row block (plan, row-block algorithms): element range [x, y);
  // z bit 0 = has a long row, bit 1 = has an assisted row
  const uint4 *__restrict__ blk;
};

template <typename T>
struct csr_smem {
  union {
    struct {
      uint32_t rp[kBlock + 1];
      uint32_t longs[kBlock];
      uint32_t assists[kBlock];
      uint32_t nlong, nassist;
      uint32_t wc[kBlock / 32];
      T acc[kBlock];
      __align__(16) T prod[kChunkPad];
    } m;
    struct {
      double a[kBlock / 32];
      double b[kBlock / 32];
    } p;
  };
};

// Ordered compaction of the threads whose flag is set; returns the count.
template <typename T>
__device__ __forceinline__ uint32_t compact_ordered(bool flag, uint32_t value, uint32_t *list,
                                                    csr_smem<T> &sm, uint32_t *count_slot) {
  const uint32_t t = threadIdx.x;
  const uint32_t ballot = __ballot_sync(0xffffffffu, flag);
  if ((t & 31u) == 0) sm.m.wc[t >> 5] = __popc(ballot);
  __syncthreads();
  if (t == 0) {
    uint32_t s = 0;
    for (int w = 0; w < kBlock / 32; ++w) {
      const uint32_t c = sm.m.wc[w];
      sm.m.wc[w] = s;
      s += c;
    }
    *count_slot = s;
  }
  __syncthreads();
  if (flag) list[sm.m.wc[t >> 5] + __popc(ballot & ((1u << (t & 31u)) - 1u))] = value;
  __syncthreads();
  return *count_slot;
}

// CSR scalar (MODE 0) and CSR vector (MODE 1) share the row-block skeleton:
// CTA b owns rows [b*256, b*256+256); the elements of its rows, minus rows
// above the long threshold, are staged in chunks; then
//   scalar: thread t adds the products of row t one by one in CSR order;
//   vector: row j is reduced by lane group j % (256/L), lane l taking the
//           elements rs + l + k*L, then a shuffle tree over the group;
// and in both, rows above the assist threshold are reduced by a warp.
//
// The reduction of one staged chunk [c0, c1) (local base `base`) for the rows
// [run_lo, run_hi) of the block.
template <typename T, int MODE>
__device__ __forceinline__ void rowblock_chunk(const csr_args<T> &A, csr_smem<T> &sm, uint32_t run_lo,
                                               uint32_t run_hi, uint32_t c0, uint32_t c1, uint32_t base, bool own,
                                               uint32_t rs, uint32_t re, uint32_t nassist, T &acc) {
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  if (MODE == 0) {
    if (own && t >= run_lo && t < run_hi) {
      const uint32_t lo = max(rs, c0), hi = min(re, c1);
      if (lo < hi) acc = seq_sum<T, false>(acc, sm.m.prod, lo - base, hi - base);
    }
  } else {
    const uint32_t L = A.lanes;
    // rows of the run that intersect [c0, c1): [jlo, jhi), by binary search
    uint32_t jlo, jhi;
    {
      uint32_t lo_ = run_lo, hi_ = run_hi;  // first j with rp[j + 1] > c0
      while (lo_ < hi_) {
        const uint32_t mid = (lo_ + hi_) >> 1;
        if (sm.m.rp[mid + 1] > c0) hi_ = mid; else lo_ = mid + 1;
      }
      jlo = lo_;
      hi_ = run_hi;  // first j with rp[j] >= c1
      while (lo_ < hi_) {
        const uint32_t mid = (lo_ + hi_) >> 1;
        if (sm.m.rp[mid] >= c1) hi_ = mid; else lo_ = mid + 1;
      }
      jhi = lo_;
    }
    const uint32_t G = kBlock / L, g = t / L, gl = t % L;
    const uint32_t rounds = (jhi - jlo + G - 1u) / G;  // uniform over the CTA
    for (uint32_t it = 0; it < rounds; ++it) {
      const uint32_t j = jlo + g + it * G;
      T part = T(0);
      bool valid = false;
      if (j < jhi) {
        const uint32_t js = sm.m.rp[j], je = sm.m.rp[j + 1];
        const uint32_t len = je - js;
        if (len <= A.assist_thr) {
          const uint32_t s = max(js, c0), e = min(je, c1);
          if (s < e) {
            valid = true;
            part = strided_sum(sm.m.prod, s - base, e - base, (gl - (s - js)) & (L - 1u), L);
          }
        }
      }
      part = group_reduce_down(part, (int)L);
      if (valid && gl == 0) sm.m.acc[j] = add_rn(sm.m.acc[j], part);
    }
  }
  // rows above the assist threshold: one warp per row segment
  for (uint32_t q = warp; q < nassist; q += kBlock / 32) {
    const uint32_t j = sm.m.assists[q];
    const uint32_t js = sm.m.rp[j], je = sm.m.rp[j + 1];
    const uint32_t s = max(js, c0), e = min(je, c1);
    if (s < e) {
      T part = strided_sum(sm.m.prod, s - base, e - base, (lane - (s - js)) & 31u, 32u);
      part = group_reduce_down(part, 32);
      if (lane == 0) sm.m.acc[j] = add_rn(sm.m.acc[j], part);
    }
  }
}

// Blocks without long rows (their element range [a, b) from the plan): the
// first chunk's loads and x gathers are issued together with the row_ptr
// window's, before the first barrier.  A separate instantiation (FAST), since
// the extra state costs registers: measured faster on long rows (banded 8M,
// mean 32: CSR scalar 0.424 -> 0.404 ms) and for lanes per row (0.669 ->
// 0.596 ms), slower on the power-law matrix (mean 7.5: 0.191 -> 0.199 ms).
template <typename T, int MODE, bool VEC>
__device__ __forceinline__ void csr_rowblock_fast(const csr_args<T> &A, csr_smem<T> &sm, uint64_t pol, uint32_t r0,
                                                  uint32_t nr, uint4 br) {
  const uint32_t t = threadIdx.x;
  const uint32_t a = br.x, b = br.y;
  for (uint32_t i = t; i <= nr; i += kBlock) sm.m.rp[i] = A.row_ptr[r0 + i];
  sm.m.acc[t] = T(0);
  uint32_t c0 = a, base = a & ~3u;
  uint32_t c1 = min(b, base + (uint32_t)kChunk);
  if (c0 < c1) stage<T, VEC, false>(A.vals, A.cols, nullptr, x_global<T>{A.x}, c0, c1, sm.m.prod, nullptr, pol);
  __syncthreads();
  const bool has = t < nr;
  const uint32_t rs = has ? sm.m.rp[t] : 0u, re = has ? sm.m.rp[t + 1] : 0u;
  const bool is_assist = has && (re - rs > A.assist_thr);
  uint32_t nassist = 0;
  if (br.z & 2u) nassist = compact_ordered<T>(is_assist, t, sm.m.assists, sm, &sm.m.nassist);
  T acc = T(0);
  for (;;) {
    rowblock_chunk<T, MODE>(A, sm, 0u, nr, c0, c1, base, has && !is_assist, rs, re, nassist, acc);
    __syncthreads();
    if (c1 >= b) break;
    c0 = c1;
    base = c0 & ~3u;
    c1 = min(b, base + (uint32_t)kChunk);
    stage<T, VEC, false>(A.vals, A.cols, nullptr, x_global<T>{A.x}, c0, c1, sm.m.prod, nullptr, pol);
    __syncthreads();
  }
  if (has) A.y[r0 + t] = (MODE == 0 && !is_assist) ? acc : sm.m.acc[t];
}

template <typename T, int MODE, bool VEC, bool FAST>
__device__ __forceinline__ void csr_rowblock_main(const csr_args<T> &A, csr_smem<T> &sm, uint64_t pol,
                                                  uint32_t blk) {
  const uint32_t r0 = blk * kBlock;
  const uint32_t nr = min((uint32_t)kBlock, A.n_rows - r0);
  const uint32_t t = threadIdx.x;
  if (FAST) {
    const uint4 br = A.blk[blk];
    if (!(br.z & 1u)) {
      csr_rowblock_fast<T, MODE, VEC>(A, sm, pol, r0, nr, br);
      return;
    }
  }
  for (uint32_t i = t; i <= nr; i += kBlock) sm.m.rp[i] = A.row_ptr[r0 + i];
  if (t < kBlock) sm.m.acc[t] = T(0);
  __syncthreads();
  const bool has = t < nr;
  const uint32_t rs = has ? sm.m.rp[t] : 0u, re = has ? sm.m.rp[t + 1] : 0u;
  const bool is_long = has && (re - rs > A.long_thr);
  const bool is_assist = has && !is_long && (re - rs > A.assist_thr);
  uint32_t nlong = 0, nassist = 0;
  if (__syncthreads_or(is_long || is_assist)) {
    nlong = compact_ordered<T>(is_long, t, sm.m.longs, sm, &sm.m.nlong);
    nassist = compact_ordered<T>(is_assist, t, sm.m.assists, sm, &sm.m.nassist);
  }
  T acc = T(0);  // scalar: running sum of this thread's row
  uint32_t run_lo = 0;
  for (uint32_t k = 0; k <= nlong; ++k) {
    const uint32_t run_hi = k < nlong ? sm.m.longs[k] : nr;
    if (run_lo < run_hi) {
      const uint32_t a = sm.m.rp[run_lo], b = sm.m.rp[run_hi];
      for (uint32_t c0 = a; c0 < b;) {
        const uint32_t base = c0 & ~3u;
        const uint32_t c1 = min(b, base + (uint32_t)kChunk);
        stage<T, VEC, false>(A.vals, A.cols, nullptr, x_global<T>{A.x}, c0, c1, sm.m.prod, nullptr, pol);
        __syncthreads();
        rowblock_chunk<T, MODE>(A, sm, run_lo, run_hi, c0, c1, base, has && !is_long && !is_assist, rs, re,
                                nassist, acc);
        __syncthreads();
        c0 = c1;
      }
    }
    run_lo = run_hi + 1;
  }
  if (has && !is_long) {
    if (MODE == 0 && !is_assist)
      A.y[r0 + t] = acc;
    else
      A.y[r0 + t] = sm.m.acc[t];
  }
}

// CSR-Adaptive: bin [row_blocks[b], row_blocks[b+1]).  Many-row bins are
// staged whole (the binning caps their elements at bin_nnz <= kChunk - 4) and
// reduced from shared memory by power-of-two lane groups; a single-row bin is
// reduced by the whole CTA straight from global memory; a single row above
// the long threshold belongs to pieces.  SEQ (CSR scalar on short rows): the
// same bins, each row summed by one thread in CSR order (rows above the
// assist threshold by a warp).
template <typename T, bool VEC, bool SEQ = false>
__device__ __forceinline__ void csr_adaptive_main(const csr_args<T> &A, csr_smem<T> &sm, uint64_t pol,
                                                  uint32_t blk) {
  const uint32_t rb = A.row_blocks[blk], re = A.row_blocks[blk + 1];
  const uint32_t nrows = re - rb;
  const uint32_t t = threadIdx.x;
  if (nrows == 0) return;
  const uint32_t a = A.row_ptr[rb], b = A.row_ptr[re];
  if (nrows == 1) {
    if (b - a > A.long_thr) return;
    acc_plain<T, VEC> acc;
    cta_range_dot<T, VEC>(A.vals, A.cols, A.x, a, b, acc, pol);
    const T r = block_reduce<T, kBlock>(acc.v, reinterpret_cast<T *>(sm.p.a));
    if (t == 0) A.y[rb] = r;
    return;
  }
  const uint32_t base = a & ~3u;
  for (uint32_t i = t; i <= nrows && i <= (uint32_t)kBlock; i += kBlock) sm.m.rp[i] = A.row_ptr[rb + i];
  if (t == 0) sm.m.nassist = 0u;
  if (b > a) stage<T, VEC, false>(A.vals, A.cols, nullptr, x_global<T>{A.x}, a, b, sm.m.prod, nullptr, pol);
  __syncthreads();
  // Rows are summed by power-of-two lane groups (one thread per row once the
  // bin holds more than 128 rows); a row longer than the assist threshold
  // that would get fewer than 32 lanes is queued for a whole warp instead, so
  // one long row does not hold up its CTA.  A row's sum order depends only on
  // its length and position, so results repeat bit for bit.
  // (at least 9 elements per queued row: a bin's <= 2044 elements queue at
  // most 227 rows, within the 256-entry list)
  const uint32_t athr = max(A.assist_thr, 8u);
  uint32_t tpr = 1;
  if (!SEQ && nrows <= (uint32_t)kBlock) {
    tpr = kBlock / nrows;  // >= 1
    tpr = tpr >= 32 ? 32u : (1u << (31 - __clz(tpr)));
    const uint32_t grp = t / tpr, lane = t % tpr;
    T acc = T(0);
    bool valid = grp < nrows;
    if (valid) {
      const uint32_t s = sm.m.rp[grp], e = sm.m.rp[grp + 1];
      if (tpr < 32 && e - s > athr) {
        valid = false;
        if (lane == 0) sm.m.assists[atomicAdd(&sm.m.nassist, 1u)] = grp;
      } else if (s < e) {
        acc = strided_sum(sm.m.prod, s - base, e - base, lane, tpr);
      }
    }
    acc = group_reduce_down(acc, (int)tpr);
    if (valid && lane == 0) A.y[rb + grp] = acc;
  } else {
    for (uint32_t r = t; r < nrows; r += kBlock) {
      const uint32_t s = A.row_ptr[rb + r], e = A.row_ptr[rb + r + 1];
      if (e - s > athr)
        sm.m.assists[atomicAdd(&sm.m.nassist, 1u)] = r;
      else
        A.y[rb + r] = s < e ? seq_sum(T(0), sm.m.prod, s - base, e - base) : T(0);
    }
  }
  if (tpr == 32) return;  // whole warps already
  __syncthreads();
  const uint32_t nas = sm.m.nassist, lane = t & 31u;
  for (uint32_t q = t >> 5; q < nas; q += kBlock / 32) {
    const uint32_t r = sm.m.assists[q];
    const uint32_t s = A.row_ptr[rb + r], e = A.row_ptr[rb + r + 1];
    T part = strided_sum(sm.m.prod, s - base, e - base, lane, 32u);
    part = group_reduce_down(part, 32);
    if (lane == 0) A.y[rb + r] = part;
  }
}

template <typename T, int ALGO, bool VEC, bool FAST = false>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? (ALGO != 1 ? MFP_CSR_MINBLOCKS : MFP_CSR_MINBLOCKS_VEC) : (ALGO == 0 ? MFP_CSR_MINBLOCKS64 : MFP_CSR_MINBLOCKS64_OTHER)) csr_kernel(const csr_args<T> A) {
  __shared__ csr_smem<T> sm;
  const uint64_t pol = policy_evict_first();
  // the hardware starts blocks in index order: with A.order the heaviest work
  // items (by element count) start first, which shortens the tail; without
  // it, long-row pieces take the first block indices or the last
  uint32_t w;
  if (A.order)
    w = A.order[blockIdx.x];
  else if (MFP_PIECES_FIRST)
    w = blockIdx.x < A.n_pieces ? A.n_main + blockIdx.x : blockIdx.x - A.n_pieces;
  else
    w = blockIdx.x;
  if (w >= A.n_main) {
    const long_piece pc = A.pieces[w - A.n_main];
    run_piece<T, VEC>(pc, A.vals, A.cols, A.x, A.y, A.partials, A.counters, sm.p.a, sm.p.b, pol);
    return;
  }
  const uint32_t b = w;
  if (ALGO == 2 || ALGO == 3)
    csr_adaptive_main<T, VEC, ALGO == 3>(A, sm, pol, b);
  else
    csr_rowblock_main<T, ALGO, VEC, FAST>(A, sm, pol, b);
}

// ---------------------------------------------------------------------------
// ELL: thread per 4 consecutive rows (16-byte loads per slot) or per row.
// Sums slots in order 0..width-1 like the reference loop, padding included.
// ---------------------------------------------------------------------------
template <typename T, bool VEC>
__global__ void __launch_bounds__(kBlock) ell_kernel(uint32_t n_rows, uint32_t width,
                                                     const T *__restrict__ data,
                                                     const uint32_t *__restrict__ cols,
                                                     const T *__restrict__ x, T *__restrict__ y) {
  const uint64_t pol = policy_evict_first();
  if (VEC) {
    const uint32_t r = (blockIdx.x * kBlock + threadIdx.x) * 4u;
    if (r >= n_rows) return;
    T acc[4] = {T(0), T(0), T(0), T(0)};
    const size_t stride = n_rows;
    for (uint32_t k = 0; k < width; ++k) {
      T v[4];
      uint32_t c[4];
      ld_stream4(data + k * stride + r, v, pol);
      ld_stream4(cols + k * stride + r, c, pol);
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[j] = add_rn(acc[j], mul_rn(v[j], ld_x(x + c[j])));
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) y[r + j] = acc[j];
  } else {
    const uint32_t r = blockIdx.x * kBlock + threadIdx.x;
    if (r >= n_rows) return;
    T acc = T(0);
    const size_t stride = n_rows;
    for (uint32_t k = 0; k < width; ++k) {
      const size_t o = k * stride + r;
      acc = add_rn(acc, mul_rn(ld_stream1(data + o, pol), ld_x(x + ld_stream1(cols + o, pol))));
    }
    y[r] = acc;
  }
}

// COO workspace header: the first and last row that hold elements (written
// by the warp pass, read by the fix-up pass, which zeroes the empty rows
// before and after them over its whole grid) and an error word that no COO
// kernel sets (the two passes have no waits).
struct coo_ws_header {
  uint32_t first_row;
  uint32_t last_row;
  uint32_t error;
  uint32_t pad;
};

constexpr uint32_t kNoRow = 0xffffffffu;

// ---------------------------------------------------------------------------
// COO in two passes (the default COO and hybrid-tail path).
// Pass 1, coo_warp_kernel: warp w reduces the 256 elements [256 w, 256 w + 256):
// lane l loads elements 8 l .. 8 l + 7 (32-byte loads) and sums its runs of
// equal rows in order; a segmented scan over the lanes (shuffles) carries the
// runs that cross lanes.  Rows that start and end inside the warp tile are
// written to y; the tile's head row (continuing from the previous tile) and
// tail row (continuing into the next) leave partial sums and flags in the
// workspace.  Pass 2, coo_fixup_kernel: one thread per warp tile finishes the
// row that starts in its tile and continues past it, adding the partials of
// the following tiles in tile order.  No block barriers and no waits between
// CTAs; every row is summed in a fixed order, so results repeat bit for bit.
// ---------------------------------------------------------------------------
constexpr uint32_t kWarpTile = 32u * kEpt;
constexpr uint32_t kHeadCont = 1u, kTailCont = 2u, kOneRow = 4u;

template <typename T>
struct coo_carry {
  T *head, *tail;
  uint32_t *flags, *tail_row;
};

// Row ids at or above n_rows (invalid input) are dropped, never written.
template <typename T, bool ACCUM>
__device__ __forceinline__ void coo_put(T *y, uint32_t n_rows, uint32_t row, T v) {
  if (row < n_rows) y[row] = ACCUM ? add_rn(y[row], v) : v;
}

// The reduction of one warp tile ending at c1 (of nnz elements), lane l's
// group starting at g0 + 8 l, the lane's cnt products pr and rows rw in hand
// (rows non-decreasing); prv / nxt are the rows of the elements just before
// and after the tile (kNoRow at the ends).
template <typename T, bool ACCUM>
__device__ __forceinline__ void warp_tile_reduce(uint32_t wt, uint32_t g0, uint32_t c1, uint32_t nnz,
                                                 uint32_t n_rows, const T (&pr)[kEpt], const uint32_t (&rw)[kEpt],
                                                 uint32_t cnt, uint32_t prv, uint32_t nxt, T *__restrict__ y,
                                                 const coo_carry<T> &cw, coo_ws_header *hdr) {
  const uint32_t lane = threadIdx.x & 31u;
  const bool active = cnt > 0;
  const uint32_t last_lane = (c1 - g0 - 1u) / kEpt;
  // runs inside the lane: the first and last run's sums; middle runs are whole rows
  uint32_t rf = kNoRow, rl = kNoRow;
  T sf = T(0), sl = T(0);
  if (active) {
    rf = rw[0];
    uint32_t cur = rf;
    T acc = pr[0];
    bool first = true;
#pragma unroll
    for (uint32_t k = 1; k < kEpt; ++k) {
      if (k < cnt) {
        if (rw[k] == cur) {
          acc = add_rn(acc, pr[k]);
        } else {
          if (first) sf = acc;
          else coo_put<T, ACCUM>(y, n_rows, cur, acc);
          if (!ACCUM)
            for (uint32_t r = cur + 1u; r < rw[k] && r < n_rows; ++r) y[r] = T(0);
          first = false;
          cur = rw[k];
          acc = pr[k];
        }
      }
    }
    if (first) sf = acc;
    sl = acc;
    rl = cur;  // the last run's row (no dynamic index: rw stays in registers)
  }
  const bool single = active && rf == rl;
  const uint32_t prev_last = __shfl_up_sync(0xffffffffu, rl, 1);
  const uint32_t next_first = __shfl_down_sync(0xffffffffu, rf, 1);
  const uint32_t tile_first = __shfl_sync(0xffffffffu, rf, 0);  // lane 0 is always active
  // the lane's first row continues the previous lane's last row
  const bool cont = active && lane > 0 && rf == prev_last;
  // Segmented inclusive scan of the lanes' last-run sums.  A lane closes its
  // segment unless it holds a single run that continues the previous lane;
  // rows are sorted, so an unclosed chain of lanes is one row and only the
  // sums travel by shuffle (the closed state of a window comes from the mask).
  const uint32_t closed = __ballot_sync(0xffffffffu, !(single && cont));
  T v = active ? (single ? sf : sl) : T(0);
#pragma unroll
  for (uint32_t o = 1; o < 32; o <<= 1) {
    const T a = __shfl_up_sync(0xffffffffu, v, o);
    // this lane's window is lanes (lane - o, lane]; add the window before it
    // unless a lane of this window closes the segment
    if (lane >= o && (closed & (((1u << o) - 1u) << (lane + 1u - o))) == 0u) v = add_rn(a, v);
  }
  const T cin_val = __shfl_up_sync(0xffffffffu, v, 1);  // lane - 1's chain: the row rf when cont
  if (!active) return;
  // the lane's first run, with the carry of the lanes before it
  const T ftot = cont ? add_rn(cin_val, sf) : sf;
  // rows are sorted: the first run reaches back beyond the tile exactly when
  // its row is the row before the tile
  const bool from_prev = rf == prv;
  // empty rows before this lane's first row; those before the matrix's first
  // row are left to the fix-up pass, which spreads them over its grid
  if (!ACCUM) {
    if (lane == 0 && prv == kNoRow) {
      hdr->first_row = rf;
    } else {
      const uint32_t lo = lane == 0 ? prv + 1u : prev_last + 1u;
      for (uint32_t r = lo; r < rf && r < n_rows; ++r) y[r] = T(0);
    }
  }
  const uint32_t after = lane < last_lane ? next_first : nxt;  // row of the element after this lane
  if (!single) {
    // first run ends inside the lane
    if (from_prev) cw.head[wt] = ftot;
    else coo_put<T, ACCUM>(y, n_rows, rf, ftot);
  }
  // last run (the first run too when single)
  const T ltot = single ? ftot : sl;
  const bool l_from_prev = single && from_prev;
  if (after != rl) {
    if (l_from_prev) cw.head[wt] = ltot;
    else coo_put<T, ACCUM>(y, n_rows, rl, ltot);
  } else if (lane == last_lane) {
    // the tail row continues into the next tile
    cw.tail[wt] = ltot;
    cw.tail_row[wt] = rl;
    if (l_from_prev) cw.head[wt] = ltot;
  }
  if (lane == last_lane) {
    uint32_t f = 0u;
    if (tile_first == prv) f |= kHeadCont;  // the tile's first row began in an earlier tile
    if (rl == nxt) f |= kTailCont;          // its last row goes on in the next tile
    if (tile_first == rl) f |= kOneRow;
    cw.flags[wt] = f;
    if (!ACCUM && c1 == nnz) hdr->last_row = rl;  // the fix-up pass zeroes the rows after it
  }
}

// A group of 8 elements whose rows are 16-bit offsets rel from a base row
// (compact COO / SCOO rows, 2 bytes per element instead of 4).  As
// load_run_group, with one 32-byte load per array for vals and cols (VEC 2)
// and one 16-byte load for the offsets.
template <typename T, int VEC, typename XS>
__device__ __forceinline__ uint32_t load_run_group16(const T *__restrict__ vals, const uint32_t *__restrict__ cols,
                                                     const uint16_t *__restrict__ rel, uint32_t base, XS xs,
                                                     uint32_t g, uint32_t c0, uint32_t c1, T (&p)[kEpt],
                                                     uint32_t (&r)[kEpt], uint32_t &i0, uint64_t pol) {
  i0 = max(g, c0);
  const uint32_t i1 = min(g + kEpt, c1);
  if (i0 >= i1) return 0u;
  const uint32_t cnt = i1 - i0;
  if (VEC == 2 && cnt == kEpt) {
    T v[8];
    uint32_t k[8], w[4];
    ld_stream8(vals + i0, v, pol);
    ld_stream8(cols + i0, k, pol);
    ld_stream8_u16(rel + i0, w, pol);
    T xv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) xv[j] = xs(k[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      p[j] = mul_rn(v[j], xv[j]);
      r[j] = base + ((j & 1) ? (w[j >> 1] >> 16) : (w[j >> 1] & 0xffffu));
    }
  } else {
#pragma unroll
    for (uint32_t k = 0; k < kEpt; ++k) {
      if (k < cnt) {
        const uint32_t e = i0 + k;
        r[k] = base + ld_stream_u16(rel + e, pol);
        p[k] = mul_rn(ld_stream1(vals + e, pol), xs(ld_stream1(cols + e, pol)));
      }
    }
  }
  return cnt;
}

// A group of 8 elements whose rows are 8-bit offsets rel from a base row
// (compact COO rows of tiles that span at most 256 rows): as
// load_run_group16, with one 8-byte load for the offsets.
template <typename T, int VEC, typename XS>
__device__ __forceinline__ uint32_t load_run_group8(const T *__restrict__ vals, const uint32_t *__restrict__ cols,
                                                    const uint8_t *__restrict__ rel, uint32_t base, XS xs,
                                                    uint32_t g, uint32_t c0, uint32_t c1, T (&p)[kEpt],
                                                    uint32_t (&r)[kEpt], uint32_t &i0, uint64_t pol) {
  i0 = max(g, c0);
  const uint32_t i1 = min(g + kEpt, c1);
  if (i0 >= i1) return 0u;
  const uint32_t cnt = i1 - i0;
  if (VEC == 2 && cnt == kEpt) {
    T v[8];
    uint32_t k[8], w[2];
    ld_stream8(vals + i0, v, pol);
    ld_stream8(cols + i0, k, pol);
    ld_stream8_u8(rel + i0, w, pol);
    T xv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) xv[j] = xs(k[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      p[j] = mul_rn(v[j], xv[j]);
      r[j] = base + ((w[j >> 2] >> (8 * (j & 3))) & 0xffu);
    }
  } else {
#pragma unroll
    for (uint32_t k = 0; k < kEpt; ++k) {
      if (k < cnt) {
        const uint32_t e = i0 + k;
        r[k] = base + ld_stream_u8(rel + e, pol);
        p[k] = mul_rn(ld_stream1(vals + e, pol), xs(ld_stream1(cols + e, pol)));
      }
    }
  }
  return cnt;
}

// Compact COO rows.  Step 1, one warp per 256-element tile: the tile's
// widest offset rows[e] - rows[tile's first element] (unsigned: an unsorted
// row counts as wide).  flag[0] |= 1 when some offset exceeds 65,535 (no
// 16-bit layout); flag[1] counts the tiles with an offset above 255.
__global__ void coo_rows_span_kernel(uint32_t nnz, const uint32_t *__restrict__ rows, uint32_t *flag) {
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
  if ((uint64_t)t * kWarpTile >= nnz) return;  // whole warps
  const uint32_t c0 = t * kWarpTile, c1 = min(nnz, c0 + kWarpTile), base = rows[c0];
  uint32_t dmax = 0;
  for (uint32_t e = c0 + lane; e < c1; e += 32u) dmax = max(dmax, rows[e] - base);
  dmax = __reduce_max_sync(0xffffffffu, dmax);
  if (lane == 0 && dmax > 0xffffu) atomicOr(flag, 1u);
  if (lane == 0 && dmax > 0xffu) atomicAdd(flag + 1, 1u);
}

// 8-bit layout, tile_base bit 31: the tile spans more than 256 rows and its
// rows come from the 32-bit array (rows below 2^31 only).
constexpr uint32_t kWideTile = 0x80000000u;

// Step 2, 8-bit layout (one warp per tile): each element's offset from its
// tile's first row, and that row per tile, marked kWideTile (offsets left 0)
// when an offset does not fit.
__global__ void coo_rows8_kernel(uint32_t nnz, const uint32_t *__restrict__ rows, uint32_t *__restrict__ tile_base,
                                 uint8_t *__restrict__ rel) {
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
  if ((uint64_t)t * kWarpTile >= nnz) return;
  const uint32_t c0 = t * kWarpTile, c1 = min(nnz, c0 + kWarpTile), base = rows[c0];
  uint32_t dmax = 0;
  for (uint32_t e = c0 + lane; e < c1; e += 32u) dmax = max(dmax, rows[e] - base);
  const bool wide = __reduce_max_sync(0xffffffffu, dmax) > 0xffu;
  for (uint32_t e = c0 + lane; e < c1; e += 32u) rel[e] = wide ? 0u : (uint8_t)(rows[e] - base);
  if (lane == 0) tile_base[t] = base | (wide ? kWideTile : 0u);
}

// Step 2, 16-bit layout (every offset fits): offsets and the first row per tile.
__global__ void coo_rows16_kernel(uint32_t nnz, const uint32_t *__restrict__ rows, uint32_t *__restrict__ tile_base,
                                  uint16_t *__restrict__ rel) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  const uint32_t t = e / kWarpTile;
  const uint32_t base = rows[t * kWarpTile];
  if (e % kWarpTile == 0) tile_base[t] = base;
  rel[e] = (uint16_t)(rows[e] - base);
}

// Compact SCOO rows: r_index[e] - s * slice_size for the elements of slice s
// (one CTA per slice); *flag |= 1 when an offset exceeds 65,535.
__global__ void scoo_rows16_kernel(uint32_t slice_size, const uint32_t *__restrict__ slices_ptr,
                                   const uint32_t *__restrict__ rows, uint16_t *__restrict__ rel, uint32_t *flag) {
  const uint32_t s = blockIdx.x;
  const uint32_t row0 = s * slice_size;
  for (uint32_t e = slices_ptr[s] + threadIdx.x; e < slices_ptr[s + 1]; e += blockDim.x) {
    const uint32_t d = rows[e] - row0;
    if (d > 0xffffu) atomicOr(flag, 1u);
    rel[e] = (uint16_t)d;
  }
}

// R16 / R8: rows as 16-bit offsets rel / 8-bit offsets rel8 from
// tile_base[tile] (compact COO rows; R8 with WIDE: some tiles read rows).
template <typename T, int VEC, bool ACCUM, bool R16 = false, bool R8 = false, bool WIDE = false>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? MFP_COO_MINBLOCKS : MFP_COO_MINBLOCKS64)
    coo_warp_kernel(uint32_t n_rows, uint32_t nnz, const T *__restrict__ vals, const uint32_t *__restrict__ cols,
                    const uint32_t *__restrict__ rows, const T *__restrict__ x, T *__restrict__ y,
                    coo_carry<T> cw, coo_ws_header *hdr, const uint16_t *__restrict__ rel = nullptr,
                    const uint32_t *__restrict__ tile_base = nullptr, const uint8_t *__restrict__ rel8 = nullptr) {
  if (ACCUM) griddep_wait();  // y holds the ELL part written by the preceding launch
  const uint64_t pol = policy_evict_first();
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t wt = blockIdx.x * (kBlock / 32u) + (threadIdx.x >> 5);
  if ((uint64_t)wt * kWarpTile >= nnz) return;  // whole warps only
  const uint32_t c0 = wt * kWarpTile, c1 = min(nnz, c0 + kWarpTile);
  T pr[kEpt];
  uint32_t rw[kEpt], i0 = 0;
  uint32_t cnt, prv, nxt;
  if (R8) {
    // WIDE: a tile marked kWideTile takes its rows from the 32-bit array; its
    // loads go out after the gathers, so other tiles wait for nothing extra
    const uint32_t tb = __ldg(tile_base + wt);
    cnt = load_run_group8<T, VEC>(vals, cols, rel8, WIDE ? tb & ~kWideTile : tb, x_global<T>{x}, c0 + lane * kEpt,
                                  c0, c1, pr, rw, i0, pol);
    if (WIDE && (tb & kWideTile)) {
#pragma unroll
      for (uint32_t k = 0; k < kEpt; ++k)
        if (k < cnt) rw[k] = __ldg(rows + i0 + k);
    }
    if (WIDE) {
      prv = kNoRow;  // row before the tile
      if (c0 > 0) {
        const uint32_t pb = __ldg(tile_base + wt - 1u);
        prv = (pb & kWideTile) ? __ldg(rows + c0 - 1u) : pb + ld_stream_u8(rel8 + c0 - 1u, pol);
      }
      nxt = c1 < nnz ? __ldg(tile_base + wt + 1u) & ~kWideTile : kNoRow;  // the next tile's first row
    } else {
      prv = c0 > 0 ? __ldg(tile_base + wt - 1u) + ld_stream_u8(rel8 + c0 - 1u, pol) : kNoRow;
      nxt = c1 < nnz ? __ldg(tile_base + wt + 1u) : kNoRow;
    }
  } else if (R16) {
    cnt = load_run_group16<T, VEC>(vals, cols, rel, __ldg(tile_base + wt), x_global<T>{x}, c0 + lane * kEpt, c0, c1,
                                   pr, rw, i0, pol);
    prv = c0 > 0 ? __ldg(tile_base + wt - 1u) + ld_stream_u16(rel + c0 - 1u, pol) : kNoRow;  // row before the tile
    nxt = c1 < nnz ? __ldg(tile_base + wt + 1u) : kNoRow;  // row after the tile: the next tile's base
  } else {
    cnt = load_run_group<T, VEC>(vals, cols, rows, x_global<T>{x}, c0 + lane * kEpt, c0, c1, pr, rw, i0, pol);
    prv = c0 > 0 ? __ldg(rows + c0 - 1u) : kNoRow;  // row before the tile
    nxt = c1 < nnz ? __ldg(rows + c1) : kNoRow;     // row after the tile
  }
  warp_tile_reduce<T, ACCUM>(wt, c0, c1, nnz, n_rows, pr, rw, cnt, prv, nxt, y, cw, hdr);
}

// ---------------------------------------------------------------------------
// CSR in warp tiles: the COO warp pass with each element's row taken from
// row_ptr instead of a stored row id.  Warp w owns the 256 elements
// [256 w, 256 w + 256); while their values, column ids and x gathers are in
// flight, the warp reads the row starts that fall inside the tile
// (row_ptr[prev + 1 ...], 32 per round; prev = the row of element 256 w - 1,
// from the plan), counts them per element position in shared memory, and a
// prefix count gives every element its row.  The reduction and the fix-up
// pass are the COO ones.  Used for CSR vector on short rows: the lanes of a
// warp share the rows' elements (8 each) and combine them with the segmented
// shuffle scan, whatever the rows' lengths.
// ---------------------------------------------------------------------------
template <typename T, int VEC>
__device__ __forceinline__ uint32_t load_product_group(const T *__restrict__ vals, const uint32_t *__restrict__ cols,
                                                       const T *__restrict__ x, uint32_t g, uint32_t c1,
                                                       T (&p)[kEpt], uint64_t pol) {
  if (g >= c1) return 0u;
  const uint32_t cnt = min(kEpt, c1 - g);
  if (VEC == 2 && cnt == kEpt) {  // g a multiple of 8: 32-byte aligned
    T v[8];
    uint32_t k[8];
    ld_stream8(vals + g, v, pol);
    ld_stream8(cols + g, k, pol);
    T xv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) xv[j] = ld_x(x + k[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j) p[j] = mul_rn(v[j], xv[j]);
  } else if (VEC == 1 && cnt == kEpt) {  // 16-byte aligned: two loads per array
    T v0[4], v1[4];
    uint32_t k0[4], k1[4];
    ld_stream4(vals + g, v0, pol);
    ld_stream4(vals + g + 4, v1, pol);
    ld_stream4(cols + g, k0, pol);
    ld_stream4(cols + g + 4, k1, pol);
    T x0[4], x1[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x0[k] = ld_x(x + k0[k]);
      x1[k] = ld_x(x + k1[k]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      p[k] = mul_rn(v0[k], x0[k]);
      p[4 + k] = mul_rn(v1[k], x1[k]);
    }
  } else {
#pragma unroll
    for (uint32_t k = 0; k < kEpt; ++k)
      if (k < cnt) p[k] = mul_rn(ld_stream1(vals + g + k, pol), ld_x(x + ld_stream1(cols + g + k, pol)));
  }
  return cnt;
}

constexpr uint32_t kTileCnt = kWarpTile + 4;  // per-warp start counts: positions 0..256, padded to 16 bytes

template <typename T, int VEC, bool WIDE = false>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? MFP_COO_MINBLOCKS : MFP_COO_MINBLOCKS64)
    csr_tile_kernel(uint32_t n_rows, uint32_t nnz, const T *__restrict__ vals, const uint32_t *__restrict__ cols,
                    const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ tile_prev,
                    const T *__restrict__ x, T *__restrict__ y, coo_carry<T> cw, coo_ws_header *hdr) {
  __shared__ __align__(16) uint32_t s_cnt[kBlock / 32][kTileCnt];
  const uint64_t pol = policy_evict_first();
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t wt = blockIdx.x * (kBlock / 32) + warp;
  if ((uint64_t)wt * kWarpTile >= nnz) return;  // whole warps only
  const uint32_t c0 = wt * kWarpTile, c1 = min(nnz, c0 + kWarpTile);
  T pr[kEpt];
  const uint32_t g = c0 + lane * kEpt;
  const uint32_t cnt = load_product_group<T, VEC>(vals, cols, x, g, c1, pr, pol);
  uint32_t *sc = s_cnt[warp];
  for (uint32_t i = lane; i < kTileCnt; i += 32u) sc[i] = 0u;
  const uint32_t prv = __ldg(tile_prev + wt);  // row of element c0 - 1; kNoRow for the first tile
  // row starts at positions [c0, lim]: lim = c1 locates the row after the
  // tile, which the last tile does not need
  const uint32_t lim = c1 < nnz ? c1 : c1 - 1u;
  __syncwarp();
  // 32 row starts per round trip, or 64 (WIDE) when a tile holds more than
  // 32 rows on average
  for (uint32_t j0 = prv + 1u;; j0 += WIDE ? 64u : 32u) {  // prv + 1 wraps to 0 for the first tile
    const uint32_t ja = j0 + lane;
    const uint32_t ba = ja < n_rows ? __ldg(row_ptr + ja) : 0xffffffffu;  // start of row ja (>= c0)
    if (WIDE) {
      const uint32_t jb = ja + 32u;
      const uint32_t bb = jb < n_rows ? __ldg(row_ptr + jb) : 0xffffffffu;
      if (ba <= lim) atomicAdd(&sc[ba - c0], 1u);
      if (bb <= lim) atomicAdd(&sc[bb - c0], 1u);
      if (__any_sync(0xffffffffu, bb > lim)) break;  // rows are sorted by start: bb >= ba
    } else {
      if (ba <= lim) atomicAdd(&sc[ba - c0], 1u);
      if (__any_sync(0xffffffffu, ba > lim)) break;
    }
  }
  __syncwarp();
  // row of each element: prv + the row starts at or before it
  uint32_t q[kEpt];
  {
    const uint4 a = *reinterpret_cast<const uint4 *>(sc + lane * kEpt);
    const uint4 b = *reinterpret_cast<const uint4 *>(sc + lane * kEpt + 4);
    q[0] = a.x; q[1] = a.y; q[2] = a.z; q[3] = a.w;
    q[4] = b.x; q[5] = b.y; q[6] = b.z; q[7] = b.w;
  }
  uint32_t tot = 0;
#pragma unroll
  for (uint32_t k = 0; k < kEpt; ++k) tot += q[k];
  uint32_t inc = tot;  // inclusive scan of the lanes' counts
#pragma unroll
  for (uint32_t o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  const uint32_t all = __shfl_sync(0xffffffffu, inc, 31);
  uint32_t rw[kEpt];
  uint32_t run = prv + (inc - tot);
#pragma unroll
  for (uint32_t k = 0; k < kEpt; ++k) {
    run += q[k];
    rw[k] = run;
  }
  const uint32_t nxt = c1 < nnz ? prv + all + sc[kWarpTile] : kNoRow;  // row of element c1
  warp_tile_reduce<T, false>(wt, c0, c1, nnz, n_rows, pr, rw, cnt, prv, nxt, y, cw, hdr);
}

// Pass 2: the row starting in tile w that continues past it.  The tiles that
// follow are read 16 at a time (their loads in flight together) and walked in
// order in registers: a row of 50,000 elements spans 195 tiles, and one
// dependent load per tile would make it the launch's critical path.
// Without ACCUM the whole grid then zeroes the rows before the first row and
// after the last row that hold elements (grid-stride; the grid may be larger
// than one thread per tile for that).
#ifndef MFP_FIXUP_BATCH
#define MFP_FIXUP_BATCH 16
#endif
template <typename T, bool ACCUM>
__global__ void __launch_bounds__(kBlock) coo_fixup_kernel(uint32_t n_tiles, uint32_t n_rows, coo_carry<T> cw,
                                                           const coo_ws_header *hdr, T *__restrict__ y) {
  constexpr uint32_t B = MFP_FIXUP_BATCH;
  griddep_wait();  // the warp pass's partial sums and rows of y
  const uint32_t w = blockIdx.x * kBlock + threadIdx.x;
  if (!ACCUM) {
    const uint32_t first = min(hdr->first_row, n_rows);
    const uint32_t last = hdr->last_row;
    const uint32_t step = gridDim.x * kBlock;
    for (uint32_t r = w; r < first; r += step) y[r] = T(0);
    if (last < n_rows)
      for (uint32_t r = last + 1u + w; r < n_rows; r += step) y[r] = T(0);
  }
  const uint32_t f = w < n_tiles ? cw.flags[w] : 0u;
  // this thread's tile starts a row that goes on into the next tile
  const bool chain = (f & kTailCont) && !((f & kOneRow) && (f & kHeadCont));
  T acc = T(0);
  uint32_t row = 0, next = 0;  // next: the first tile not examined yet
  bool more = false;           // the row goes on beyond the first batch
  if (chain) {
    acc = cw.tail[w];
    row = cw.tail_row[w];
    // the row ends in the first following tile that does not hold only this
    // row and continue; the last tile never continues, so that tile exists
    uint32_t g[B];
    T t[B];
#pragma unroll
    for (uint32_t j = 0; j < B; ++j) {
      const uint32_t k = w + 1u + j;
      g[j] = k < n_tiles ? cw.flags[k] : 0u;
      t[j] = k < n_tiles ? cw.tail[k] : T(0);
    }
    uint32_t end = B;
#pragma unroll
    for (uint32_t j = 0; j < B; ++j) {
      if (end == B) {
        if ((g[j] & kOneRow) && (g[j] & kTailCont)) acc = add_rn(acc, t[j]);
        else end = j;
      }
    }
    if (end < B) acc = add_rn(acc, cw.head[w + 1u + end]);
    else more = true, next = w + 1u + B;
  }
  // Rows longer than the first batch (a few per matrix, up to hundreds of
  // tiles): the whole warp walks them, 256 tiles per round (lane l holds
  // tiles base + 8 l .. base + 8 l + 7, so lane order is tile order); the
  // round's tails are summed by a fixed shuffle tree.
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t todo = __ballot_sync(0xffffffffu, more); todo; todo &= todo - 1u) {
    const uint32_t src = __ffs(todo) - 1u;
    uint32_t base = __shfl_sync(0xffffffffu, next, src);
    T racc = T(0);  // the sum of the rounds so far (same value in every lane)
    uint32_t end_tile = 0;
    for (;;) {
      uint32_t g[8];
      T t[8];
#pragma unroll
      for (uint32_t j = 0; j < 8; ++j) {
        const uint32_t k = base + 8u * lane + j;
        g[j] = k < n_tiles ? cw.flags[k] : 0u;
        t[j] = k < n_tiles ? cw.tail[k] : T(0);
      }
      uint32_t first_np = 8;  // first tile of this lane that ends the row
#pragma unroll
      for (uint32_t j = 0; j < 8; ++j)
        if (first_np == 8 && !((g[j] & kOneRow) && (g[j] & kTailCont))) first_np = j;
      const uint32_t np = __ballot_sync(0xffffffffu, first_np < 8);
      const uint32_t end_lane = np ? __ffs(np) - 1u : 32u;
      T part = T(0);
      const uint32_t upto = lane < end_lane ? 8u : (lane == end_lane ? first_np : 0u);
#pragma unroll
      for (uint32_t j = 0; j < 8; ++j)
        if (j < upto) part = add_rn(part, t[j]);
      part = group_reduce_down(part, 32);
      racc = add_rn(racc, __shfl_sync(0xffffffffu, part, 0));
      if (np) {
        end_tile = base + 8u * end_lane + __shfl_sync(0xffffffffu, first_np, end_lane);
        break;
      }
      base += 256u;
    }
    if (lane == src) acc = add_rn(add_rn(acc, racc), cw.head[end_tile]);
  }
  if (chain) coo_put<T, ACCUM>(y, n_rows, row, acc);
}

// ---------------------------------------------------------------------------
// SCOO: one CTA per slice; row accumulators and (optionally) the slice's x
// window live in dynamic shared memory.
// ---------------------------------------------------------------------------
// SCOO in warp tiles: a slice of up to kScooTiles tiles (131,072 elements)
// keeps its tiles' carries in shared memory.
constexpr uint32_t kScooTiles = 512;
template <typename T>
struct scoo_smem_static {
  union {
    seg_scan_smem<T> scan;
    struct {
      T head[kScooTiles], tail[kScooTiles];
      uint32_t flags[kScooTiles], tail_row[kScooTiles];
    } t;
  };
};

// R16: rel holds each element's row as a 16-bit offset from its slice's
// first row (compact SCOO rows; ridx stays for the whole-CTA chunk path).
template <typename T, int VEC, bool XWIN, bool R16 = false>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? MFP_SCOO_MINBLOCKS : MFP_COO_MINBLOCKS64) scoo_kernel(uint32_t n_rows, uint32_t slice_size,
                                                      const T *__restrict__ vals,
                                                      const uint32_t *__restrict__ cidx,
                                                      const uint32_t *__restrict__ ridx,
                                                      const uint32_t *__restrict__ slices_ptr,
                                                      const uint32_t *__restrict__ windows,
                                                      uint32_t max_window,
                                                      const uint32_t *__restrict__ order,
                                                      const T *__restrict__ x, T *__restrict__ y,
                                                      const uint16_t *__restrict__ rel = nullptr) {
  __shared__ scoo_smem_static<T> sm;
  extern __shared__ __align__(16) unsigned char dyn[];
  T *acc = reinterpret_cast<T *>(dyn);                       // slice_size (rounded to 4)
  T *s_x = acc + ((slice_size + 3u) & ~3u);                  // max_window + 4 when XWIN
  const uint64_t pol = policy_evict_first();
  // the hardware starts blocks in index order: with `order` (slices by element
  // count, descending) the heaviest slices start first and the tail is short
  const uint32_t s = order ? order[blockIdx.x] : blockIdx.x;
  const uint32_t row0 = s * slice_size;
  if (row0 >= n_rows) return;
  const uint32_t nrows = min(slice_size, n_rows - row0);
  const uint32_t eb = slices_ptr[s], ee = slices_ptr[s + 1];
  for (uint32_t i = threadIdx.x; i < nrows; i += kBlock) acc[i] = T(0);
  bool use_win = false;
  uint32_t wlo = 0;
  if (XWIN && eb < ee) {
    wlo = windows[2 * s];
    const uint32_t whi = windows[2 * s + 1];
    if (whi > wlo && whi - wlo <= max_window) {
      use_win = true;
      for (uint32_t i = threadIdx.x; i < whi - wlo; i += kBlock) s_x[i] = ld_x(x + wlo + i);
    }
  }
  __syncthreads();
  {
    // Warp tiles: warp w reduces the slice's 256-element tiles w, w + 8, ...
    // with the COO warp-tile reduction, rows that start and end in a tile
    // going straight into the accumulator; after one barrier, each row that
    // crosses tiles is summed in tile order from the tiles' carries.  No
    // barrier per chunk; the same bits on every run.
    const uint32_t base8 = eb & ~7u;
    const uint32_t n_tiles = eb < ee ? (ee - base8 + kWarpTile - 1u) / kWarpTile : 0u;
    if (n_tiles <= kScooTiles) {
      const uint32_t lane = threadIdx.x & 31u;
      coo_carry<T> cw;
      cw.head = sm.t.head;
      cw.tail = sm.t.tail;
      cw.flags = sm.t.flags;
      cw.tail_row = sm.t.tail_row;
      // rows go in slice-local (r - row0, unsigned): a row id outside the
      // slice (invalid input) fails the bound checks and is dropped
      for (uint32_t t = threadIdx.x >> 5; t < n_tiles; t += kBlock / 32u) {
        const uint32_t g0 = base8 + t * kWarpTile;
        const uint32_t c0 = max(eb, g0), c1 = min(ee, g0 + kWarpTile);
        T pr[kEpt];
        uint32_t rw[kEpt], i0 = 0;
        const uint32_t g = g0 + lane * kEpt;
        uint32_t cnt, prv, nxt;
        if (R16) {  // the offsets are the slice-local rows
          cnt = (XWIN && use_win)
                    ? load_run_group16<T, VEC>(vals, cidx, rel, 0u, x_window<T>{s_x, wlo}, g, c0, c1, pr, rw, i0, pol)
                    : load_run_group16<T, VEC>(vals, cidx, rel, 0u, x_global<T>{x}, g, c0, c1, pr, rw, i0, pol);
          prv = c0 > eb ? ld_stream_u16(rel + c0 - 1u, pol) : kNoRow;
          nxt = c1 < ee ? ld_stream_u16(rel + c1, pol) : kNoRow;
        } else {
          cnt = (XWIN && use_win)
                    ? load_run_group<T, VEC>(vals, cidx, ridx, x_window<T>{s_x, wlo}, g, c0, c1, pr, rw, i0, pol)
                    : load_run_group<T, VEC>(vals, cidx, ridx, x_global<T>{x}, g, c0, c1, pr, rw, i0, pol);
#pragma unroll
          for (int k = 0; k < kEpt; ++k) rw[k] -= row0;
          prv = c0 > eb ? __ldg(ridx + c0 - 1u) - row0 : kNoRow;
          nxt = c1 < ee ? __ldg(ridx + c1) - row0 : kNoRow;
        }
        warp_tile_reduce<T, true>(t, g0, c1, ee, nrows, pr, rw, cnt, prv, nxt, acc, cw, nullptr);
      }
      __syncthreads();
      // a row that starts in tile t and goes on: its tail, then the following
      // tiles' heads in order, up to the tile where it ends
      for (uint32_t t = threadIdx.x; t < n_tiles; t += kBlock) {
        const uint32_t f = sm.t.flags[t];
        if (!(f & kTailCont) || ((f & kOneRow) && (f & kHeadCont))) continue;
        T sum = sm.t.tail[t];
        for (uint32_t u = t + 1u; u < n_tiles; ++u) {
          const uint32_t fu = sm.t.flags[u];
          sum = add_rn(sum, sm.t.head[u]);
          if (!((fu & kOneRow) && (fu & kTailCont))) break;
        }
        const uint32_t lr = sm.t.tail_row[t];
        if (lr < nrows) acc[lr] = sum;
      }
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < nrows; i += kBlock) y[row0 + i] = acc[i];
      return;
    }
  }
  // a slice of more than kScooTiles tiles: whole-CTA chunks of 2048 elements
  auto emit = [&](uint32_t row, T total, bool, bool) {
    const uint32_t lr = row - row0;
    if (lr < nrows) acc[lr] = add_rn(acc[lr], total);
  };
  auto gap = [](uint32_t, uint32_t) {};
  for (uint32_t c0 = eb; c0 < ee;) {
    const uint32_t base8 = c0 & ~7u;
    const uint32_t c1 = min(ee, base8 + (uint32_t)kChunk);
    T pr[kEpt];
    uint32_t rw[kEpt], i0 = 0;
    const uint32_t g = base8 + threadIdx.x * kEpt;
    const uint32_t cnt = (XWIN && use_win)
                             ? load_run_group<T, VEC>(vals, cidx, ridx, x_window<T>{s_x, wlo}, g, c0, c1, pr, rw, i0, pol)
                             : load_run_group<T, VEC>(vals, cidx, ridx, x_global<T>{x}, g, c0, c1, pr, rw, i0, pol);
    // the chunk's emits into acc[] finish before the next chunk's scan
    // barriers, which every thread passes only after its own emits
    block_segmented_reduce_regs<T>(pr, rw, cnt, i0, c0, c1, rows_u32{ridx}, emit, gap, sm.scan);
    c0 = c1;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nrows; i += kBlock) y[row0 + i] = acc[i];
}


// SCOO with the slices' elements in column order (the reference's sort_cols
// layout, scoo_matrix_class.cpp:102-138): rows are not contiguous within a
// slice, so each product is added into its row's shared-memory accumulator
// with an atomic, as the reference's scoo_spmv_kernel does (gpu/scoo_spmv.cu:
// 46-129).  Column order makes the x reads of a slice ascend.  The order of the
// additions into a row is not fixed.
template <typename T, bool XWIN>
__global__ void __launch_bounds__(kBlock) scoo_unsorted_kernel(uint32_t n_rows, uint32_t slice_size,
                                                               const T *__restrict__ vals,
                                                               const uint32_t *__restrict__ cidx,
                                                               const uint32_t *__restrict__ ridx,
                                                               const uint32_t *__restrict__ slices_ptr,
                                                               const uint32_t *__restrict__ windows,
                                                               uint32_t max_window,
                                                               const uint32_t *__restrict__ order,
                                                               const T *__restrict__ x, T *__restrict__ y) {
  extern __shared__ __align__(16) unsigned char dyn[];
  T *acc = reinterpret_cast<T *>(dyn);
  T *s_x = acc + ((slice_size + 3u) & ~3u);
  const uint64_t pol = policy_evict_first();
  const uint32_t s = order ? order[blockIdx.x] : blockIdx.x;
  const uint32_t row0 = s * slice_size;
  if (row0 >= n_rows) return;
  const uint32_t nrows = min(slice_size, n_rows - row0);
  const uint32_t eb = slices_ptr[s], ee = slices_ptr[s + 1];
  for (uint32_t i = threadIdx.x; i < nrows; i += kBlock) acc[i] = T(0);
  bool use_win = false;
  uint32_t wlo = 0;
  if (XWIN && eb < ee) {
    wlo = windows[2 * s];
    const uint32_t whi = windows[2 * s + 1];
    if (whi > wlo && whi - wlo <= max_window) {
      use_win = true;
      for (uint32_t i = threadIdx.x; i < whi - wlo; i += kBlock) s_x[i] = ld_x(x + wlo + i);
    }
  }
  __syncthreads();
  // 4 elements per thread in flight, coalesced across the CTA
  for (uint32_t e0 = eb + threadIdx.x; e0 < ee; e0 += 4u * kBlock) {
    T v[4];
    uint32_t c[4], r[4];
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
      const uint32_t e = e0 + k * kBlock;
      if (e < ee) {
        v[k] = ld_stream1(vals + e, pol);
        c[k] = ld_stream1(cidx + e, pol);
        r[k] = ld_stream1(ridx + e, pol);
      }
    }
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
      const uint32_t e = e0 + k * kBlock;
      if (e < ee) {
        const T xv = (XWIN && use_win) ? s_x[c[k] - wlo] : ld_x(x + c[k]);
        const uint32_t lr = r[k] - row0;
        if (lr < nrows) atomicAdd(&acc[lr], mul_rn(v[k], xv));
      }
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nrows; i += kBlock) y[row0 + i] = acc[i];
}

template <typename T>
__global__ void fill_kernel(uint64_t n, T *v, T value) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = value;
}

}  // namespace dev
}  // namespace mfp
