// Streaming CSR SpMV for sm_100a: persistent CTAs, TMA bulk prefetch,
// gathers overlapped with reductions.
//
// The element arrays (values, column ids) are cut into fixed chunks of CH
// elements; CTA c owns the contiguous chunk range [c*K, c*K + K).  For each
// chunk a single thread issues TMA bulk copies (cp.async.bulk) of the
// chunk's values and column ids into a ring of S shared-memory stages, S-1
// chunks ahead.  Every thread then gathers x for its 4 elements of chunk k
// and, while those L2 gathers are in flight, reduces chunk k-1 from the
// product buffer.  The rows of a chunk are given by the host plan
// (chunk_row[k] = first row starting at or after the chunk) and the row_ptr
// segment, which is prefetched the same way.
//
// Row -> thread mapping per algorithm (the reference algorithm it mirrors):
//   scalar   L = 1: one thread adds a row's products one by one in CSR order
//            (csr_spmv_kernel, gpu_matrix_multiplier.cu:22-43); exact with the
//            reference CPU loop for rows up to the assist threshold, also
//            across chunk boundaries;
//   vector   L lanes per row, lane-strided + shuffle tree
//            (csr_spmv_vector_kernel, gpu_matrix_multiplier.cu:331-362);
//   adaptive L = 256 / rows-in-chunk (power of two, <= 32): the chunk is the
//            nnz-balanced row block of CSR-Stream (csr_adaptive_spmv.cu:42-116).
// Rows whose segment in a chunk exceeds the assist threshold are reduced by a
// whole warp.  A row continuing past a chunk carries its partial sum to the
// next chunk of the same CTA (FP64 for rows longer than 4096 elements); a row
// split between two CTAs meets in an ordered partial-sum slot, summed by the
// last contributor.
#pragma once

#include "spmv_kernels.cuh"

namespace mfp {
namespace dev {

constexpr uint32_t kNoPiece = 0xffffffffu;
constexpr uint32_t kMbarLimit = 1u << 26;
constexpr uint32_t kCrowCap = 256;  // chunk_row entries of a CTA cached in shared memory

struct stream_edge {
  uint32_t head;  // contribution index for a row entering the CTA's range, or kNoPiece
  uint32_t tail;  // contribution index for a row leaving it, or kNoPiece
};

template <typename T>
struct stream_args {
  uint32_t n_rows, nnz, nchunks, chunks_per_cta;
  const uint32_t *__restrict__ row_ptr;
  const uint32_t *__restrict__ cols;
  const T *__restrict__ vals;
  const T *__restrict__ x;
  T *__restrict__ y;
  const uint32_t *__restrict__ chunk_row;  // nchunks + 1
  const stream_edge *__restrict__ edges;   // one per CTA
  const long_piece *__restrict__ contrib;  // boundary contributions (row, slot_base, piece, npieces, counter)
  double *partials;
  uint32_t *counters;
  uint32_t *error;
  uint32_t assist_thr;
  uint32_t lanes;     // vector mode
  uint32_t fp64_thr;  // rows longer than this carry their sum in FP64
};

template <typename T>
struct carry_state {
  double d;       // FP64 running sum (long rows)
  T t;            // running sum in T (exact chaining for short rows)
  uint32_t row;
  uint32_t active, foreign, fp64;
};

// Per-stage row_ptr window: entries [rp_lo, rp_lo + RPC) of row_ptr, rp_lo a
// multiple of 4 (16-byte TMA alignment).
template <int CH>
struct stream_rpc {
  static constexpr int value = CH / 4 + 16;
};

template <typename T, int CH, int S>
struct stream_smem {
  __align__(128) T vals[S][CH];
  __align__(128) uint32_t cols[S][CH];
  __align__(128) uint32_t rp[S][stream_rpc<CH>::value];
  __align__(16) T prod[CH + 64];
  uint32_t rp_lo[S];   // first row_ptr index held by the stage's window
  uint32_t rp_n[S];    // entries of the window loaded by TMA (0: read row_ptr from global)
  uint64_t full[S];
  uint32_t assists[kBlock];
  uint32_t nassist;
  carry_state<T> cs[2];
  double red_a[kBlock / 32], red_b[kBlock / 32];
  // followed in dynamic shared memory by chunk_row[k0 .. k1] of the CTA
};

template <typename T>
__device__ __forceinline__ void contribute(const stream_args<T> &A, uint32_t piece, double value) {
  if (piece == kNoPiece) return;
  const long_piece pc = A.contrib[piece];
  A.partials[pc.slot_base + pc.piece] = value;
  __threadfence();
  const uint32_t arrived = atomicAdd(A.counters + pc.counter, 1u);
  if (arrived == pc.npieces - 1) {
    __threadfence();
    comp_sum s;
    for (uint32_t k = 0; k < pc.npieces; ++k) s.add(__ldcg(A.partials + pc.slot_base + k));
    A.y[pc.row] = (T)s.value();
    A.counters[pc.counter] = 0u;
  }
}

template <typename T>
__device__ __forceinline__ double carry_value(const carry_state<T> &c) {
  return c.fp64 ? c.d : (double)c.t;
}

// Reduce chunk k (products in sm.prod, row_ptr segment in sm.rp[b] or global).
// MODE 0 scalar, 1 vector, 2 adaptive.
template <typename T, int MODE, int CH, int S>
__device__ __forceinline__ void stream_reduce(const stream_args<T> &A, stream_smem<T, CH, S> &sm, uint32_t k,
                                              uint32_t r0, uint32_t r1, uint32_t st, uint32_t cin, uint32_t cout,
                                              bool first_chunk, uint32_t head_piece) {
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t c0 = k * (uint32_t)CH;
  const uint32_t c1 = min(A.nnz, c0 + (uint32_t)CH);
  const uint32_t nr = r1 - r0;
  const uint32_t lo = sm.rp_lo[st], nwin = sm.rp_n[st];
  const uint32_t *win = sm.rp[st];
  // RP(j) = row_ptr[r0 + j] for j in [-1, nr]: from the stage window when held there
  auto RP = [&](int j) -> uint32_t {
    const uint32_t i = r0 + j - lo;
    return i < nwin ? win[i] : A.row_ptr[r0 + j];
  };
  const uint32_t rp0 = RP(0);
  const bool has_in = (rp0 > c0) && (r0 > 0);
  if (t == 0) sm.nassist = 0;
  __syncthreads();

  // ---- carry-in row r0 - 1: elements [c0, min(rp0, c1)) -------------------
  if (warp == 0) {
    carry_state<T> cur = sm.cs[cin];
    if (has_in) {
      if (first_chunk) {
        cur.row = r0 - 1;
        cur.active = 1;
        cur.foreign = 1;
        cur.fp64 = (rp0 - RP(-1)) > A.fp64_thr;
        cur.d = 0.0;
        cur.t = T(0);
      }
      const uint32_t e = min(rp0, c1) - c0;
      if (MODE == 0 && !cur.fp64 && e <= A.assist_thr) {
        if (lane == 0) cur.t = seq_sum(cur.t, sm.prod, 0u, e);
      } else {
        T part = strided_sum(sm.prod, 0u, e, lane, 32u);
        part = group_reduce_down(part, 32);
        if (cur.fp64)
          cur.d = __dadd_rn(cur.d, (double)part);
        else
          cur.t = add_rn(cur.t, part);
      }
      if (lane == 0) {
        if (rp0 <= c1 && nr > 0) {  // the row ends in this chunk
          const double v = carry_value(cur);
          if (cur.foreign)
            contribute(A, head_piece, v);
          else
            A.y[cur.row] = cur.fp64 ? (T)v : cur.t;
          cur.active = 0;
        } else if (rp0 <= c1 && nr == 0 && rp0 == c1) {
          const double v = carry_value(cur);
          if (cur.foreign)
            contribute(A, head_piece, v);
          else
            A.y[cur.row] = cur.fp64 ? (T)v : cur.t;
          cur.active = 0;
        }
        if (nr == 0) sm.cs[cout] = cur;  // the whole chunk belonged to this row
      }
    } else if (lane == 0 && nr == 0) {
      sm.cs[cout] = cur;
    }
  }

  // ---- rows starting in this chunk ------------------------------------------
  uint32_t L;
  if (MODE == 0)
    L = 1;
  else if (MODE == 1)
    L = A.lanes;
  else {
    const uint32_t q = nr ? (uint32_t)kBlock / nr : 32u;
    L = q >= 32 ? 32u : (q == 0 ? 1u : (1u << (31 - __clz(q))));
  }
  const uint32_t G = kBlock / L, g = t / L, gl = t % L;
  const uint32_t rounds = (nr + G - 1) / G;
  for (uint32_t it = 0; it < rounds; ++it) {
    const uint32_t j = g + it * G;
    const bool valid = j < nr;
    uint32_t s = 0, e = 0, rs = 0, re = 0;
    if (valid) {
      rs = RP(j);
      re = RP(j + 1);
      s = rs - c0;
      e = min(re, c1) - c0;
    }
    const bool longseg = valid && (e - s > A.assist_thr);
    bool overflow = false;  // assist list full: the group reduces the row itself
    if (longseg && gl == 0) {
      const uint32_t q = atomicAdd(&sm.nassist, 1u);
      if (q < (uint32_t)kBlock)
        sm.assists[q] = j;
      else
        overflow = true;
    }
    if (L > 1) overflow = __shfl_sync(0xffffffffu, overflow ? 1u : 0u, lane & ~(L - 1u)) != 0u;
    const bool mine = valid && (!longseg || overflow);
    T part = T(0);
    if (mine && s < e) part = L == 1 ? seq_sum(T(0), sm.prod, s, e) : strided_sum(sm.prod, s, e, gl, L);
    if (L > 1) part = group_reduce_down(part, (int)L);
    if (mine && gl == 0) {
      if (re <= c1) {
        A.y[r0 + j] = part;
      } else {  // continues into the next chunk: becomes the carry
        carry_state<T> c;
        c.row = r0 + j;
        c.active = 1;
        c.foreign = 0;
        c.fp64 = (re - rs) > A.fp64_thr;
        c.t = c.fp64 ? T(0) : part;
        c.d = c.fp64 ? (double)part : 0.0;
        sm.cs[cout] = c;
      }
    }
  }
  __syncthreads();
  // ---- long segments: one warp each ----------------------------------------
  const uint32_t na = min(sm.nassist, (uint32_t)kBlock);
  for (uint32_t q = warp; q < na; q += kBlock / 32) {
    const uint32_t j = sm.assists[q];
    const uint32_t rs = RP(j), re = RP(j + 1);
    const uint32_t s = rs - c0, e = min(re, c1) - c0;
    T part = strided_sum(sm.prod, s, e, lane, 32u);
    part = group_reduce_down(part, 32);
    if (lane == 0) {
      if (re <= c1) {
        A.y[r0 + j] = part;
      } else {
        carry_state<T> c;
        c.row = r0 + j;
        c.active = 1;
        c.foreign = 0;
        c.fp64 = (re - rs) > A.fp64_thr;
        c.t = c.fp64 ? T(0) : part;
        c.d = c.fp64 ? (double)part : 0.0;
        sm.cs[cout] = c;
      }
    }
  }
  // rows that end in this chunk leave no carry
  if (t == 0 && nr > 0) {
    const uint32_t last_end = RP(nr);
    if (last_end <= c1) sm.cs[cout].active = 0;
  }
}

template <typename T, int MODE, int CH, int S>
__global__ void __launch_bounds__(kBlock) csr_stream_kernel(const stream_args<T> A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  auto &sm = *reinterpret_cast<stream_smem<T, CH, S> *>(smem_raw);
  uint32_t *crow = reinterpret_cast<uint32_t *>(smem_raw + sizeof(stream_smem<T, CH, S>));
  constexpr uint32_t RPC = stream_rpc<CH>::value;
  constexpr uint32_t EPT = CH / kBlock;  // elements per thread per chunk (multiple of 4)
  const uint32_t t = threadIdx.x;
  const uint32_t k0 = blockIdx.x * A.chunks_per_cta;
  const uint32_t k1 = min(A.nchunks, k0 + A.chunks_per_cta);
  if (k0 >= k1) return;
  const uint32_t m = k1 - k0;
  const uint64_t pol = policy_evict_first();
  const stream_edge edge = A.edges[blockIdx.x];

  for (uint32_t i = t; i <= m && i < kCrowCap; i += kBlock) crow[i] = A.chunk_row[k0 + i];
  auto CR = [&](uint32_t i) -> uint32_t { return i < kCrowCap ? crow[i] : A.chunk_row[k0 + i]; };
  if (t == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&sm.full[s], 1);
    fence_mbar_init();
    carry_state<T> z;
    z.active = z.foreign = z.fp64 = 0;
    z.t = T(0);
    z.d = 0.0;
    z.row = 0;
    sm.cs[0] = z;
    sm.cs[1] = z;
  }
  __syncthreads();
  // Thread 0 loads chunk k0 + j into stage j % S: values, column ids and the
  // row_ptr window of its rows, all with TMA bulk copies.
  auto issue = [&](uint32_t j) {
    const uint32_t k = k0 + j, s = j % S;
    const uint32_t c0 = k * (uint32_t)CH;
    const uint32_t n = min((uint32_t)CH, A.nnz - c0);
    const uint32_t n4 = n & ~3u;
    const uint32_t r0 = CR(j), r1 = CR(j + 1);
    const uint32_t want_lo = r0 ? r0 - 1 : 0;
    const uint32_t lo = want_lo & ~3u;
    const uint32_t hi = min((r1 + 1 + 3) & ~3u, (A.n_rows + 1) & ~3u);  // TMA'd entries end (exclusive)
    uint32_t nw = hi > lo ? hi - lo : 0;
    if (nw > RPC) nw = 0;  // many rows (empty rows): read row_ptr from global
    sm.rp_lo[s] = lo;
    sm.rp_n[s] = nw;
    mbar_arrive_expect_tx(&sm.full[s], n4 * (uint32_t)(sizeof(T) + 4) + nw * 4u);
    if (n4) {
      tma_load_1d(sm.vals[s], A.vals + c0, n4 * (uint32_t)sizeof(T), &sm.full[s], pol);
      tma_load_1d(sm.cols[s], A.cols + c0, n4 * 4u, &sm.full[s], pol);
    }
    if (nw) tma_load_1d(sm.rp[s], A.row_ptr + lo, nw * 4u, &sm.full[s], pol);
  };
  if (t == 0)
    for (uint32_t j = 0; j < (uint32_t)S && j < m; ++j) issue(j);

  for (uint32_t j = 0; j <= m; ++j) {
    T p[EPT];
    if (j < m) {
      const uint32_t k = k0 + j, s = j % S;
      const uint32_t c0 = k * (uint32_t)CH;
      const uint32_t n = min((uint32_t)CH, A.nnz - c0);
      if (!mbar_wait(&sm.full[s], (j / S) & 1u, kMbarLimit)) atomicOr(A.error, 4u);
      const uint32_t n4 = n & ~3u;
#pragma unroll
      for (uint32_t g = 0; g < EPT / 4; ++g) {
        const uint32_t i0 = 4u * (t + g * kBlock);
        if (i0 < n4) {
          const uint4 cc = *reinterpret_cast<const uint4 *>(&sm.cols[s][i0]);
          p[4 * g + 0] = ld_x(A.x + cc.x);
          p[4 * g + 1] = ld_x(A.x + cc.y);
          p[4 * g + 2] = ld_x(A.x + cc.z);
          p[4 * g + 3] = ld_x(A.x + cc.w);
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint32_t i = i0 + q;
            p[4 * g + q] = (i < n) ? ld_x(A.x + ld_stream1(A.cols + c0 + i, pol)) : T(0);
          }
        }
      }
    }
    if (j > 0) {
      const uint32_t jp = j - 1;
      stream_reduce<T, MODE, CH, S>(A, sm, k0 + jp, CR(jp), CR(jp + 1), jp % S, jp & 1u, j & 1u, jp == 0,
                                    edge.head);
    }
    if (j < m) {
      // multiply by the staged values (the x gathers complete here)
      const uint32_t k = k0 + j, s = j % S;
      const uint32_t c0 = k * (uint32_t)CH;
      const uint32_t n = min((uint32_t)CH, A.nnz - c0);
      const uint32_t n4 = n & ~3u;
#pragma unroll
      for (uint32_t g = 0; g < EPT / 4; ++g) {
        const uint32_t i0 = 4u * (t + g * kBlock);
        T v[4];
        if (i0 < n4) {
          if (sizeof(T) == 4) {
            const float4 vv = *reinterpret_cast<const float4 *>(&sm.vals[s][i0]);
            v[0] = vv.x; v[1] = vv.y; v[2] = vv.z; v[3] = vv.w;
          } else {
            const double2 a = *reinterpret_cast<const double2 *>(&sm.vals[s][i0]);
            const double2 bb = *reinterpret_cast<const double2 *>(&sm.vals[s][i0 + 2]);
            v[0] = a.x; v[1] = a.y; v[2] = bb.x; v[3] = bb.y;
          }
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) v[q] = (i0 + q < n) ? ld_stream1(A.vals + c0 + i0 + q, pol) : T(0);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) p[4 * g + q] = mul_rn(v[q], p[4 * g + q]);
      }
    }
    __syncthreads();  // chunk j-1 reduced (its stage and the product buffer are free)
    if (j < m) {
      if (t == 0 && j >= 1 && j - 1 + S < m) issue(j - 1 + S);  // refill the stage of chunk j-1
#pragma unroll
      for (uint32_t g = 0; g < EPT / 4; ++g) {
        T q4[4] = {p[4 * g], p[4 * g + 1], p[4 * g + 2], p[4 * g + 3]};
        store_group4<T>(sm.prod, 4u * (t + g * kBlock), q4);
      }
    }
    __syncthreads();
  }
  // a row still open at the end of the range continues in the next CTA
  if (t == 0) {
    const carry_state<T> c = sm.cs[m & 1u];
    if (c.active) contribute(A, edge.tail, carry_value(c));
  }
}

}  // namespace dev
}  // namespace mfp
