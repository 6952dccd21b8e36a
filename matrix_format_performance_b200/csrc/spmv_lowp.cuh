// Reduced-precision CSR: 16-bit values (BF16 or FP16) with one FP32 scale
// per row, FP32 accumulation, and optionally 16-bit column deltas.
//
// Layout (engine extension; the reference has only float and double CSR):
//   row_ptr[rows+1]  uint32 (as CSR)
//   values[nnz]      uint16 bit patterns of q_ij = round(a_ij / scale_i)
//   scale[rows]      float, scale_i = max_j |a_ij| (1 for an empty/zero row)
//   either cols[nnz] uint32 column ids
//   or     delta[nnz] uint16 with col = base[e / 2048] + delta[e], base one
//          uint32 per 2048-element chunk (built only when every chunk's
//          column span fits 16 bits: stencil and banded matrices)
// y_i = scale_i * sum_j float(q_ij) * x_j, the sum in FP32.
//
// Two kernels:
//   lowp_kernel      row blocks of 256 rows, elements staged through shared
//                    memory as FP32 products in chunks of up to 4096 (plain
//                    16-byte loads), thread t adds row t's products in CSR
//                    order.  Any alignment.
//   lowp_tma_kernel  persistent, warp-specialised: a producer warp copies each
//                    row block's values, indices and row_ptr window into
//                    shared-memory stages with TMA bulk copies; consumer
//                    threads read their row straight from the stage.  Needs
//                    16-byte-aligned arrays.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>
#include <type_traits>

#include "spmv_kernels.cuh"

namespace mfp {
namespace dev {

constexpr uint32_t kLowpChunkShift = 11;  // 2048 elements per delta base

template <int VT>  // 2 = bf16, 3 = fp16
__device__ __forceinline__ float lowp_to_float(uint32_t bits) {
  if (VT == 2) return __uint_as_float(bits << 16);
  return __half2float(__ushort_as_half((unsigned short)bits));
}

// The two 16-bit values of a 32-bit word as floats (low half first).
template <int VT>
__device__ __forceinline__ float2 lowp_pair(uint32_t w) {
  if (VT == 2) return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
  __half2 h;
  memcpy(&h, &w, sizeof(w));
  return __half22float2(h);
}


template <int VT, bool D16>
struct lowp_args {
  uint32_t n_rows;
  const uint32_t *__restrict__ row_ptr;
  const uint16_t *__restrict__ vals;
  const float *__restrict__ scale;
  const uint32_t *__restrict__ cols;      // !D16
  const uint16_t *__restrict__ delta;     // D16
  const uint32_t *__restrict__ base;      // D16
  const float *__restrict__ x;
  float *__restrict__ y;
};

template <int VT, bool D16>
__device__ __forceinline__ uint32_t lowp_col(const lowp_args<VT, D16> &A, uint32_t e, uint64_t pol) {
  if (D16) return A.base[e >> kLowpChunkShift] + ld_stream_u16(A.delta + e, pol);
  return ld_stream1(A.cols + e, pol);
}

// ---------------------------------------------------------------------------
// Row-block kernel
// ---------------------------------------------------------------------------
constexpr uint32_t kLowpChunk = 4096;  // elements staged per phase (16 per thread)

// One 8-element group: 16-byte loads of values and column deltas (or two of
// column ids) for elements [e0, e0 + 8).
template <int VT, bool D16>
struct lowp_group {
  uint32_t v[4];
  uint32_t c[8];
  __device__ __forceinline__ void load(const lowp_args<VT, D16> &A, uint32_t e0, uint64_t pol) {
    ld_stream8_u16(A.vals + e0, v, pol);
    if (D16) {
      uint32_t d[4];
      ld_stream8_u16(A.delta + e0, d, pol);
      const uint32_t cb = A.base[e0 >> kLowpChunkShift];  // 8 | 2048: a group never straddles two bases
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        c[2 * k] = cb + (d[k] & 0xffffu);
        c[2 * k + 1] = cb + (d[k] >> 16);
      }
    } else {
      ld_stream8_any(A.cols + e0, c, pol);
    }
  }
  __device__ __forceinline__ void products(const lowp_args<VT, D16> &A, float *dst, uint32_t i) const {
    float xv[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) xv[k] = ld_x(A.x + c[k]);
    float p0[4], p1[4];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      p0[2 * k] = mul_rn(lowp_to_float<VT>(v[k] & 0xffffu), xv[2 * k]);
      p0[2 * k + 1] = mul_rn(lowp_to_float<VT>(v[k] >> 16), xv[2 * k + 1]);
      p1[2 * k] = mul_rn(lowp_to_float<VT>(v[2 + k] & 0xffffu), xv[4 + 2 * k]);
      p1[2 * k + 1] = mul_rn(lowp_to_float<VT>(v[2 + k] >> 16), xv[4 + 2 * k + 1]);
    }
    store_group4<float>(dst, i, p0);
    store_group4<float>(dst, i + 4, p1);
  }
};

// Products of elements [a, b) (b - (a & ~7) <= kLowpChunk) into dst at
// swizzled local index e - (a & ~7).  Two groups per thread per round, both
// groups' loads issued before their x gathers.
template <int VT, bool D16, bool VEC>
__device__ __forceinline__ void stage_lowp(const lowp_args<VT, D16> &A, uint32_t a, uint32_t b, float *dst,
                                           uint64_t pol) {
  const uint32_t base8 = a & ~7u;
  if (VEC) {
    const uint32_t a8 = (a + 7u) & ~7u, b8 = b & ~7u;
    if (a8 < b8) {
      for (uint32_t e = a + threadIdx.x; e < a8; e += kBlock)
        dst[swz(e - base8)] = mul_rn(lowp_to_float<VT>(ld_stream_u16(A.vals + e, pol)), ld_x(A.x + lowp_col(A, e, pol)));
      for (uint32_t e = b8 + threadIdx.x; e < b; e += kBlock)
        dst[swz(e - base8)] = mul_rn(lowp_to_float<VT>(ld_stream_u16(A.vals + e, pol)), ld_x(A.x + lowp_col(A, e, pol)));
      const uint32_t ng = (b8 - a8) >> 3;
      uint32_t g = threadIdx.x;
      for (; g + kBlock < ng; g += 2 * kBlock) {
        lowp_group<VT, D16> g0, g1;
        g0.load(A, a8 + 8u * g, pol);
        g1.load(A, a8 + 8u * (g + kBlock), pol);
        g0.products(A, dst, a8 + 8u * g - base8);
        g1.products(A, dst, a8 + 8u * (g + kBlock) - base8);
      }
      if (g < ng) {
        lowp_group<VT, D16> g0;
        g0.load(A, a8 + 8u * g, pol);
        g0.products(A, dst, a8 + 8u * g - base8);
      }
      return;
    }
  }
  for (uint32_t e = a + threadIdx.x; e < b; e += kBlock)
    dst[swz(e - base8)] = mul_rn(lowp_to_float<VT>(ld_stream_u16(A.vals + e, pol)), ld_x(A.x + lowp_col(A, e, pol)));
}

// Rows with more elements than this are summed by a warp (lane-strided, then a
// shuffle tree) instead of by their own thread, so a row of 50,000 elements
// costs its CTA ~1,600 steps per lane, not 50,000 in one thread.
constexpr uint32_t kLowpAssist = 128;

template <int VT, bool D16, bool VEC>
__global__ void __launch_bounds__(kBlock, 6) lowp_kernel(const lowp_args<VT, D16> A) {
  __shared__ uint32_t s_rp[kBlock + 1];
  __shared__ uint32_t s_assist[kBlock];
  __shared__ uint32_t s_wc[kBlock / 32 + 1];
  __shared__ float s_acc[kBlock];
  __shared__ __align__(16) float prod[kLowpChunk + 64];
  const uint64_t pol = policy_evict_first();
  const uint32_t r0 = blockIdx.x * kBlock;
  const uint32_t nr = min((uint32_t)kBlock, A.n_rows - r0);
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  for (uint32_t i = t; i <= nr; i += kBlock) s_rp[i] = A.row_ptr[r0 + i];
  s_acc[t] = 0.f;
  __syncthreads();
  const bool has = t < nr;
  const uint32_t rs = has ? s_rp[t] : 0u, re = has ? s_rp[t + 1] : 0u;
  const bool assist = has && re - rs > kLowpAssist;
  uint32_t nassist = 0;
  if (__syncthreads_or(assist)) {
    // ordered list of the block's long rows
    const uint32_t ballot = __ballot_sync(0xffffffffu, assist);
    if (lane == 0) s_wc[warp] = __popc(ballot);
    __syncthreads();
    if (t == 0) {
      uint32_t sum = 0;
      for (uint32_t w = 0; w < kBlock / 32; ++w) {
        const uint32_t c = s_wc[w];
        s_wc[w] = sum;
        sum += c;
      }
      s_wc[kBlock / 32] = sum;
    }
    __syncthreads();
    if (assist) s_assist[s_wc[warp] + __popc(ballot & ((1u << lane) - 1u))] = t;
    __syncthreads();
    nassist = s_wc[kBlock / 32];
  }
  const uint32_t a = s_rp[0], b = s_rp[nr];
  float acc = 0.f;
  for (uint32_t c0 = a; c0 < b;) {
    const uint32_t base8 = c0 & ~7u;
    const uint32_t c1 = min(b, base8 + kLowpChunk);
    stage_lowp<VT, D16, VEC>(A, c0, c1, prod, pol);
    __syncthreads();
    if (has && !assist) {
      const uint32_t lo = max(rs, c0), hi = min(re, c1);
      if (lo < hi) acc = seq_sum<float, true>(acc, prod, lo - base8, hi - base8);
    }
    for (uint32_t q = warp; q < nassist; q += kBlock / 32) {
      const uint32_t j = s_assist[q];
      const uint32_t js = s_rp[j], je = s_rp[j + 1];
      const uint32_t lo = max(js, c0), hi = min(je, c1);
      if (lo < hi) {
        // lane l takes the row's elements js + l + 32 k, whichever chunk they fall in
        float part = strided_sum(prod, lo - base8, hi - base8, (lane - (lo - js)) & 31u, 32u);
        part = group_reduce_down(part, 32);
        if (lane == 0) s_acc[j] = add_rn(s_acc[j], part);
      }
    }
    __syncthreads();
    c0 = c1;
  }
  if (has) A.y[r0 + t] = (assist ? s_acc[t] : acc) * A.scale[r0 + t];
}

// ---------------------------------------------------------------------------
// Pipelined kernel (16-byte-aligned arrays): warp-specialised persistent CTAs.
// A producer warp walks the CTA's row blocks (256 rows each, blocks
// blockIdx.x, blockIdx.x + gridDim.x, ...), cuts each block's element range
// into sub-chunks of at most CAP elements, and copies every sub-chunk's values,
// column deltas (or ids) and, for the first sub-chunk, the block's row_ptr
// window into one of S shared-memory stages with TMA bulk copies.  The 256
// consumer threads (thread t owns row t of the block) read their row straight
// from the stage — no product staging, no CTA-wide barrier — and release the
// stage with one mbarrier arrival per warp, so the copies of the next stages
// overlap the gathers and sums of this one.
//
// Bank conflicts: rows of equal length n put the threads' row starts n
// elements apart; when n is a multiple of 8 (16-bit indices) or 4 (uint32
// ids) that maps a warp's reads onto a few banks.  Such rows are read as
// 32-bit words (two elements per read) starting at word (t mod words) and
// wrapping around, which spreads the warp over all banks.  Other rows are read
// element by element in CSR order (neighbouring rows then gather neighbouring
// x entries together).  A row's order of additions is fixed by its length and
// position, so results are reproducible; they can differ from lowp_kernel's
// in the last bits.
// ---------------------------------------------------------------------------
constexpr uint32_t kLowpRows = 256;                       // rows per block = consumer threads
constexpr uint32_t kLowpThreads = kLowpRows + 32;         // + the producer warp
constexpr uint32_t kLowpEnd = 0xffffffffu;                // terminator task
constexpr uint32_t kLowpWaitLimit = 1u << 26;

struct lowp_task {
  uint32_t blk;   // row block, kLowpEnd = no more work
  uint32_t c0;    // sub-chunk element range [c0, c1), c0 a multiple of 8
  uint32_t c1;
  uint32_t tend;  // [c0, tend) is in the stage; [tend, c1) (< 8 elements) is read from global memory
  uint32_t rp_n;  // row_ptr entries r0 .. r0 + rp_n - 1 in the stage (first sub-chunk only)
  uint32_t first, last, pad;
};

template <bool D16, uint32_t CAP>
struct lowp_stage {
  using idx_t = typename std::conditional<D16, uint16_t, uint32_t>::type;
  __align__(16) uint16_t vals[CAP];
  __align__(16) idx_t idx[CAP];
  __align__(16) uint32_t rp[kLowpRows + 4];
  lowp_task task;
};

template <bool D16, uint32_t CAP, uint32_t S>
struct lowp_pipe {
  lowp_stage<D16, CAP> st[S];
  uint64_t full[S];
  uint64_t empty[S];
};

template <bool D16, uint32_t CAP, uint32_t S>
constexpr size_t lowp_pipe_bytes() {
  return sizeof(lowp_pipe<D16, CAP, S>);
}

__device__ uint32_t g_lowp_error;  // bit 0: a pipeline wait gave up

// Column of element e from a 16-bit delta: base[e >> 11] + delta.  `bi` and
// (cb0, cb1) cache base[bi], base[bi + 1] for the thread's current row.
struct delta_bases {
  const uint32_t *base;
  uint32_t nbase, bi, cb0, cb1;
  __device__ __forceinline__ void at(uint32_t e) {
    bi = e >> kLowpChunkShift;
    cb0 = base[bi];
    cb1 = bi + 1 < nbase ? base[bi + 1] : 0u;
  }
  __device__ __forceinline__ uint32_t col(uint32_t e, uint32_t d) const {
    return ((e >> kLowpChunkShift) == bi ? cb0 : cb1) + d;
  }
  // true when [e, e + n) needs no other base than base[bi], base[bi + 1]
  __device__ __forceinline__ bool covers(uint32_t e, uint32_t n) const {
    return ((e + n - 1u) >> kLowpChunkShift) <= bi + 1u && (e >> kLowpChunkShift) >= bi;
  }
};

// acc += the products of stage elements [lo, hi) in CSR order, 8 at a time
// (all reads and gathers of a group issued before its adds).
template <int VT, bool D16, typename I>
__device__ __forceinline__ float stage_elem_sum(const lowp_args<VT, D16> &A, const uint16_t *sv, const I *si,
                                                uint32_t c0, uint32_t lo, uint32_t hi, delta_bases &db,
                                                float acc) {
  uint32_t e = lo;
  if (D16 && lo < hi && !db.covers(lo, hi - lo)) db.at(lo);
  for (; e + 8u <= hi; e += 8u) {
    if (D16 && !db.covers(e, 8u)) db.at(e);
    uint32_t q[8], c[8];
    float xv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      q[j] = sv[e + j - c0];
      c[j] = D16 ? db.col(e + j, si[e + j - c0]) : (uint32_t)si[e + j - c0];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) xv[j] = ld_x(A.x + c[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j) acc = add_rn(acc, mul_rn(lowp_to_float<VT>(q[j]), xv[j]));
  }
  for (; e < hi; ++e) {
    if (D16 && !db.covers(e, 1u)) db.at(e);
    const uint32_t c = D16 ? db.col(e, si[e - c0]) : (uint32_t)si[e - c0];
    acc = add_rn(acc, mul_rn(lowp_to_float<VT>(sv[e - c0]), ld_x(A.x + c)));
  }
  return acc;
}

// acc += the products of the nw whole 32-bit words of the stage from word wlo
// (stage positions [2 wlo, 2 wlo + 2 nw)): one shared-memory read yields two
// values (and two deltas, or one 8-byte read two column ids).  Words are
// visited rot, rot + 1, ..., nw - 1, 0, ..., rot - 1 in batches of 8: all
// reads and x gathers of a batch are issued before its first FMA; a partial
// last batch re-reads word wlo for its missing words and drops their products.
// BM: 0 uint32 column ids; 1 one delta base (cb) for all the words; 2 the two
// bases cached in `db`; 3 any base (base[] read per element).
constexpr int kLowpWords = 8;
template <int VT, bool D16, int BM, typename I>
__device__ __forceinline__ float stage_words_sum(const lowp_args<VT, D16> &A, const uint16_t *sv, const I *si,
                                                 uint32_t c0, uint32_t wlo, uint32_t nw, uint32_t rot,
                                                 const delta_bases &db, uint32_t cb, float acc) {
  const uint32_t *svw = reinterpret_cast<const uint32_t *>(sv);
  for (uint32_t j = 0; j < nw; j += kLowpWords) {
    float q[2 * kLowpWords], xv[2 * kLowpWords];
#pragma unroll
    for (int k = 0; k < kLowpWords; ++k) {
      const bool v = j + k < nw;
      uint32_t r = (v ? j + k : 0u) + rot;
      r = r >= nw ? r - nw : r;
      const uint32_t w = wlo + r;
      const float2 f = lowp_pair<VT>(svw[w]);
      uint32_t ca, cb2;
      if (D16) {
        const uint32_t dw = reinterpret_cast<const uint32_t *>(si)[w];
        const uint32_t da = dw & 0xffffu, dd = dw >> 16;
        if (BM == 1) {
          ca = cb + da;
          cb2 = cb + dd;
        } else {
          const uint32_t e = c0 + 2u * w;
          ca = BM == 2 ? db.col(e, da) : A.base[e >> kLowpChunkShift] + da;
          cb2 = BM == 2 ? db.col(e + 1u, dd) : A.base[(e + 1u) >> kLowpChunkShift] + dd;
        }
      } else {
        const uint2 cw = reinterpret_cast<const uint2 *>(si)[w];
        ca = cw.x;
        cb2 = cw.y;
      }
      q[2 * k] = v ? f.x : 0.f;
      q[2 * k + 1] = v ? f.y : 0.f;
      xv[2 * k] = ld_x(A.x + ca);
      xv[2 * k + 1] = ld_x(A.x + cb2);
    }
#pragma unroll
    for (int k = 0; k < 2 * kLowpWords; ++k) acc = __fmaf_rn(q[k], xv[k], acc);
  }
  return acc;
}

// A row's stage elements [lo, hi) read as words, rotated by `rot` words: an
// odd first and an odd last element one by one, the words between them by
// stage_words_sum (c0 is even, so element parity = stage position parity).
template <int VT, bool D16, typename I>
__device__ __forceinline__ float stage_rotated_sum(const lowp_args<VT, D16> &A, const uint16_t *sv, const I *si,
                                                   uint32_t c0, uint32_t lo, uint32_t hi, uint32_t rot,
                                                   delta_bases &db, float acc) {
  if (D16 && (lo >> kLowpChunkShift) != db.bi) db.at(lo);
  // the cached bases cover the row unless it is longer than 2048
  const bool two = !D16 || ((hi - 1u) >> kLowpChunkShift) <= db.bi + 1u;
  auto one = [&](uint32_t e) {
    const uint32_t d = (uint32_t)si[e - c0];
    const uint32_t c = !D16 ? d : two ? db.col(e, d) : A.base[e >> kLowpChunkShift] + d;
    acc = __fmaf_rn(lowp_to_float<VT>(sv[e - c0]), ld_x(A.x + c), acc);
  };
  uint32_t a = lo, b = hi;
  if (a & 1u) one(a++);
  if (a < b && (b & 1u)) one(--b);
  if (a >= b) return acc;
  const uint32_t wlo = (a - c0) >> 1, nw = (b - a) >> 1;
  const uint32_t r = rot % nw;
  if (!D16) return stage_words_sum<VT, D16, 0>(A, sv, si, c0, wlo, nw, r, db, 0u, acc);
  const uint32_t b0 = a >> kLowpChunkShift, b1 = (b - 1u) >> kLowpChunkShift;
  if (b0 == b1 && b0 <= db.bi + 1u)
    return stage_words_sum<VT, D16, 1>(A, sv, si, c0, wlo, nw, r, db, b0 == db.bi ? db.cb0 : db.cb1, acc);
  if (two) return stage_words_sum<VT, D16, 2>(A, sv, si, c0, wlo, nw, r, db, 0u, acc);
  return stage_words_sum<VT, D16, 3>(A, sv, si, c0, wlo, nw, r, db, 0u, acc);
}

template <int VT, bool D16, uint32_t CAP, uint32_t S>
__global__ void __launch_bounds__(kLowpThreads, 3) lowp_tma_kernel(const lowp_args<VT, D16> A, uint32_t nnz) {
  extern __shared__ __align__(128) unsigned char lowp_smem_raw[];
  auto &P = *reinterpret_cast<lowp_pipe<D16, CAP, S> *>(lowp_smem_raw);
  const uint32_t t = threadIdx.x;
  const uint32_t n_blocks = (A.n_rows + kLowpRows - 1u) / kLowpRows;
  if (t == 0) {
    for (uint32_t s = 0; s < S; ++s) {
      mbar_init(&P.full[s], 1u);
      mbar_init(&P.empty[s], kLowpRows / 32u);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (t >= kLowpRows) {
    // ---- producer warp (lane 0) ----
    if (t != kLowpRows) return;
    const uint64_t pol = policy_evict_first();
    uint32_t use = 0;
    bool ok = true;
    auto acquire = [&](uint32_t &s) -> bool {
      s = use % S;
      const uint32_t k = use / S;
      return k == 0 || mbar_wait(&P.empty[s], (k - 1u) & 1u, kLowpWaitLimit);
    };
    // the next block's element range is loaded one block ahead
    uint32_t na = 0, nb = 0;
    if (blockIdx.x < n_blocks) {
      na = A.row_ptr[blockIdx.x * kLowpRows];
      nb = A.row_ptr[min(A.n_rows, (blockIdx.x + 1u) * kLowpRows)];
    }
    for (uint32_t blk = blockIdx.x; ok && blk < n_blocks; blk += gridDim.x) {
      const uint32_t r0 = blk * kLowpRows;
      const uint32_t nr = min(kLowpRows, A.n_rows - r0);
      const uint32_t a = na, b = nb;
      const uint32_t nxt = blk + gridDim.x;
      if (nxt < n_blocks) {
        na = A.row_ptr[nxt * kLowpRows];
        nb = A.row_ptr[min(A.n_rows, (nxt + 1u) * kLowpRows)];
      }
      const uint32_t a8 = a & ~7u;
      uint32_t c0 = a8;
      do {
        const uint32_t c1 = min(b, c0 + CAP);
        const uint32_t tend = max(c0, c1 & ~7u);
        uint32_t s;
        if (!acquire(s)) {
          ok = false;
          break;
        }
        auto &st = P.st[s];
        const bool first = c0 == a8;
        const uint32_t rp_n = first ? ((nr + 1u) & ~3u) : 0u;
        st.task = lowp_task{blk, c0, c1, tend, rp_n, first ? 1u : 0u, c1 == b ? 1u : 0u, 0u};
        const uint32_t n = tend - c0;
        const uint32_t bv = n * 2u, bi = n * (D16 ? 2u : 4u), br = rp_n * 4u;
        mbar_arrive_expect_tx(&P.full[s], bv + bi + br);
        if (n) {
          tma_load_1d(st.vals, A.vals + c0, bv, &P.full[s], pol);
          if (D16)
            tma_load_1d(st.idx, A.delta + c0, bi, &P.full[s], pol);
          else
            tma_load_1d(st.idx, A.cols + c0, bi, &P.full[s], pol);
        }
        if (br) tma_load_1d(st.rp, A.row_ptr + r0, br, &P.full[s], pol);
        ++use;
        c0 = c1;
      } while (c0 < b);
    }
    uint32_t s;
    if (ok && acquire(s)) {
      P.st[s].task.blk = kLowpEnd;
      mbar_arrive(&P.full[s]);
    } else {
      atomicOr(&g_lowp_error, 1u);
    }
    return;
  }

  // ---- consumers: thread t owns row r0 + t of every task ----
  const uint32_t lane = t & 31u;
  const uint64_t pol = policy_evict_first();
  uint32_t use = 0, rs = 0, re = 0;
  float acc = 0.f, sc = 0.f;
  delta_bases db{A.base, (nnz + (1u << kLowpChunkShift) - 1u) >> kLowpChunkShift, 0xffffffffu, 0u, 0u};
  for (;;) {
    const uint32_t s = use % S, k = use / S;
    // every lane polls; the warp leaves together if any lane gave up
    if (!__all_sync(0xffffffffu, mbar_wait(&P.full[s], k & 1u, kLowpWaitLimit))) {
      if (lane == 0) atomicOr(&g_lowp_error, 1u);
      break;
    }
    const auto &st = P.st[s];
    const lowp_task tk = st.task;
    if (tk.blk == kLowpEnd) break;
    const uint32_t r0 = tk.blk * kLowpRows;
    const bool has = t < min(kLowpRows, A.n_rows - r0);
    if (tk.first) {
      if (has) {
        rs = t < tk.rp_n ? st.rp[t] : A.row_ptr[r0 + t];
        re = t + 1u < tk.rp_n ? st.rp[t + 1] : A.row_ptr[r0 + t + 1];
        sc = A.scale[r0 + t];
      } else {
        rs = re = 0u;
      }
      acc = 0.f;
    }
    if (has) {
      const uint32_t lo = max(rs, tk.c0), hi = min(re, tk.c1);
      const uint32_t mid = max(lo, min(hi, tk.tend));
      if (lo < mid) {
        const uint32_t n = mid - lo;
        if ((n & (D16 ? 7u : 3u)) == 0u)
          acc = stage_rotated_sum<VT, D16>(A, st.vals, st.idx, tk.c0, lo, mid, t, db, acc);
        else
          acc = stage_elem_sum<VT, D16>(A, st.vals, st.idx, tk.c0, lo, mid, db, acc);
      }
      for (uint32_t e = max(lo, tk.tend); e < hi; ++e) {  // the sub-chunk's last < 8 elements
        const uint32_t c = lowp_col(A, e, pol);
        acc = add_rn(acc, mul_rn(lowp_to_float<VT>(ld_stream_u16(A.vals + e, pol)), ld_x(A.x + c)));
      }
      if (tk.last) A.y[r0 + t] = acc * sc;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&P.empty[s]);
    ++use;
  }
}

// ---------------------------------------------------------------------------
// Reduced-precision ELL: column-major slots [k * rows + row] (the reference's
// ELL order), 16-bit values q with one FP32 scale per row, and either uint32
// column ids or 16-bit column offsets from the row (col = row + off - 32768).
// Padding slots hold q = 0 and a column of their row.  A thread owns 8 rows:
// VEC (rows % 8 == 0, 16-byte-aligned arrays) 8 consecutive rows, one 16-byte
// load of 8 values and one of 8 offsets (or two of ids) per slot; otherwise 8
// rows interleaved across its warp (row = warp base + 32 j + lane), so each
// 2-byte load and each x gather is contiguous over the warp.  Slots in order
// 0..width-1, FMA accumulation; y = acc * scale.
// With 16-bit offsets, a lane whose 8 rows have the same offset in a slot
// (stencil rows away from the grid's faces) reads their 8 consecutive x
// entries with two or three 16-byte loads instead of 8 gathers: a warp's
// x reads then cover 8 cache lines per instruction instead of 32 sectors,
// which lifts the L1 limit of the gathers.  Other lanes gather.
// ---------------------------------------------------------------------------
template <int VT, bool D16>
struct lowp_ell_args {
  uint32_t n_rows, width, n_cols;
  const uint16_t *__restrict__ q;
  const float *__restrict__ scale;
  const uint32_t *__restrict__ cols;  // !D16
  const uint16_t *__restrict__ off;   // D16
  const float *__restrict__ x;
  float *__restrict__ y;
};

// CTAs per SM the 16-bit ELL kernel (16-bit offsets, 8 rows per thread) is
// register-limited to: 8 (32 registers) holds the 27-point 128^3 stencil's
// 1,024 CTAs in one wave on 148 SMs (6, at 40 registers, left a second wave
// of 136 CTAs).  The uint32-column variants keep 6 (40 registers, which they
// need without spilling).
#ifndef MFP_LOWP_ELL_MINBLOCKS
#define MFP_LOWP_ELL_MINBLOCKS 8
#endif

// x[c .. c + 7] from the 16-byte-aligned words at c & ~3 (needs (c & ~3) + 12 <= n).
__device__ __forceinline__ void ld_x8_run(const float *__restrict__ x, uint32_t c, float (&xv)[8]) {
  const uint32_t a = c & ~3u, sh = c & 3u;
  const float4 v0 = __ldg(reinterpret_cast<const float4 *>(x + a));
  const float4 v1 = __ldg(reinterpret_cast<const float4 *>(x + a + 4));
  const float4 v2 = sh ? __ldg(reinterpret_cast<const float4 *>(x + a + 8)) : make_float4(0.f, 0.f, 0.f, 0.f);
  const float w[12] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w, v2.x, v2.y, v2.z, v2.w};
#pragma unroll
  for (int j = 0; j < 8; ++j) xv[j] = sh == 0 ? w[j] : sh == 1 ? w[j + 1] : sh == 2 ? w[j + 2] : w[j + 3];
}

// XRUN (16-bit offsets, 16-byte-aligned x, y and scale): a thread whose 8
// rows share one offset in a slot reads their 8 consecutive x entries as
// three 16-byte loads instead of 8 gathers, and the scales and y move 16
// bytes at a time.  One slot is in flight, to stay within 32 registers.
template <int VT, bool D16, bool VEC, bool XRUN = false>
__global__ void __launch_bounds__(kBlock, D16 && VEC ? MFP_LOWP_ELL_MINBLOCKS : 6)
    lowp_ell_kernel(const lowp_ell_args<VT, D16> A) {
  const uint64_t pol = policy_evict_first();
  const size_t stride = A.n_rows;
  if (VEC) {
    const uint32_t r = (blockIdx.x * kBlock + threadIdx.x) * 8u;
    if (r >= A.n_rows) return;
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = 0.f;
#pragma unroll(XRUN ? 1 : 2)
    for (uint32_t k = 0; k < A.width; ++k) {
      const size_t o = (size_t)k * stride + r;
      uint32_t qv[4], c[8];
      ld_stream8_u16(A.q + o, qv, pol);
      bool run = false;
      if (D16) {
        uint32_t dv[4];
        ld_stream8_u16(A.off + o, dv, pol);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          c[2 * j] = r + 2u * j + (dv[j] & 0xffffu) - 32768u;
          c[2 * j + 1] = r + 2u * j + 1u + (dv[j] >> 16) - 32768u;
        }
        if (XRUN) {
          // the 8 rows share one offset: their columns are c[0] .. c[0] + 7
          const uint32_t d2 = (dv[0] & 0xffffu) | (dv[0] << 16);
          run = dv[0] == d2 && dv[1] == d2 && dv[2] == d2 && dv[3] == d2 && A.n_cols >= 12u &&
                c[0] <= A.n_cols - 12u;  // (c[0] & ~3) + 12 <= n_cols, overflow-free
        }
      } else {
        ld_stream8_any(A.cols + o, c, pol);
      }
      float xv[8];
      if (run) {
        ld_x8_run(A.x, c[0], xv);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) xv[j] = ld_x(A.x + c[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float2 f = lowp_pair<VT>(qv[j]);
        acc[2 * j] = __fmaf_rn(f.x, xv[2 * j], acc[2 * j]);
        acc[2 * j + 1] = __fmaf_rn(f.y, xv[2 * j + 1], acc[2 * j + 1]);
      }
    }
    if (XRUN && ((reinterpret_cast<uintptr_t>(A.y) | reinterpret_cast<uintptr_t>(A.scale)) & 31u) == 0) {
      // 32-byte-aligned y and scale (r is a multiple of 8): one sector each
      float sc[8];
      ld_stream8(A.scale + r, sc, pol);
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] *= sc[j];
      st_global8(A.y + r, acc);
    } else if (XRUN) {  // 16-byte-aligned y and scale
      const float4 s0 = __ldg(reinterpret_cast<const float4 *>(A.scale + r));
      const float4 s1 = __ldg(reinterpret_cast<const float4 *>(A.scale + r + 4));
      *reinterpret_cast<float4 *>(A.y + r) = make_float4(acc[0] * s0.x, acc[1] * s0.y, acc[2] * s0.z, acc[3] * s0.w);
      *reinterpret_cast<float4 *>(A.y + r + 4) =
          make_float4(acc[4] * s1.x, acc[5] * s1.y, acc[6] * s1.z, acc[7] * s1.w);
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) A.y[r + j] = acc[j] * A.scale[r + j];
    }
  } else {
    // 8 rows per thread, interleaved across the warp: row = warp base + 32 j +
    // lane, so every load and every x gather of a warp is contiguous
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wbase = (blockIdx.x * kBlock + (threadIdx.x & ~31u)) * 8u;
    if (wbase >= A.n_rows) return;
    float acc[8];
    bool ok[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      acc[j] = 0.f;
      ok[j] = wbase + 32u * j + lane < A.n_rows;
    }
    for (uint32_t k = 0; k < A.width; ++k) {
      const size_t o = (size_t)k * stride + wbase + lane;
      uint32_t qv[8], c[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t r = wbase + 32u * j + lane;
        qv[j] = ok[j] ? ld_stream_u16(A.q + o + 32u * j, pol) : 0u;
        c[j] = ok[j] ? (D16 ? r + ld_stream_u16(A.off + o + 32u * j, pol) - 32768u : ld_stream1(A.cols + o + 32u * j, pol))
                     : 0u;
      }
      float xv[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) xv[j] = ok[j] ? ld_x(A.x + c[j]) : 0.f;
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] = __fmaf_rn(lowp_to_float<VT>(qv[j]), xv[j], acc[j]);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (ok[j]) A.y[wbase + 32u * j + lane] = acc[j] * A.scale[wbase + 32u * j + lane];
  }
}

}  // namespace dev
}  // namespace mfp
