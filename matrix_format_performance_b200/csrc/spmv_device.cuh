// Device helpers shared by every SpMV format kernel (sm_100a).
//
// SpMV moves ~6-12 bytes per multiply-add, so every kernel here is bound by
// HBM bandwidth and by the L2 gathers of x.  The helpers encode the three
// rules all kernels follow:
//  1. matrix arrays (values, column ids, row ids) are read exactly once:
//     16-byte vector loads, L1 no-allocate, L2 evict-first, so they do not
//     push x out of L1/L2;
//  2. x is gathered through the read-only path (L1-cached, normal L2 priority);
//  3. products are formed with an explicitly rounded multiply and summed with
//     an explicitly rounded add (no FMA contraction), so a row summed in CSR
//     order gives exactly the result of the reference CPU loop
//     (cpu/cpu_matrix_multiplier.cpp:34-43), not merely a close one.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mfp {
namespace dev {

constexpr int kWarp = 32;

__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// ---- streaming loads -------------------------------------------------------
__device__ __forceinline__ void ld_stream4(const float *p, float (&v)[4], uint64_t pol) {
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
               : "l"(p), "l"(pol));
}
// Four doubles are one 32-byte sector when p is 32-byte aligned: one 256-bit
// load then (two 16-byte loads of one sector would ask L2 for it twice),
// else two 16-byte loads.  Callers' alignment is uniform over a warp.
__device__ __forceinline__ void ld_stream4(const double *p, double (&v)[4], uint64_t pol) {
  if ((reinterpret_cast<uintptr_t>(p) & 31u) == 0) {
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f64 {%0,%1,%2,%3}, [%4], %5;"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
                 : "l"(p), "l"(pol));
    return;
  }
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
               : "=d"(v[0]), "=d"(v[1])
               : "l"(p), "l"(pol));
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
               : "=d"(v[2]), "=d"(v[3])
               : "l"(p + 2), "l"(pol));
}
__device__ __forceinline__ void ld_stream4(const uint32_t *p, uint32_t (&v)[4], uint64_t pol) {
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "l"(p), "l"(pol));
}
// 32-byte streaming loads (sm_100 256-bit vectors; p 32-byte aligned): a lane
// that reads a whole sector asks L2 for it once.  Two 16-byte loads of the
// same sector miss in L1 twice and send two requests.
__device__ __forceinline__ void ld_stream8(const float *p, float (&v)[8], uint64_t pol) {
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
               : "l"(p), "l"(pol));
}
__device__ __forceinline__ void ld_stream8(const double *p, double (&v)[8], uint64_t pol) {
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f64 {%0,%1,%2,%3}, [%4], %5;"
               : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
               : "l"(p), "l"(pol));
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f64 {%0,%1,%2,%3}, [%4], %5;"
               : "=d"(v[4]), "=d"(v[5]), "=d"(v[6]), "=d"(v[7])
               : "l"(p + 4), "l"(pol));
}
__device__ __forceinline__ void ld_stream8(const uint32_t *p, uint32_t (&v)[8], uint64_t pol) {
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "l"(p), "l"(pol));
}
// 16-bit words: 8 (16 bytes, p 16-byte aligned, packed two per register) or one.
__device__ __forceinline__ void ld_stream8_u16(const uint16_t *p, uint32_t (&w)[4], uint64_t pol) {
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3])
               : "l"(p), "l"(pol));
}
__device__ __forceinline__ uint32_t ld_stream_u16(const uint16_t *p, uint64_t pol) {
  unsigned short v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
  return v;
}
// 8 bytes (p 8-byte aligned) and one byte, streamed like the above.
__device__ __forceinline__ void ld_stream8_u8(const uint8_t *p, uint32_t (&w)[2], uint64_t pol) {
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;"
               : "=r"(w[0]), "=r"(w[1])
               : "l"(p), "l"(pol));
}
__device__ __forceinline__ uint32_t ld_stream_u8(const uint8_t *p, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u8 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}

// 32-byte store (p 32-byte aligned).
__device__ __forceinline__ void st_global8(float *p, const float (&v)[8]) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]),
               "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}

// 8 consecutive 4-byte words (p 16-byte aligned): one 32-byte load when p is
// 32-byte aligned, else two 16-byte loads.
template <typename W>
__device__ __forceinline__ void ld_stream8_any(const W *p, W (&v)[8], uint64_t pol) {
  static_assert(sizeof(W) == 4, "4-byte words");
  if ((reinterpret_cast<uintptr_t>(p) & 31u) == 0) {
    ld_stream8(p, v, pol);
    return;
  }
  W a[4], b[4];
  ld_stream4(p, a, pol);
  ld_stream4(p + 4, b, pol);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = a[k];
    v[4 + k] = b[k];
  }
}
__device__ __forceinline__ float ld_stream1(const float *p, uint64_t pol) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(v)
               : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_stream1(const double *p, uint64_t pol) {
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
               : "=d"(v)
               : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_stream1(const uint32_t *p, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
               : "=r"(v)
               : "l"(p), "l"(pol));
  return v;
}

// x gathers: read-only path, cached in L1.
template <typename T>
__device__ __forceinline__ T ld_x(const T *p) {
  return __ldg(p);
}

// ---- arithmetic without contraction ---------------------------------------
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// Neumaier-compensated double accumulator (used for rows longer than 4096
// elements and for combining long-row partial sums).
struct comp_sum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v) {
    const double t = __dadd_rn(s, v);
    if (fabs(s) >= fabs(v))
      c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, t), v));
    else
      c = __dadd_rn(c, __dadd_rn(__dsub_rn(v, t), s));
    s = t;
  }
  __device__ __forceinline__ void add(const comp_sum &o) {
    add(o.s);
    c = __dadd_rn(c, o.c);
  }
  __device__ __forceinline__ double value() const { return __dadd_rn(s, c); }
};

// ---- reductions ------------------------------------------------------------
// Tree over lane offsets width/2 .. 1 with shuffle-down, the same tree as the
// reference warp_reduce (gpu/reduce.cuh:6-20) when width == 32; the result is
// in the first lane of each group.
template <typename T>
__device__ __forceinline__ T group_reduce_down(T v, int width) {
  for (int off = width >> 1; off > 0; off >>= 1) v = add_rn(v, __shfl_down_sync(0xffffffffu, v, off, width));
  return v;
}

template <typename T, int BLOCK>
__device__ __forceinline__ T block_reduce(T v, T *s_scratch /* >= BLOCK/32 */) {
  v = group_reduce_down(v, kWarp);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_scratch[warp] = v;
  __syncthreads();
  T r = T(0);
  if (warp == 0) {
    r = lane < BLOCK / 32 ? s_scratch[lane] : T(0);
    r = group_reduce_down(r, kWarp);
  }
  return r;  // valid in thread 0
}

template <int BLOCK>
__device__ __forceinline__ comp_sum block_reduce_comp(comp_sum v, double *s_s, double *s_c) {
  for (int off = 16; off > 0; off >>= 1) {
    comp_sum o;
    o.s = __shfl_down_sync(0xffffffffu, v.s, off);
    o.c = __shfl_down_sync(0xffffffffu, v.c, off);
    v.add(o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
    s_s[warp] = v.s;
    s_c[warp] = v.c;
  }
  __syncthreads();
  comp_sum r;
  if (warp == 0) {
    if (lane < BLOCK / 32) {
      r.s = s_s[lane];
      r.c = s_c[lane];
    }
    for (int off = 16; off > 0; off >>= 1) {
      comp_sum o;
      o.s = __shfl_down_sync(0xffffffffu, r.s, off);
      o.c = __shfl_down_sync(0xffffffffu, r.c, off);
      r.add(o);
    }
  }
  return r;  // valid in thread 0
}

// Exclusive block scan of small unsigned counts (one per thread).
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *s_warp /* BLOCK/32+1 */,
                                                         uint32_t *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, inc, off);
    if (lane >= off) inc += o;
  }
  __syncthreads();
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < BLOCK / 32 ? s_warp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, wi, off);
      if (lane >= off) wi += o;
    }
    if (lane < BLOCK / 32) s_warp[lane] = wi - w;
    if (lane == BLOCK / 32 - 1) s_warp[BLOCK / 32] = wi;
  }
  __syncthreads();
  *total = s_warp[BLOCK / 32];
  return s_warp[warp] + inc - v;
}

// Programmatic dependent launch: waits until the preceding kernel of the
// stream has completed and its writes are visible (a no-op when the launch did
// not allow early start).  Hardware-managed; not a poll on memory.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace dev
}  // namespace mfp

// ---- TMA bulk copies and mbarriers (sm_90+ PTX, used on sm_100a) -----------
namespace mfp {
namespace dev {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One arrival that also announces `bytes` of asynchronous transfer.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Plain arrival (no transaction bytes); release semantics at CTA scope.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// Bounded wait: false if the phase did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// Global -> shared bulk copy (TMA, 1D).  dst, src 16-byte aligned; bytes a
// multiple of 16.  Completion is counted on `bar` in bytes.
__device__ __forceinline__ void tma_load_1d(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                            uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

}  // namespace dev
}  // namespace mfp
