// Load-ceiling probe for SpMV (a measurement kernel, not a format).
//
// It issues the memory operations of an SpMV over nnz (value, column) pairs
// and nothing else: no rows, no reduction by row, one partial sum per CTA.
//   mode 0  stream the values and column ids (a 32-byte load per array and
//           thread, on 32-byte-aligned arrays), no x gathers
//   mode 1  stream the column ids and gather x[col]
//   mode 2  stream both arrays and gather x[col] (the loads of any format
//           that reads each nonzero and its x entry once)
//   mode 3  as mode 1 with every gather folded into x[0, 4096) (16 KB, held
//           in L1): separates the L1 request rate from the L2 side
// Its time on a matrix is a floor for every format's kernel on that matrix:
// whatever a format does by row comes on top of these loads.  The x path is
// selectable to compare the L1-cached read-only gather with L2-only gathers.
//   mode 4  stream the column ids and gather x with TMA tile::gather4 (four
//           16-byte rows of x per instruction into shared memory, outside
//           the L1 request path); each lane then reads its entries there
//   mode 5  half of the gathers as in mode 4, the other half as in mode 1
//           (whether the two paths add up)
#pragma once

#include <cuda.h>

#include "spmv_device.cuh"

namespace mfp {
namespace dev {

constexpr int kProbeBlock = 256;
constexpr int kProbeEpt = 8;  // elements per thread per step: one 32-byte sector per array

template <int XPATH>
__device__ __forceinline__ float probe_x(const float *p) {
  float v;
  if (XPATH == 0) {
    v = __ldg(p);
  } else if (XPATH == 1) {
    asm volatile("ld.global.cg.f32 %0, [%1];" : "=f"(v) : "l"(p));
  } else {
    asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  }
  return v;
}

template <int MODE, int XPATH>
__global__ void __launch_bounds__(kProbeBlock) probe_loads_kernel(uint32_t nnz, const float *__restrict__ vals,
                                                                  const uint32_t *__restrict__ cols,
                                                                  const float *__restrict__ x, float *__restrict__ out) {
  __shared__ float s_red[kProbeBlock / 32];
  const uint64_t pol = policy_evict_first();
  const uint32_t groups = nnz / kProbeEpt;
  float acc = 0.f;
  uint32_t cacc = 0u;
  for (uint32_t g = blockIdx.x * kProbeBlock + threadIdx.x; g < groups; g += gridDim.x * kProbeBlock) {
    const uint32_t e = g * kProbeEpt;
    float v[8];
    uint32_t c[8];
    if (MODE == 0 || MODE == 2) ld_stream8_any(vals + e, v, pol);
    ld_stream8_any(cols + e, c, pol);
    if (MODE == 3) {
#pragma unroll
      for (int k = 0; k < 8; ++k) c[k] &= 4095u;
    }
    if (MODE == 0) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        acc += v[k];
        cacc ^= c[k];
      }
    } else {
      float xv[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) xv[k] = probe_x<XPATH>(x + c[k]);
#pragma unroll
      for (int k = 0; k < 8; ++k) acc += MODE == 2 ? v[k] * xv[k] : xv[k];
    }
  }
  // the last nnz % 8 elements
  if (blockIdx.x == 0 && threadIdx.x < nnz % kProbeEpt) {
    const uint32_t e = groups * kProbeEpt + threadIdx.x;
    const uint32_t c = MODE == 3 ? (cols[e] & 4095u) : cols[e];
    if (MODE == 0) {
      acc += vals[e];
      cacc ^= c;
    } else {
      acc += MODE == 2 ? vals[e] * probe_x<XPATH>(x + c) : probe_x<XPATH>(x + c);
    }
  }
  acc += (float)(cacc & 1u);
  const float s = block_reduce<float, kProbeBlock>(acc, s_red);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// ---- TMA gather4 probe ------------------------------------------------------
// x is seen as a 2-D tensor of rows of 4 floats (16 bytes); one tile::gather4
// copies four such rows (64 bytes) into a 128-byte-aligned shared-memory slot.
// Each lane owns two slots; one mbarrier per warp counts the bytes.  Waits are
// bounded: a warp that gives up stops, waits once more for its copies (also
// bounded) and flags its CTA's output with NaN.
constexpr int kG4Warps = 4;
constexpr uint32_t kG4Slot = 128;
constexpr uint32_t kG4WaitLimit = 1u << 24;
constexpr size_t kG4DynBytes = kG4Warps * 32 * 2 * kG4Slot + 128;  // + alignment slack

__device__ __forceinline__ void tma_gather4(uint32_t dst, const CUtensorMap *map, uint32_t r0, uint32_t r1,
                                            uint32_t r2, uint32_t r3, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3),
      "r"(smem_addr(bar))
      : "memory");
}

template <int MODE>  // 4: every gather by TMA; 5: half by TMA, half by ld.global.nc
__global__ void __launch_bounds__(kG4Warps * 32) probe_gather4_kernel(uint32_t nnz, const uint32_t *__restrict__ cols,
                                                                      const float *__restrict__ x,
                                                                      const __grid_constant__ CUtensorMap map,
                                                                      float *__restrict__ out) {
  extern __shared__ unsigned char g4_dyn[];
  __shared__ uint64_t bars[kG4Warps];
  __shared__ float s_red[kG4Warps];
  __shared__ uint32_t s_bad;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t base = (smem_addr(g4_dyn) + 127u) & ~127u;
  const unsigned char *gbase = g4_dyn + (base - smem_addr(g4_dyn));
  if (threadIdx.x == 0) s_bad = 0u;
  if (lane == 0) mbar_init(&bars[warp], 1);
  fence_mbar_init();
  __syncthreads();
  const uint32_t slot = base + (warp * 32u + lane) * 2u * kG4Slot;
  const float *sx = reinterpret_cast<const float *>(gbase + (warp * 32u + lane) * 2u * kG4Slot);
  const uint64_t pol = policy_evict_first();
  const uint32_t steps = nnz / 256u;  // a warp step covers 256 elements, 8 per lane
  const uint32_t bytes = 32u * (MODE == 4 ? 128u : 64u);
  uint32_t parity = 0;
  float acc = 0.f;
  bool ok = true;
  for (uint32_t st = blockIdx.x * kG4Warps + warp; st < steps; st += gridDim.x * kG4Warps) {
    const uint32_t e = st * 256u + lane * 8u;
    uint32_t c[8];
    ld_stream8_any(cols + e, c, pol);
    if (lane == 0) mbar_arrive_expect_tx(&bars[warp], bytes);
    __syncwarp();
    tma_gather4(slot, &map, c[0] >> 2, c[1] >> 2, c[2] >> 2, c[3] >> 2, &bars[warp]);
    float xl[4] = {0.f, 0.f, 0.f, 0.f};
    if (MODE == 4) {
      tma_gather4(slot + kG4Slot, &map, c[4] >> 2, c[5] >> 2, c[6] >> 2, c[7] >> 2, &bars[warp]);
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) xl[k] = __ldg(x + c[4 + k]);
    }
    ok = __all_sync(0xffffffffu, mbar_wait(&bars[warp], parity, kG4WaitLimit));
    if (!ok) break;
    parity ^= 1u;
#pragma unroll
    for (int k = 0; k < 4; ++k) acc += sx[4 * k + (c[k] & 3u)];
    if (MODE == 4) {
#pragma unroll
      for (int k = 0; k < 4; ++k) acc += sx[32 + 4 * k + (c[4 + k] & 3u)];
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) acc += xl[k];
    }
    __syncwarp();
  }
  if (!ok) {
    mbar_wait(&bars[warp], parity, kG4WaitLimit);  // the copies still in flight land before the CTA exits
    if (lane == 0) s_bad = 1u;
  }
  __syncthreads();
  const float s = block_reduce<float, kG4Warps * 32>(acc, s_red);
  if (threadIdx.x == 0) out[blockIdx.x] = s_bad ? __int_as_float(0x7fc00000) : s;
}

}  // namespace dev
}  // namespace mfp
