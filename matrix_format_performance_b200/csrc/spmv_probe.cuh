// Load-ceiling probe for SpMV (a measurement kernel, not a format).
//
// It issues the memory operations of an SpMV over nnz (value, column) pairs
// and nothing else: no rows, no reduction by row, one partial sum per CTA.
//   mode 0  stream the values and column ids (16-byte loads), no x gathers
//   mode 1  stream the column ids and gather x[col]
//   mode 2  stream both arrays and gather x[col] (the loads of any format
//           that reads each nonzero and its x entry once)
// Its time on a matrix is a floor for every format's kernel on that matrix:
// whatever a format does by row comes on top of these loads.  The x path is
// selectable to compare the L1-cached read-only gather with L2-only gathers.
#pragma once

#include "spmv_device.cuh"

namespace mfp {
namespace dev {

constexpr int kProbeBlock = 256;
constexpr int kProbeEpt = 8;  // elements per thread per step: two 16-byte loads per array

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
    if (MODE != 1) {
      float a[4], b[4];
      ld_stream4(vals + e, a, pol);
      ld_stream4(vals + e + 4, b, pol);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        v[k] = a[k];
        v[k + 4] = b[k];
      }
    }
    {
      uint32_t a[4], b[4];
      ld_stream4(cols + e, a, pol);
      ld_stream4(cols + e + 4, b, pol);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        c[k] = a[k];
        c[k + 4] = b[k];
      }
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
    const uint32_t c = cols[e];
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

}  // namespace dev
}  // namespace mfp
