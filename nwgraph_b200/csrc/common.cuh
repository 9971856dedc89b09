// Device helpers shared by the PageRank kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nwgpu {

constexpr unsigned kFullMask = 0xffffffffu;

// Streaming loads/stores for arrays touched once per sweep (col, row_ptr,
// rank, degree): evict-first so the gathered contribution vector keeps L2.
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p) { return __ldcs(p); }
__device__ __forceinline__ uint4 ld_stream4(const uint4* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(float* p, float v) { __stcs(p, v); }

// L2 evict-last policy for the gathered vector (PTX createpolicy, sm_80+).
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// L2 evict-first policy for data read or written once per sweep.
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// Read-only gather through L1 with the L2 evict-last hint.
__device__ __forceinline__ float ld_gather(const float* p, uint64_t pol) {
  float v;
  asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
// Cold gather: L2 evict-last, but no L1 allocation, so L1 keeps hot lines.
__device__ __forceinline__ float ld_gather_cold(const float* p, uint64_t pol) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float4 ld_gather4(const float4* p, uint64_t pol) {
  float4 v;
  asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p), "l"(pol));
  return v;
}
// Store of the next sweep's gather source, kept in L2.
__device__ __forceinline__ void st_keep(float* p, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}

__device__ __forceinline__ void st_keep4(float4* p, float4 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z),
               "f"(v.w), "l"(pol)
               : "memory");
}

// Deterministic warp sum: fixed shuffle-down tree, result valid in lane 0.
__device__ __forceinline__ double warp_sum_lane0(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFullMask, v, off);
  return v;
}
__device__ __forceinline__ float warp_sum_lane0(float v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFullMask, v, off);
  return v;
}

}  // namespace nwgpu
