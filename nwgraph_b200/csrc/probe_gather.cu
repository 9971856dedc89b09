// Measured ceiling of random 4-byte gathers from an L2-resident table.
//
// The pull sweep's cold gathers are `ld.global.nc.L1::no_allocate` with an L2
// evict-last hint (ld_gather_cold): every one costs one L1-to-L2 request for a
// 32-byte sector, and on a graph whose contribution vector fits in L2 the rate
// of those requests, not DRAM bandwidth, bounds the sweep. This probe issues
// the same load, 8 in flight per thread, from one 1024-thread CTA per SM (the
// sweep's launch shape), at uniformly random indices into a table of
// 2^log2_len floats, and reports loads per second. It is a measuring tool for
// the benchmark, not part of the solve.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace {

__global__ void __launch_bounds__(1024, 1) gather_probe_kernel(const float* __restrict__ table, uint32_t mask,
                                                               uint32_t iters, float* __restrict__ sink) {
  const uint64_t pol = nwgpu::policy_evict_last();
  uint32_t       x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 0x9e3779b9u;
  float          acc = 0.f;
  for (uint32_t i = 0; i < iters; ++i) {
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      x ^= x << 13;  // xorshift32
      x ^= x >> 17;
      x ^= x << 5;
      v[q] = nwgpu::ld_gather_cold(table + (x & mask), pol);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += v[q];
  }
  if (acc == -1.0f) sink[0] = acc;  // never true for the table's contents; keeps the loads
}

__global__ void fill_kernel(float* t, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    t[i] = 1.0f / (float)(1u + (uint32_t)(i & 1023u));
}

}  // namespace

// Loads per second (best of `reps` timed launches after one warm-up launch) and
// that launch's milliseconds. Returns 0 or a cudaError_t value. Uses the
// current device; allocates and frees its own table.
extern "C" int nwprobe_gather_rate(uint32_t log2_len, uint32_t iters, uint32_t reps, double* loads_per_s,
                                   double* best_ms) {
  if (log2_len < 10 || log2_len > 30 || iters == 0 || reps == 0 || !loads_per_s || !best_ms)
    return (int)cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return (int)e;
  const uint64_t n = 1ull << log2_len;
  float*         table = nullptr;
  float*         sink = nullptr;
  cudaEvent_t    e0 = nullptr, e1 = nullptr;
  if ((e = cudaMalloc(&table, n * sizeof(float))) != cudaSuccess) return (int)e;
  if ((e = cudaMalloc(&sink, sizeof(float))) == cudaSuccess && (e = cudaEventCreate(&e0)) == cudaSuccess &&
      (e = cudaEventCreate(&e1)) == cudaSuccess) {
    fill_kernel<<<sms * 8, 256>>>(table, n);
    gather_probe_kernel<<<sms, 1024>>>(table, (uint32_t)(n - 1), iters, sink);  // warm-up: the table into L2
    e = cudaGetLastError();
    float best = 0.f;
    for (uint32_t r = 0; r < reps && e == cudaSuccess; ++r) {
      cudaEventRecord(e0);
      gather_probe_kernel<<<sms, 1024>>>(table, (uint32_t)(n - 1), iters, sink);
      cudaEventRecord(e1);
      if ((e = cudaEventSynchronize(e1)) == cudaSuccess) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r == 0 || ms < best) best = ms;
      }
    }
    if (e == cudaSuccess) {
      const double loads = (double)sms * 1024.0 * (double)iters * 8.0;
      *best_ms = best;
      *loads_per_s = loads / (best * 1e-3);
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(sink);
  cudaFree(table);
  return (int)e;
}
