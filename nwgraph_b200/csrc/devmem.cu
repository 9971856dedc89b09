// Device memory of graph handles: one stream-ordered pool per device.
//
// A graph handle holds a few arrays of the graph's size, and creating one
// needs temporaries of the same order (the relabelling sort, the chunk table).
// cudaMalloc / cudaFree of GB-sized arrays map and unmap pages and synchronise
// the device; on some machines that cost more than the upload and the solve
// together. The pool keeps freed blocks mapped, so a program that creates
// and destroys handles repeatedly (a service answering one graph per request,
// a benchmark loop) pays the mapping once. The small pinned host blocks of
// the handles' solve states are cached the same way. nwgpu_release_cached_memory()
// hands the unused blocks of both back to the driver.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "handle.h"

namespace nwgpu {
namespace {
constexpr int   kMaxPoolDevices = 64;
std::mutex      g_pool_mu;
cudaMemPool_t   g_pools[kMaxPoolDevices] = {};

cudaError_t pool_for_current(cudaMemPool_t* out) {
  int         dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxPoolDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;  // never trim at stream synchronisation
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return e;
    }
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return cudaSuccess;
}
}  // namespace

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  cudaMemPool_t pool;
  cudaError_t   e = pool_for_current(&pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s);
}

void pool_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

namespace {
std::mutex         g_host_mu;
std::vector<void*> g_host_free;  // cached blocks, each one cudaHostAlloc of kHostBlock bytes
}  // namespace

cudaError_t host_block_get(void** p) {
  *p = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_host_mu);
    if (!g_host_free.empty()) {
      *p = g_host_free.back();
      g_host_free.pop_back();
    }
  }
  if (!*p) {
    cudaError_t e = cudaHostAlloc(p, kHostBlock, cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) {
      *p = nullptr;
      return e;
    }
  }
  memset(*p, 0, kHostBlock);
  return cudaSuccess;
}

void host_block_put(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_host_mu);
  try {
    g_host_free.push_back(p);
  } catch (...) {
    cudaFreeHost(p);
  }
}

}  // namespace nwgpu

extern "C" int nwgpu_release_cached_memory(void) {
  nwgpu::clear_error();
  std::lock_guard<std::mutex> lock(nwgpu::g_pool_mu);
  for (int d = 0; d < nwgpu::kMaxPoolDevices; ++d) {
    if (!nwgpu::g_pools[d]) continue;
    cudaError_t e = cudaMemPoolTrimTo(nwgpu::g_pools[d], 0);
    if (e != cudaSuccess) return nwgpu::cuda_fail(e, "cudaMemPoolTrimTo");
  }
  std::lock_guard<std::mutex> hlock(nwgpu::g_host_mu);
  for (void* p : nwgpu::g_host_free) cudaFreeHost(p);
  nwgpu::g_host_free.clear();
  return NWGPU_OK;
}
