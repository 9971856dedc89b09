// nwgpu_pr_run_noalloc: PageRank with no allocation (declared in include/nwgpu.h).
//
// Some callers must not allocate. Code running under a memory manager that
// owns the whole device (an application's pool, a capped process) cannot have
// a library call cudaMalloc behind its back, and a latency path cannot afford
// the device synchronisation that cudaMalloc / cudaFree may cause. This entry
// point runs the merge-path sweep of pr_plain.cu (the kernel used for graphs
// kept in input order) directly on the caller's device arrays. Everything the
// sweep needs besides its inputs and output lives in one file-scope device
// array of fixed size:
//   contrib ping-pong    2 x (NWGPU_NOALLOC_MAX_VERTICES + kPad) floats
//   tile table           2 x (kMaxTiles + 2) uint32
//   tile partials        2 x (kMaxTiles + 2) floats (cpart, epart)
//   residual partials    kMaxTiles + kMaxTiles / 256 + 2 doubles
//   error trace          kErrCap doubles
//   solve state, validation flags
// which is about 8.8 MB and bounds the graph it can solve.
//
// No cudaMalloc / cudaFree / cudaHostAlloc / stream or event creation is made
// here. The host reads the solve state back into a stack variable.
#include <chrono>
#include <mutex>

#include "handle.h"

namespace nwgpu {
namespace {

constexpr uint64_t kMaxN = NWGPU_NOALLOC_MAX_VERTICES;
constexpr uint64_t kMaxE = NWGPU_NOALLOC_MAX_ENTRIES;
constexpr SweepVariant kVariant{kSweepThreads, 8, false};
constexpr uint64_t kTileItems = (uint64_t)kSweepThreads * 8;
constexpr uint64_t kMaxTiles = (kMaxN + kMaxE + kTileItems - 1) / kTileItems;
constexpr uint64_t kMaxRes = kMaxTiles + kMaxTiles / 256 + 2;  // sweep grid <= tiles, finish grid = ceil(tiles/256)
constexpr uint32_t kErrCap = 4096;

constexpr uint64_t up256(uint64_t b) { return (b + 255) & ~255ull; }
constexpr uint64_t kOffContrib0 = 0;
constexpr uint64_t kOffContrib1 = kOffContrib0 + up256((kMaxN + kPad) * sizeof(float));
constexpr uint64_t kOffTileRow = kOffContrib1 + up256((kMaxN + kPad) * sizeof(float));
constexpr uint64_t kOffTileNnz = kOffTileRow + up256((kMaxTiles + 2) * sizeof(uint32_t));
constexpr uint64_t kOffCpart = kOffTileNnz + up256((kMaxTiles + 2) * sizeof(uint32_t));
constexpr uint64_t kOffEpart = kOffCpart + up256((kMaxTiles + 2) * sizeof(float));
constexpr uint64_t kOffRes = kOffEpart + up256((kMaxTiles + 2) * sizeof(float));
constexpr uint64_t kOffErrHist = kOffRes + up256(kMaxRes * sizeof(double));
constexpr uint64_t kOffState = kOffErrHist + up256((uint64_t)kErrCap * sizeof(double));
constexpr uint64_t kOffFlags = kOffState + up256(sizeof(PrState));
constexpr uint64_t kScratchBytes = kOffFlags + 256;

// The working memory of every no-alloc solve on a device. Everything from
// kOffTileRow on is cleared at the start of each call; the contrib vectors
// are fully written by the init kernel and the first sweep before any read.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex    g_scratch_mu;
void*         g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on device `dev` (the current device),
// looked up on the first call for that device.
int scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(NWGPU_ERR_UNSUPPORTED, "device ordinal %d >= %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void*       p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    if (!p) return fail(NWGPU_ERR_CUDA, "cudaGetSymbolAddress(no-alloc scratch) returned NULL");
    g_scratch_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
  return NWGPU_OK;
}

__global__ void noalloc_state_kernel(PrState* st, unsigned long long max_iters, double threshold) {
  PrState h = {};
  h.max_iters = max_iters;
  h.chunk_end = kGraphChunk;
  h.threshold = threshold;
  h.done = (max_iters == 0ull) ? 1u : 0u;
  *st = h;
}

// The pointer must be device (or managed) memory usable on device `dev`, and
// 16-byte aligned: the sweep's bulk copies start each slice at a 16-byte word
// of the array (they round down at the start; at the end of an array they
// stop before its last partial word, which is read with plain loads).
int check_device_array(const void* p, int dev, const char* name) {
  if (reinterpret_cast<uintptr_t>(p) & 15u) return fail(NWGPU_ERR_INVALID_ARG, "%s is not 16-byte aligned", name);
  cudaPointerAttributes at = {};
  cudaError_t           e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(NWGPU_ERR_INVALID_ARG, "%s is not a CUDA pointer (%s)", name, cudaGetErrorString(e));
  }
  if (at.type == cudaMemoryTypeManaged) return NWGPU_OK;
  if (at.type != cudaMemoryTypeDevice)
    return fail(NWGPU_ERR_INVALID_ARG, "%s must point to device memory (no-alloc solves read their inputs in place)", name);
  if (at.device != dev) return fail(NWGPU_ERR_INVALID_ARG, "%s is on device %d, the current device is %d", name, at.device, dev);
  return NWGPU_OK;
}

}  // namespace
}  // namespace nwgpu

using namespace nwgpu;

extern "C" int nwgpu_pr_run_noalloc(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, uint64_t nnz,
                                    const uint32_t* out_degree, float* ranks, float damping, float threshold,
                                    uint64_t max_iters, void* stream, nwgpu_pr_stats* stats) {
  clear_error();
  if (n > kMaxN)
    return fail(NWGPU_ERR_INVALID_ARG, "n = %llu exceeds the no-alloc limit of %llu vertices (NWGPU_NOALLOC_MAX_VERTICES)",
                (unsigned long long)n, (unsigned long long)kMaxN);
  if (nnz > kMaxE)
    return fail(NWGPU_ERR_INVALID_ARG, "nnz = %llu exceeds the no-alloc limit of %llu entries (NWGPU_NOALLOC_MAX_ENTRIES)",
                (unsigned long long)nnz, (unsigned long long)kMaxE);
  if (!(damping >= 0.0f && damping <= 1.0f)) return fail(NWGPU_ERR_INVALID_ARG, "damping %g outside [0, 1]", (double)damping);
  if (!row_ptr) return fail(NWGPU_ERR_INVALID_ARG, "row_ptr is NULL");
  if (nnz && !col) return fail(NWGPU_ERR_INVALID_ARG, "col is NULL with nnz > 0");
  if (n && (!out_degree || !ranks)) return fail(NWGPU_ERR_INVALID_ARG, "out_degree / ranks is NULL");
  if (stats) {
    double*  eb = stats->errors;
    uint64_t ec = stats->errors_cap;
    memset(stats, 0, sizeof(*stats));
    stats->errors = eb;
    stats->errors_cap = ec;
    stats->bytes_per_iter = 4.0 * (double)nnz + 4.0 * (double)(n + 1) + 20.0 * (double)n;
  }
  if (n == 0) {
    // The reference's sweep reduces over an empty range: error 0.
    const uint64_t its = (max_iters == 0) ? 0 : ((0.0 < (double)threshold) ? 1 : max_iters);
    if (stats) {
      stats->iterations = its;
      stats->converged = its > 0 && 0.0 < (double)threshold;
    }
    return NWGPU_OK;
  }
  int dev = 0, sms = 0;
  int rc = check_device(&dev, &sms);
  if (rc) return rc;
  if ((rc = check_device_array(row_ptr, dev, "row_ptr"))) return rc;
  if (nnz && (rc = check_device_array(col, dev, "col"))) return rc;
  if ((rc = check_device_array(out_degree, dev, "out_degree"))) return rc;
  if ((rc = check_device_array(ranks, dev, "ranks"))) return rc;
  unsigned char* base = nullptr;
  if ((rc = scratch_address(dev, &base))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  float*        contrib0 = reinterpret_cast<float*>(base + kOffContrib0);
  float*        contrib1 = reinterpret_cast<float*>(base + kOffContrib1);
  uint32_t*     tile_row = reinterpret_cast<uint32_t*>(base + kOffTileRow);
  uint32_t*     tile_nnz = reinterpret_cast<uint32_t*>(base + kOffTileNnz);
  float*        cpart = reinterpret_cast<float*>(base + kOffCpart);
  float*        epart = reinterpret_cast<float*>(base + kOffEpart);
  double*       res_part = reinterpret_cast<double*>(base + kOffRes);
  double*       err_hist = reinterpret_cast<double*>(base + kOffErrHist);
  PrState*      st = reinterpret_cast<PrState*>(base + kOffState);
  unsigned int* bad = reinterpret_cast<unsigned int*>(base + kOffFlags);

  // Clear everything but the contrib vectors (tile table, partials, residuals,
  // error trace, state, validation flags).
  CK(cudaMemsetAsync(base + kOffTileRow, 0, kScratchBytes - kOffTileRow, s), "clear no-alloc scratch");

  // Validate before any kernel indexes with these arrays.
  CK(validate_csr(row_ptr, col, n, nnz, bad, sms, s), "validate");
  unsigned int h_bad = 0;
  CK(cudaMemcpyAsync(&h_bad, bad, sizeof(h_bad), cudaMemcpyDeviceToHost, s), "copy validation flags");
  CK(cudaStreamSynchronize(s), "validate");
  if (h_bad)
    return fail(NWGPU_ERR_INVALID_GRAPH, "invalid CSR:%s%s%s", (h_bad & 1u) ? " row_ptr[0] != 0 or row_ptr[n] != nnz;" : "",
                (h_bad & 2u) ? " row_ptr decreases;" : "", (h_bad & 4u) ? " col index >= n;" : "");

  const uint32_t D = kVariant.tile_items();
  const uint32_t T = (uint32_t)((n + nnz + D - 1) / D);
  CK(fill_tiling(row_ptr, n, nnz, D, T, tile_row, tile_nnz, s), "tiling");
  const uint32_t hot_ids = 0xffffffffu;  // input order: every gather may allocate in L1
  const uint64_t want = (uint64_t)sms * (uint64_t)sweep_blocks_per_sm(kVariant, hot_ids);
  const int      grid = (int)(want < T ? want : T);
  const int      finish_grid = finish_grid_for(T);

  noalloc_state_kernel<<<1, 1, 0, s>>>(st, (unsigned long long)max_iters, (double)threshold);
  CK(cudaGetLastError(), "no-alloc state");

  SweepArgs a = {};
  a.row_ptr = row_ptr;
  a.col = col;
  a.tile_row = tile_row;
  a.tile_nnz = tile_nnz;
  a.num_tiles = T;
  a.tile_items = D;
  a.contrib0 = contrib0;
  a.contrib1 = contrib1;
  a.rank = ranks;
  a.deg = out_degree;
  a.cpart = cpart;
  a.epart = epart;
  a.res_part = res_part;
  a.sweep_grid = (uint32_t)grid;
  a.st = st;
  a.err_hist = err_hist;
  a.err_cap = kErrCap;
  a.abort_word = nullptr;
  a.use_cond = 0;
  a.damping = damping;
  // page_rank.hpp:92-94: N = graph.size(); constants in double, stored as Real.
  a.base = (float)((1.0 - (double)damping) / (double)n);
  a.teleport = kTeleportUniform;
  a.seed = 0;
  a.hot_ids = hot_ids;
  // The caller's arrays end exactly at n + 1, nnz, n and n elements: the
  // tile copies load the last partial 16-byte word of each with plain loads.
  a.exact_ends = 1;
  a.n_rows = (uint32_t)n;
  a.n_entries = (uint32_t)nnz;
  CK(launch_pr_init(a, n, (float)(1.0 / (double)n), sms, s), "pr_init");
  CK(cudaStreamSynchronize(s), "no-alloc set-up");

  const auto t0 = std::chrono::steady_clock::now();
  PrState    fin = {};
  uint64_t   launched = 0;
  for (;;) {
    const uint64_t batch = (max_iters - launched) < kGraphChunk ? (max_iters - launched) : kGraphChunk;
    for (uint64_t b = 0; b < batch; ++b) {
      CK(launch_pr_sweep(a, kVariant, grid, s), "pr_sweep");
      CK(launch_pr_finish(a, finish_grid, s), "pr_finish");
    }
    launched += batch;
    CK(cudaMemcpyAsync(&fin, st, sizeof(PrState), cudaMemcpyDeviceToHost, s), "copy state");
    CK(cudaStreamSynchronize(s), "sweep loop");
    if (fin.done || launched >= max_iters) break;
  }
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (fin.fault) return fail(NWGPU_ERR_CUDA, "a bounded device wait gave up (fault word %u)", fin.fault);
  if (stats) {
    stats->iterations = fin.iter;
    stats->final_error = fin.last_error;
    stats->converged = (int32_t)fin.converged;
    stats->device_ms = ms;
    stats->ms_per_iter = fin.iter ? ms / (double)fin.iter : 0.0;
    stats->gteps = ms > 0 ? (double)nnz * (double)fin.iter / (ms * 1e6) : 0.0;
    if (stats->errors && stats->errors_cap) {
      uint64_t m = fin.iter < stats->errors_cap ? fin.iter : stats->errors_cap;
      if (m > kErrCap) m = kErrCap;
      if (m) {
        CK(cudaMemcpyAsync(stats->errors, err_hist, m * sizeof(double), cudaMemcpyDeviceToHost, s), "copy errors");
        CK(cudaStreamSynchronize(s), "copy errors");
      }
    }
  }
  return NWGPU_OK;
}
