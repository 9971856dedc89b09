// Autotuners of the sweeps' launch parameters: the destination-blocked sweep
// (autotune_blocked, below) and the degree-binned sweep.
//
// No counterpart in the reference (its page_rank has no tunables beyond the
// TBB grain). The binned sweep's runtime knobs are the launch shape (one
// 1024-thread CTA per SM with the hub contributions staged in shared memory,
// or four 256-thread CTAs per SM with the hubs in L1), how many hub
// contributions the hot shape stages, how many more ids go through L1 with
// an evict-last policy, the long-row cut-offs (the row length above which
// rows are cut into chunks, one warp each, and the chunk length) and the rows
// per warp of bin 0 (two, half a warp each, or one). The tuner times a few
// sweeps of each candidate on the resident graph with unit degrees and keeps
// the fastest: first the cut-offs at the default launch shape, then bin 0's
// rows per warp, then the launch shapes and hub tiers.
// Launch shape and hub tiers do not change the summation order (ranks are
// bitwise equal whichever is chosen); the cut-offs and bin 0's rows per warp
// do (a chunked row is summed per chunk, then over the chunks; a bin-0 row
// over 16 or 32 lanes), so a tuned graph gives the ranks of an untuned one
// created with the same NWGPU_LONG_ROW, NWGPU_CHUNK_ENTRIES and
// NWGPU_BIN0_ROWS, bit for bit, and the graph info reports all three.
//
// Choices are cached per graph signature -- the SM count, log2 of the vertex
// count in half steps, the average degree, and the share of entries in
// chunked long rows and in warp-per-row rows (5% steps) -- in the process and,
// when NWGPU_TUNE_CACHE names a file, in that file (one line per signature),
// so a graph like one already tuned reuses its choice without timing.
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "handle.h"

namespace nwgpu {
namespace {

struct Choice {
  int      hot = 1;
  uint32_t smem_ids = 0, l1_ids = 0;
  float    us = 0.f;  // measured time per sweep
  uint32_t long_row = kLongRow, chunk = kChunk, bin0_rows = kBin0Rows;
};

std::mutex                    g_mu;
std::map<std::string, Choice> g_cache;
bool                          g_loaded = false;

const char* cache_path() {
  const char* p = getenv("NWGPU_TUNE_CACHE");
  return (p && *p) ? p : nullptr;
}

void load_locked() {
  if (g_loaded) return;
  g_loaded = true;
  const char* path = cache_path();
  if (!path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  char line[512];
  while (fgets(line, sizeof line, f)) {
    char*  tab = strchr(line, '\t');
    Choice c;
    if (!tab) continue;
    *tab = 0;
    // hot smem_ids l1_ids us [long_row chunk [bin0_rows]]
    if (sscanf(tab + 1, "%d %u %u %f %u %u %u", &c.hot, &c.smem_ids, &c.l1_ids, &c.us, &c.long_row, &c.chunk,
               &c.bin0_rows) >= 4) {
      if (c.bin0_rows != 1u && c.bin0_rows != 2u) c.bin0_rows = kBin0Rows;
      g_cache[line] = c;
    }
  }
  fclose(f);
}

void store_locked(const std::string& sig, const Choice& c) {
  g_cache[sig] = c;
  const char* path = cache_path();
  if (!path) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s\t%d %u %u %.2f %u %u %u\n", sig.c_str(), c.hot, c.smem_ids, c.l1_ids, c.us, c.long_row, c.chunk,
          c.bin0_rows);
  fclose(f);
}

__global__ void fill_u32_kernel(uint32_t* __restrict__ p, uint64_t n, uint32_t v) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}

// The graph's signature, from the bins at the default cut-offs whatever the
// plan's own are (so a plan built with cached cut-offs finds its entry).
int signature(nwgpu_graph* g, bool shapes_only, std::string* out) {
  uint32_t*     d_out = nullptr;
  uint32_t      h_out[kNumBins + 2];
  uint32_t      at[2] = {0, 0};  // row_ptr at the end of the long rows and of bin 0
  CK(pool_alloc((void**)&d_out, (kNumBins + 3) * sizeof(uint32_t), g->stream), "signature");
  unsigned int* d_bad = reinterpret_cast<unsigned int*>(d_out + kNumBins + 2);
  cudaError_t   e = cudaMemsetAsync(d_bad, 0, sizeof(unsigned int), g->stream);
  if (e == cudaSuccess) e = launch_bin_bounds(g->g.row_ptr, (uint32_t)g->n, kLongRow, kChunk, d_out, d_bad, g->sms, g->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_out, d_out, sizeof(h_out), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  pool_free(d_out, g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "signature");
  CK(cudaMemcpyAsync(&at[0], g->g.row_ptr + h_out[0], sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream), "signature");
  CK(cudaMemcpyAsync(&at[1], g->g.row_ptr + h_out[1], sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream), "signature");
  CK(cudaStreamSynchronize(g->stream), "signature");
  const double nnz = g->nnz ? (double)g->nnz : 1.0;
  const double n = g->n ? (double)g->n : 1.0;
  auto         pct5 = [&](double x) { return (int)(std::lround(20.0 * x / nnz) * 5); };
  char         buf[160];
  snprintf(buf, sizeof buf, "%s sms=%d log2n=%.1f deg=%ld long=%d%% warp=%d%%",
           shapes_only ? "binned-shapes" : "binned", g->sms, std::round(2.0 * std::log2(n)) / 2.0,
           std::lround(nnz / n), pct5(at[0]), pct5((double)at[1] - at[0]));
  *out = buf;
  return NWGPU_OK;
}

int apply(nwgpu_graph* g, const Choice& c) {
  int rc = rebuild_bin_plan(g, c.long_row, c.chunk, c.bin0_rows);
  if (rc) return rc;
  BinPlan& p = g->plan;
  p.hot = c.hot != 0;
  p.bin.smem_ids = c.smem_ids;
  p.bin.l1_ids = c.l1_ids;
  p.sweep_grid = binned_sweep_grid(g->sms, p.hot);
  return NWGPU_OK;
}

// Microseconds per sweep of the plan's current settings (after one warm sweep).
int time_plan(nwgpu_graph* g, const SweepArgs& a, int sweeps, float* us) {
  const BinPlan&   p = g->plan;
  const BinnedArgs ba = make_binned_args(g, p, a, kModePlain);
  CK(launch_binned_sweep(ba, p.hot, kModePlain, p.sweep_grid, p.finish_grid, g->stream), "tune sweep");
  CK(cudaEventRecord(g->ev0, g->stream), "cudaEventRecord");
  for (int i = 0; i < sweeps; ++i)
    CK(launch_binned_sweep(ba, p.hot, kModePlain, p.sweep_grid, p.finish_grid, g->stream), "tune sweep");
  CK(cudaEventRecord(g->ev1, g->stream), "cudaEventRecord");
  CK(cudaEventSynchronize(g->ev1), "tune sweep");
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, g->ev0, g->ev1), "cudaEventElapsedTime");
  *us = 1e3f * ms / (float)sweeps;
  return NWGPU_OK;
}

// Microseconds per sweep of the blocked plan's current settings (after one warm sweep).
int time_blocked(nwgpu_graph* g, const SweepArgs& a, int sweeps, float* us) {
  const BlockPlan&  p = g->bplan;
  const BlockedArgs ba = make_blocked_args(p, a, g->n);
  CK(launch_blocked_sweep(ba, p.sweep_grid, p.loads, g->stream), "tune sweep");
  CK(cudaEventRecord(g->ev0, g->stream), "cudaEventRecord");
  for (int i = 0; i < sweeps; ++i) CK(launch_blocked_sweep(ba, p.sweep_grid, p.loads, g->stream), "tune sweep");
  CK(cudaEventRecord(g->ev1, g->stream), "cudaEventRecord");
  CK(cudaEventSynchronize(g->ev1), "tune sweep");
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, g->ev0, g->ev1), "cudaEventElapsedTime");
  *us = 1e3f * ms / (float)sweeps;
  return NWGPU_OK;
}

// Timing state of a plain solve: unit degrees, uniform start, a sweep limit
// never reached, threshold 0 (never converged).
int start_timing(nwgpu_graph* g, SweepArgs* a) {
  int rc = ensure_solve_buffers(g);
  if (rc) return rc;
  fill_u32_kernel<<<g->sms * 4, 256, 0, g->stream>>>(g->deg, g->n, 1u);
  CK(cudaGetLastError(), "tune degrees");
  PrState h = {};
  h.max_iters = ~0ull;
  h.chunk_end = ~0ull;
  h.threshold = 0.0;
  *g->h_st = h;
  CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, g->stream), "tune state");
  const float base = (float)(0.15 / (double)g->n);
  *a = make_sweep_args(g, 0.85f, base, kTeleportUniform, 0u);
  CK(launch_pr_init(*a, g->n, (float)(1.0 / (double)g->n), g->sms, g->stream), "tune init");
  return NWGPU_OK;
}

}  // namespace

// The blocked sweep's knobs: entries in flight per thread (4, 8, 16) and the
// largest work item (nnz / (f * SMs) entries for f = 1, 2, 4). The row sums
// are exact, so every choice gives bitwise-equal ranks; the tuner only times.
// Cached like the binned choices, under a "blocked" signature (SM count,
// log2 n in half steps, average degree, share of entries in the first
// block); the cache line's fields hold the loads and f.
int autotune_blocked(nwgpu_graph* g) {
  BlockPlan& p = g->bplan;
  if (!p.ok || g->n == 0 || g->nnz == 0) return NWGPU_OK;
  const double nnz = (double)g->nnz, n = (double)g->n;
  char         buf[160];
  snprintf(buf, sizeof buf, "blocked sms=%d log2n=%.1f deg=%ld first=%d%%", g->sms, std::round(2.0 * std::log2(n)) / 2.0,
           std::lround(nnz / n), (int)(std::lround(20.0 * (double)(p.block_ptr[1] - p.block_ptr[0]) / nnz) * 5));
  const std::string sig = buf;
  auto piece_of = [&](int f) { return std::max<uint64_t>(1ull << 16, g->nnz / ((uint64_t)g->sms * (uint64_t)f)); };
  {
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_cache.find(sig);
    if (it != g_cache.end()) {
      const Choice c = it->second;
      p.loads = c.hot;
      CK(set_block_items(&p, g->sms, piece_of((int)c.smem_ids), g->stream), "blocked work list");
      g->tuned = 2;
      g->tune_us = c.us;
      return NWGPU_OK;
    }
  }
  SweepArgs a;
  int       rc = start_timing(g, &a);
  if (rc) return rc;
  const int sweeps = g->nnz > (1u << 26) ? 3 : 8;
  Choice    best;
  best.us = 3.4e38f;
  for (int f : {1, 2, 4}) {
    CK(set_block_items(&p, g->sms, piece_of(f), g->stream), "blocked work list");
    for (int loads : {4, 8, 16}) {
      p.loads = loads;
      float us = 0.f;
      if ((rc = time_blocked(g, a, sweeps, &us))) return rc;
      if (us < best.us) {
        best.hot = loads;
        best.smem_ids = (uint32_t)f;
        best.l1_ids = 0;
        best.us = us;
      }
    }
  }
  p.loads = best.hot;
  CK(set_block_items(&p, g->sms, piece_of((int)best.smem_ids), g->stream), "blocked work list");
  g->tuned = 1;
  g->tune_us = best.us;
  std::lock_guard<std::mutex> lk(g_mu);
  store_locked(sig, best);
  return NWGPU_OK;
}

int cached_cutoffs(nwgpu_graph* g, uint32_t* long_row, uint32_t* chunk, uint32_t* bin0_rows) {
  if (g->n == 0) return NWGPU_OK;
  std::string sig;
  int         rc = signature(g, false, &sig);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_mu);
  load_locked();
  auto it = g_cache.find(sig);
  if (it != g_cache.end()) {
    *long_row = it->second.long_row;
    *chunk = it->second.chunk;
    *bin0_rows = it->second.bin0_rows;
  }
  return NWGPU_OK;
}

int autotune_binned(nwgpu_graph* g, bool shapes_only) {
  if (!g->plan.ok || g->n == 0) return NWGPU_OK;
  std::string sig;
  int         rc = signature(g, shapes_only, &sig);
  if (rc) return rc;
  const uint32_t lim = binned_hot_capacity();
  const uint32_t n = (uint32_t)g->n;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_cache.find(sig);
    if (it != g_cache.end()) {
      Choice c = it->second;
      if (c.smem_ids > lim) c.smem_ids = lim;
      if (c.smem_ids > n) c.smem_ids = n & ~3u;
      if (c.l1_ids < c.smem_ids) c.l1_ids = c.smem_ids;
      if ((rc = apply(g, c))) return rc;
      g->tuned = 2;
      g->tune_us = c.us;
      return NWGPU_OK;
    }
  }
  SweepArgs a;
  if ((rc = start_timing(g, &a))) return rc;
  const int sweeps = g->nnz > (1u << 26) ? 3 : 8;
  // Long-row cut-offs (row length above which rows are chunked, chunk length)
  // at the plan's launch shape and hub tiers; the default pair first, so a
  // tie keeps it. shapes_only: the plan's own cut-offs (cached under their
  // own signature, so the two kinds of choice never mix).
  Choice best;
  best.us = 3.4e38f;
  best.long_row = g->plan.bin.long_row;
  best.chunk = g->plan.bin.chunk;
  best.bin0_rows = g->plan.bin.bin0_rows;
  if (!shapes_only) {
    static const uint32_t cuts[][2] = {{kLongRow, kChunk}, {1024, 512}, {1024, 1024}, {4096, 1024},
                                       {4096, 2048}, {8192, 2048}, {512, 512}};
    Choice c;
    c.hot = g->plan.hot ? 1 : 0;
    c.smem_ids = g->plan.bin.smem_ids;
    c.l1_ids = g->plan.bin.l1_ids;
    c.bin0_rows = kBin0Rows;
    for (const auto& cut : cuts) {
      c.long_row = cut[0];
      c.chunk = cut[1];
      if ((rc = apply(g, c))) return rc;
      float us = 0.f;
      if ((rc = time_plan(g, a, sweeps, &us))) return rc;
      c.us = us;
      if (us < best.us) best = c;
    }
    // bin 0 at the chosen cut-offs: a warp per row instead of half a warp
    // (only when the bin has rows; the two differ in nothing else)
    c = best;
    c.bin0_rows = 1u;
    if ((rc = apply(g, c))) return rc;
    if (g->plan.bin.bin_row_end[0] > g->plan.bin.bin_row_begin[0]) {
      float us = 0.f;
      if ((rc = time_plan(g, a, sweeps, &us))) return rc;
      c.us = us;
      if (us < best.us) best = c;
    }
  }
  // Candidates at those cut-offs: the hot shape with 16K / 32K / 48K staged
  // ids (as the shared memory allows) and an L1 tier of 0 / 16K / 32K more;
  // the 256-thread shape with 16K / 32K / 64K ids through L1.
  const uint32_t long_row = best.long_row, chunk = best.chunk, bin0_rows = best.bin0_rows;
  std::vector<Choice> cands;
  for (uint32_t s : {16384u, 32768u, 49152u}) {
    uint32_t st = s < lim ? s : lim;
    if (st > n) st = n & ~3u;
    for (uint32_t l1 : {0u, 16384u, 32768u}) {
      Choice c;
      c.hot = 1;
      c.smem_ids = st;
      c.l1_ids = st + l1;
      c.long_row = long_row;
      c.chunk = chunk;
      c.bin0_rows = bin0_rows;
      bool dup = false;
      for (const Choice& d : cands) dup |= d.hot == 1 && d.smem_ids == c.smem_ids && d.l1_ids == c.l1_ids;
      if (!dup) cands.push_back(c);
    }
  }
  for (uint32_t l1 : {16384u, 32768u, 65536u}) {
    Choice c;
    c.hot = 0;
    c.l1_ids = l1;
    c.long_row = long_row;
    c.chunk = chunk;
    c.bin0_rows = bin0_rows;
    cands.push_back(c);
  }
  for (Choice c : cands) {
    if ((rc = apply(g, c))) return rc;
    float us = 0.f;
    if ((rc = time_plan(g, a, sweeps, &us))) return rc;
    c.us = us;
    if (us < best.us) best = c;
  }
  if ((rc = apply(g, best))) return rc;
  g->tuned = 1;
  g->tune_us = best.us;
  std::lock_guard<std::mutex> lk(g_mu);
  store_locked(sig, best);
  return NWGPU_OK;
}

}  // namespace nwgpu
