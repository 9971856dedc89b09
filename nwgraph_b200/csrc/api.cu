// C ABI of the PageRank engine (declared in include/nwgpu.h): graph handles
// and the single-vector solves.
//
// nwgpu_graph_create uploads and validates the CSR once, relabels it (hubs
// first) and tiles it on the device; nwgpu_pr_run replaces the body of
// nw::graph::page_rank / page_rank_v10 (include/nwgraph/algorithms/page_rank.hpp:92-147,
// include/nwgraph/experimental/algorithms/page_rank.hpp:383-431) with one
// CUDA-graph launch whose while loop runs the sweep and finishing kernels
// until the device-side test "error < threshold" or max_iters stops it.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <new>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "handle.h"

using namespace nwgpu;

namespace nwgpu {

namespace {
thread_local std::string g_last_error;
std::once_flag           g_config_once;
cudaError_t              g_config_err = cudaSuccess;
constexpr int            kDefaultIpt = 8;
constexpr uint32_t       kDefaultHotIds = 32768;
constexpr uint32_t       kHotL1Ids = 16384;   // ids past the staged ones that still go through L1 (hot variant)
constexpr uint32_t       kHotSmemIds = 32768; // staged ids by default (128 KB of shared memory)

// NWGPU_TRACE=1 prints "# [ phase ]: X ms" lines to stderr, like the
// reference's life_timer (include/nwgraph/util/timer.hpp:120-133).
struct PhaseTimer {
  bool                                           on;
  cudaStream_t                                   s;
  std::chrono::high_resolution_clock::time_point t0;
  explicit PhaseTimer(cudaStream_t st) : on(getenv("NWGPU_TRACE") != nullptr), s(st) {
    if (on) t0 = std::chrono::high_resolution_clock::now();
  }
  void mark(const char* what) {
    if (!on) return;
    cudaStreamSynchronize(s);
    auto t1 = std::chrono::high_resolution_clock::now();
    fprintf(stderr, "# [ nwgpu %s ]: %.3f ms\n", what, std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  }
};

int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  if (!v || !*v) return dflt;
  return atoi(v);
}

// Column ids per upload chunk of the streamed build (NWGPU_UPLOAD_CHUNK_ENTRIES
// overrides; CSRs with at most one chunk of entries are uploaded in one piece).
constexpr uint64_t kUploadChunkEntries = 32ull << 20;
constexpr uint64_t kMaxUploadChunks = 256;

// Merge-path row of diagonal d over a host copy of the row pointers: rows
// [0, i) end before item d (the device's merge_path_row). Indexes [0, n] only.
uint64_t host_merge_row(const uint32_t* rp, uint64_t n, uint64_t nnz, uint64_t d) {
  uint64_t lo = d > nnz ? d - nnz : 0, hi = d < n ? d : n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if ((uint64_t)rp[mid + 1] + mid + 1 <= d)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

const char* csr_error_text(unsigned int bits, char* buf, size_t len) {
  snprintf(buf, len, "%s%s%s", (bits & 1u) ? " row_ptr[0] != 0 or row_ptr[n] != nnz;" : "",
           (bits & 2u) ? " row_ptr decreases;" : "", (bits & 4u) ? " col index >= n;" : "");
  return buf;
}

// Upload, validation and relabelling of a host CSR with the column ids still
// in flight. The row pointers go first and are checked before any kernel
// indexes with them. The column ids follow in merge-path chunks on a second
// stream while the rows are sorted, and each chunk's entries are placed in the
// relabelled CSR (ids checked) as soon as the chunk has arrived. The result is
// the relabelled CSR of the one-piece path, entry for entry.
int upload_streamed(nwgpu_graph* g, const uint32_t* h_row_ptr, const uint32_t* h_col, uint64_t n, uint64_t nnz,
                    uint64_t chunk, PhaseTimer& trace) {
  cudaStream_t             s = g->stream, cs = nullptr;
  const uint64_t           C = std::min((nnz + chunk - 1) / chunk, kMaxUploadChunks);
  std::vector<cudaEvent_t> ev(C, nullptr);
  std::vector<uint64_t>    dg(C + 1), kk(C + 1);
  uint32_t *               d_rp = nullptr, *d_col = nullptr;
  unsigned int*            d_err = nullptr;
  unsigned int             h_err = 0;
  char                     why[160];
  auto                     done = [&](int code) {
    if (cs) cudaStreamSynchronize(cs);  // no copy may still write d_col when it is freed
    cudaStreamSynchronize(s);
    for (cudaEvent_t x : ev)
      if (x) cudaEventDestroy(x);
    if (cs) cudaStreamDestroy(cs);
    pool_free(d_rp, s);
    pool_free(d_col, s);
    pool_free(d_err, s);
    return code;
  };
  cudaError_t e;
  if ((e = dalloc(g, &d_rp, n + 1)) != cudaSuccess || (e = pool_alloc_n(&d_col, nnz + kPad, s)) != cudaSuccess ||
      (e = pool_alloc_n(&d_err, 1, s)) != cudaSuccess)
    return done(cuda_fail(e, "cudaMalloc(CSR)"));
  if ((e = cudaMemsetAsync(d_err, 0, sizeof(unsigned int), s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(d_rp, h_row_ptr, (n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = validate_row_ptr(d_rp, n, nnz, d_err, g->sms, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(&h_err, d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return done(cuda_fail(e, "upload row_ptr"));
  // Chunk c holds merge-path items [dg[c], dg[c+1]) and so entries [kk[c], kk[c+1]).
  // Clamped, so the copies stay inside col whatever the row pointers hold;
  // with valid row pointers the clamps change nothing.
  for (uint64_t c = 0; c <= C; ++c) {
    dg[c] = (n + nnz) * c / C;
    uint64_t k = c == C ? nnz : dg[c] - host_merge_row(h_row_ptr, n, nnz, dg[c]);
    if (c && k < kk[c - 1]) k = kk[c - 1];
    kk[c] = k < nnz ? k : nnz;
  }
  if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) return done(cuda_fail(e, "cudaStreamCreate"));
  for (uint64_t c = 0; c < C; ++c) {
    if ((e = cudaEventCreateWithFlags(&ev[c], cudaEventDisableTiming)) != cudaSuccess ||
        (kk[c + 1] > kk[c] && (e = cudaMemcpyAsync(d_col + kk[c], h_col + kk[c], (kk[c + 1] - kk[c]) * sizeof(uint32_t),
                                                   cudaMemcpyHostToDevice, cs)) != cudaSuccess) ||
        (e = cudaEventRecord(ev[c], cs)) != cudaSuccess)
      return done(cuda_fail(e, "upload col"));
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return done(cuda_fail(e, "validate row_ptr"));
  if (h_err) return done(fail(NWGPU_ERR_INVALID_GRAPH, "invalid CSR:%s", csr_error_text(h_err, why, sizeof(why))));
  trace.mark("upload row_ptr + validate");
  if ((e = relabel_rows(d_rp, n, nnz, g->sms, false, false, &g->g, s)) != cudaSuccess) return done(cuda_fail(e, "relabel"));
  for (uint64_t c = 0; c < C; ++c) {
    if ((e = cudaStreamWaitEvent(s, ev[c], 0)) != cudaSuccess ||
        (e = scatter_entries(d_rp, d_col, n, nnz, dg[c], dg[c + 1], g->g, d_err, g->sms, s)) != cudaSuccess)
      return done(cuda_fail(e, "relabel entries"));
  }
  if ((e = cudaMemcpyAsync(&h_err, d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return done(cuda_fail(e, "relabel entries"));
  if (h_err) return done(fail(NWGPU_ERR_INVALID_GRAPH, "invalid CSR:%s", csr_error_text(h_err, why, sizeof(why))));
  g->relabelled = true;
  trace.mark("upload col + relabel");
  return done(NWGPU_OK);
}
}  // namespace

int fail(int code, const char* fmt, ...) {
  char    buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) return fail(NWGPU_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return fail(NWGPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void clear_error() { g_last_error.clear(); }

const std::string& last_error_text() { return g_last_error; }

int check_device(int* dev_out, int* sms_out) {
  int         dev = 0, count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(NWGPU_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
  }
  CK(cudaGetDevice(&dev), "cudaGetDevice");
  int major = 0, sms = 0;
  CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev), "cudaDeviceGetAttribute");
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
  if (major != 10) return fail(NWGPU_ERR_NO_DEVICE, "device %d is sm_%d0, this build targets sm_100a only", dev, major);
  std::call_once(g_config_once, [] {
    g_config_err = configure_sweep_kernels();
    if (g_config_err == cudaSuccess) g_config_err = configure_binned_kernels();
    if (g_config_err == cudaSuccess) g_config_err = configure_blocked_kernels();
  });
  if (g_config_err != cudaSuccess) return cuda_fail(g_config_err, "configure kernels");
  *dev_out = dev;
  *sms_out = sms;
  return NWGPU_OK;
}

uint64_t residual_parts(const nwgpu_graph* g) {
  uint64_t parts = (uint64_t)g->grid + (uint64_t)g->finish_grid;
  if (g->plan.ok) {
    const int      a = binned_sweep_grid(g->sms, false), b = binned_sweep_grid(g->sms, true);
    const uint64_t bp = (uint64_t)(a > b ? a : b) + (uint64_t)g->plan.finish_grid;
    if (bp > parts) parts = bp;
  }
  return parts;
}

int ensure_solve_buffers(nwgpu_graph* g) {
  if (g->solve_ready) return NWGPU_OK;
  const uint64_t n = g->n, T = g->tiling.num_tiles;
  CK(dalloc(g, &g->rank, n), "cudaMalloc(rank)");
  CK(dalloc(g, &g->contrib[0], n), "cudaMalloc(contrib)");
  CK(dalloc(g, &g->contrib[1], n), "cudaMalloc(contrib)");
  CK(dalloc(g, &g->deg, n), "cudaMalloc(deg)");
  CK(dalloc(g, &g->stage_u32, n), "cudaMalloc(staging)");
  CK(dalloc(g, &g->cpart, T + 1), "cudaMalloc(cpart)");
  CK(dalloc(g, &g->epart, T + 1), "cudaMalloc(epart)");
  g->res_parts = residual_parts(g);
  CK(dalloc(g, &g->res_part, g->res_parts), "cudaMalloc(res_part)");
  CK(dalloc(g, &g->st, 1), "cudaMalloc(state)");
  CK(dalloc(g, &g->err_hist, g->err_cap), "cudaMalloc(err_hist)");
  static_assert(sizeof(PrState) <= kHostBlock, "state mirror fits a host block");
  CK(host_block_get((void**)&g->h_st), "cudaHostAlloc(state)");
  CK(host_block_get((void**)&g->h_abort), "cudaHostAlloc(abort)");
  CK(cudaHostGetDevicePointer((void**)&g->d_abort, g->h_abort, 0), "cudaHostGetDevicePointer(abort)");
  CK(cudaEventCreate(&g->ev0), "cudaEventCreate");
  CK(cudaEventCreate(&g->ev1), "cudaEventCreate");
  CK(cudaStreamSynchronize(g->stream), "solve buffers");
  g->solve_ready = true;
  return NWGPU_OK;
}

int load_degrees(nwgpu_graph* g, const uint32_t* out_degree, bool device_ptrs, cudaStream_t s) {
  const uint64_t n = g->n;
  if (g->relabelled) {
    const uint32_t* src = out_degree;
    if (!device_ptrs) {
      CK(cudaMemcpyAsync(g->stage_u32, out_degree, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "copy out_degree");
      src = g->stage_u32;
    }
    CK(launch_gather_u32(src, g->g.inv, g->deg, n, g->sms, s), "permute degrees");
  } else {
    CK(cudaMemcpyAsync(g->deg, out_degree, n * sizeof(uint32_t),
                       device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s),
       "copy out_degree");
  }
  return NWGPU_OK;
}

// Bin tables of the CSR (row_ptr, n rows) for the degree-binned sweep. Rows
// must be in non-increasing length order (relabelled graphs); otherwise
// p->ok stays false and the caller uses another sweep. hot: the launch shape
// with the hub contributions staged in shared memory. Rows of more than
// long_row entries are cut into chunks of `chunk` entries. bin0_rows: rows of
// bin 0 per warp, 2 (half a warp each) or 1 (a whole warp).
int build_bin_plan(nwgpu_graph* g, const uint32_t* row_ptr, uint64_t n64, bool hot, BinPlan* p, uint32_t long_row,
                   uint32_t chunk, uint32_t bin0_rows) {
  if (long_row < 256u || chunk < 256u || chunk % 256u)
    return fail(NWGPU_ERR_INVALID_ARG, "long-row cut-off %u / chunk %u: both >= 256, the chunk a multiple of 256",
                long_row, chunk);
  if (bin0_rows != 1u && bin0_rows != 2u)
    return fail(NWGPU_ERR_INVALID_ARG, "bin-0 rows per warp %u: 1 or 2", bin0_rows);
  const uint32_t n = (uint32_t)n64;
  uint32_t*      d_out = nullptr;
  unsigned int*  d_bad = nullptr;
  CK(pool_alloc((void**)&d_out, (kNumBins + 2) * sizeof(uint32_t) + sizeof(unsigned int), g->stream), "cudaMalloc(bins)");
  d_bad = reinterpret_cast<unsigned int*>(d_out + kNumBins + 2);
  uint32_t     h_out[kNumBins + 2];
  unsigned int h_bad = 0;
  cudaError_t  e = cudaMemsetAsync(d_bad, 0, sizeof(unsigned int), g->stream);
  if (e == cudaSuccess) e = launch_bin_bounds(row_ptr, n, long_row, chunk, d_out, d_bad, g->sms, g->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_out, d_out, sizeof(h_out), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, d_bad, sizeof(h_bad), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  pool_free(d_out, g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "bin bounds");
  if (h_bad) return NWGPU_OK;  // lengths not sorted
  BinnedArgs&    b = p->bin;
  const uint32_t nlong = h_out[0];
  b.long_row = long_row;
  b.chunk = chunk;
  b.bin0_rows = bin0_rows;
  b.num_long_rows = nlong;
  b.num_big_rows = h_out[kNumBins + 1] < nlong ? h_out[kNumBins + 1] : nlong;
  // rows one warp handles in each bin (pr_binned.cu: pair_bin or range_bin, group_bin<G>, empty_rows)
  const uint32_t rows_per_warp[kNumBins] = {bin0_rows, 2, 4, 8, 16, 32, 64, 128};
  uint32_t              warps = 0;
  for (int i = 0; i < kNumBins; ++i) {
    b.bin_row_begin[i] = h_out[i];
    b.bin_row_end[i] = h_out[i + 1];
    const uint64_t rows = h_out[i + 1] - h_out[i];
    warps += (uint32_t)((rows + rows_per_warp[i] - 1) / rows_per_warp[i]);
    b.bin_warp_end[i] = warps;
  }
  // chunk table of the long rows
  CK(dalloc(g, &p->first, (uint64_t)nlong + 1), "cudaMalloc(chunk table)");
  uint32_t num_chunks = 0;
  if (nlong) {
    uint32_t* cnt = nullptr;
    void*     tmp = nullptr;
    size_t    tmp_bytes = 0;
    CK(pool_alloc_n(&cnt, (uint64_t)nlong + 1, g->stream), "cudaMalloc(chunk counts)");
    e = cudaMemsetAsync(cnt + nlong, 0, sizeof(uint32_t), g->stream);
    if (e == cudaSuccess) e = launch_chunk_count(row_ptr, nlong, chunk, cnt, g->sms, g->stream);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, p->first, (int64_t)nlong + 1, g->stream);
    if (e == cudaSuccess) e = pool_alloc(&tmp, tmp_bytes, g->stream);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, p->first, (int64_t)nlong + 1, g->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&num_chunks, p->first + nlong, sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    pool_free(cnt, g->stream);
    pool_free(tmp, g->stream);
    if (e != cudaSuccess) return cuda_fail(e, "chunk table");
  }
  b.num_chunks = num_chunks;
  CK(dalloc(g, &p->chunk_row, (uint64_t)num_chunks), "cudaMalloc(chunk rows)");
  CK(dalloc(g, &p->chunk_part, (uint64_t)num_chunks), "cudaMalloc(chunk partials)");
  CK(launch_chunk_fill(p->first, nlong, p->chunk_row, g->sms, g->stream), "chunk fill");
  CK(cudaStreamSynchronize(g->stream), "chunk fill");
  b.row_first_chunk = p->first;
  b.chunk_row = p->chunk_row;
  b.chunk_part = p->chunk_part;
  // Hot shape: the first NWGPU_HOT_IDS contributions (default kHotSmemIds:
  // half the SM's L1/shared capacity, which leaves L1 room for the next tier
  // of hubs) are staged in shared memory. Otherwise hubs go through L1 only.
  p->hot = hot;
  if (hot) {
    const uint32_t lim = binned_hot_capacity();
    const long     want = env_int("NWGPU_HOT_IDS", -1);
    uint32_t       cap = want >= 0 ? (uint32_t)want & ~3u : kHotSmemIds;
    if (cap > lim) cap = lim;
    b.smem_ids = (uint32_t)(n64 < cap ? n64 & ~3ull : cap);
    b.l1_ids = b.smem_ids + (uint32_t)env_int("NWGPU_HOT_L1_IDS", (int)kHotL1Ids);
  } else {
    b.smem_ids = 0;
    b.l1_ids = g->hot_ids;
  }
  p->sweep_grid = binned_sweep_grid(g->sms, hot);
  p->finish_grid = binned_finish_grid(b);
  p->bytes = ((uint64_t)nlong + 1 + kPad + 2 * ((uint64_t)num_chunks + kPad)) * sizeof(uint32_t);
  p->ok = true;
  return NWGPU_OK;
}

int rebuild_bin_plan(nwgpu_graph* g, uint32_t long_row, uint32_t chunk, uint32_t bin0_rows) {
  BinPlan&       p = g->plan;
  if (!p.ok) return NWGPU_OK;
  if (p.bin.long_row == long_row && p.bin.chunk == chunk && p.bin.bin0_rows == bin0_rows) return NWGPU_OK;
  const bool     hot = p.hot;
  const uint32_t smem = p.bin.smem_ids, l1 = p.bin.l1_ids;
  CK(cudaStreamSynchronize(g->stream), "bin plan");
  g->device_bytes -= p.bytes;
  p.release(g->stream);
  const int rc = build_bin_plan(g, g->g.row_ptr, g->n, hot, &p, long_row, chunk, bin0_rows);
  if (rc) return rc;
  p.bin.smem_ids = smem;
  p.bin.l1_ids = l1;
  g->cg_plan = nullptr;  // a cached loop graph holds the old tables
  // more long rows can mean more finishing CTAs, each writing a residual partial
  if (g->solve_ready && residual_parts(g) > g->res_parts) {
    CK(cudaStreamSynchronize(g->stream), "residual partials");
    pool_free(g->res_part, g->stream);
    g->device_bytes -= (g->res_parts + kPad) * sizeof(double);
    g->res_part = nullptr;
    g->res_parts = residual_parts(g);
    CK(dalloc(g, &g->res_part, g->res_parts), "cudaMalloc(res_part)");
    CK(cudaStreamSynchronize(g->stream), "residual partials");
  }
  return NWGPU_OK;
}

void BinPlan::release(cudaStream_t s) {
  pool_free(first, s);
  pool_free(chunk_row, s);
  pool_free(chunk_part, s);
  *this = BinPlan();
}

// Sweep grid of a binned solve: the plan's, except the weighted and adjoint
// sweeps, which always run in the hot launch shape.
int binned_grid(nwgpu_graph* g, const BinPlan& p, int mode) {
  return mode == kModePlain ? p.sweep_grid : binned_sweep_grid(g->sms, true);
}

BinnedArgs make_binned_args(nwgpu_graph* g, const BinPlan& p, const SweepArgs& sw, int mode) {
  BinnedArgs b = p.bin;
  b.sw = sw;
  b.sw.sweep_grid = (uint32_t)binned_grid(g, p, mode);
  return b;
}

SweepArgs make_sweep_args(nwgpu_graph* g, float damping, float base, int teleport, uint32_t seed) {
  SweepArgs a = {};
  a.row_ptr = g->g.row_ptr;
  a.col = g->g.col;
  a.tile_row = g->tiling.tile_row;
  a.tile_nnz = g->tiling.tile_nnz;
  a.num_tiles = g->tiling.num_tiles;
  a.tile_items = g->tiling.tile_items;
  a.contrib0 = g->contrib[0];
  a.contrib1 = g->contrib[1];
  a.rank = g->rank;
  a.deg = g->deg;
  a.cpart = g->cpart;
  a.epart = g->epart;
  a.res_part = g->res_part;
  a.sweep_grid = (uint32_t)g->grid;
  a.st = g->st;
  a.err_hist = g->err_hist;
  a.err_cap = g->err_cap;
  a.abort_word = g->d_abort;
  a.use_cond = 0;
  a.damping = damping;
  a.base = base;
  a.teleport = teleport;
  a.seed = seed;
  a.hot_ids = g->hot_ids;
  return a;
}

bool use_blocked(const nwgpu_graph* g, const BinPlan* plan, int mode) {
  return g->bplan.ok && !g->blocked_off && mode == kModePlain && (plan == nullptr || plan == &g->plan);
}

int build_loop_graph(nwgpu_graph* g, const SweepArgs& proto, const BinPlan* plan, int mode) {
  if (g->cg_exec) {
    cudaGraphExecDestroy(g->cg_exec);
    g->cg_exec = nullptr;
  }
  if (g->cg) {
    cudaGraphDestroy(g->cg);
    g->cg = nullptr;
  }
  CK(cudaGraphCreate(&g->cg, 0), "cudaGraphCreate");
  cudaGraphNode_t arm;
  CK(add_pr_arm_node(g->cg, g->st, &arm), "cudaGraphAddKernelNode(arm)");
  cudaGraphConditionalHandle cond;
  CK(cudaGraphConditionalHandleCreate(&cond, g->cg, 1u, cudaGraphCondAssignDefault), "cudaGraphConditionalHandleCreate");
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wnode;
  CK(cudaGraphAddNode(&wnode, g->cg, &arm, 1, &cp), "cudaGraphAddNode(while)");
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  SweepArgs   a = proto;
  a.cond = cond;
  a.use_cond = 1;
  if (use_blocked(g, plan, mode))
    CK(add_blocked_nodes(body, make_blocked_args(g->bplan, a, g->n), g->bplan.sweep_grid, g->bplan.loads),
       "cudaGraphAddKernelNode(blocked)");
  else if (plan)
    CK(add_binned_nodes(body, make_binned_args(g, *plan, a, mode), plan->hot, mode, binned_grid(g, *plan, mode),
                        plan->finish_grid),
       "cudaGraphAddKernelNode(binned)");
  else
    CK(add_pr_sweep_nodes(body, a, g->variant, g->grid, g->finish_grid), "cudaGraphAddKernelNode(sweep)");
  CK(cudaGraphInstantiate(&g->cg_exec, g->cg, 0), "cudaGraphInstantiate");
  g->cg_args = proto;
  g->cg_plan = plan;
  g->cg_mode = mode;
  g->cg_blocked = use_blocked(g, plan, mode);
  return NWGPU_OK;
}

// The arguments a cached loop graph baked in.
bool same_loop(const nwgpu_graph* g, const SweepArgs& y, const BinPlan* plan, int mode) {
  const SweepArgs& x = g->cg_args;
  return g->cg_plan == plan && g->cg_mode == mode && g->cg_blocked == use_blocked(g, plan, mode) &&
         x.damping == y.damping && x.base == y.base &&
         x.teleport == y.teleport && x.seed == y.seed && x.row_ptr == y.row_ptr && x.col == y.col && x.w == y.w &&
         x.vbase == y.vbase && x.vaux == y.vaux && x.push_threshold == y.push_threshold;
}

// Runs the sweep loop from the state already on the device; fills fin.
int run_sweeps(nwgpu_graph* g, const SweepArgs& a, uint32_t launch, uint64_t max_iters, cudaStream_t s, PrState* fin,
               const BinPlan* plan, int mode) {
  if (launch == NWGPU_LAUNCH_GRAPH) {
    if (!g->cg_exec || !same_loop(g, a, plan, mode)) {
      int rc = build_loop_graph(g, a, plan, mode);
      if (rc) return rc;
    }
    const uint64_t max_launches = max_iters / kGraphChunk + 2;
    for (uint64_t launches = 0;; ++launches) {
      if (launches == max_launches)
        return fail(NWGPU_ERR_CUDA, "sweep loop did not finish after %llu graph launches", (unsigned long long)launches);
      CK(cudaGraphLaunch(g->cg_exec, s), "cudaGraphLaunch");
      CK(cudaMemcpyAsync(g->h_st, g->st, sizeof(PrState), cudaMemcpyDeviceToHost, s), "copy state");
      CK(cudaStreamSynchronize(s), "sweep loop");
      if (g->h_st->done) break;
    }
  } else {
    uint64_t launched = 0;
    for (;;) {
      const uint64_t batch = (max_iters - launched) < kGraphChunk ? (max_iters - launched) : kGraphChunk;
      const bool       blk = use_blocked(g, plan, mode);
      const BinnedArgs ba = (plan && !blk) ? make_binned_args(g, *plan, a, mode) : BinnedArgs{};
      const BlockedArgs bk = blk ? make_blocked_args(g->bplan, a, g->n) : BlockedArgs{};
      for (uint64_t b = 0; b < batch; ++b) {
        if (blk) {
          CK(launch_blocked_sweep(bk, g->bplan.sweep_grid, g->bplan.loads, s), "pr_blocked_sweep");
        } else if (plan) {
          CK(launch_binned_sweep(ba, plan->hot, mode, binned_grid(g, *plan, mode), plan->finish_grid, s), "pr_binned_sweep");
        } else {
          CK(launch_pr_sweep(a, g->variant, g->grid, s), "pr_sweep");
          CK(launch_pr_finish(a, g->finish_grid, s), "pr_finish");
        }
      }
      launched += batch;
      CK(cudaMemcpyAsync(g->h_st, g->st, sizeof(PrState), cudaMemcpyDeviceToHost, s), "copy state");
      CK(cudaStreamSynchronize(s), "sweep loop");
      if (g->h_st->done || launched >= max_iters) break;
    }
  }
  *fin = *g->h_st;
  if (fin->fault == kFaultDegrees && use_blocked(g, plan, mode)) return kRetryBinned;
  if (fin->fault) return fail(NWGPU_ERR_CUDA, "a bounded device wait gave up (fault word %u)", fin->fault);
  return NWGPU_OK;
}

nwgpu_pr_options read_options(const nwgpu_pr_options* options) {
  nwgpu_pr_options opt = {};
  if (options) memcpy(&opt, options, options->size && options->size < sizeof(opt) ? options->size : sizeof(opt));
  return opt;
}

// Shared body of nwgpu_pr_run (uniform teleport) and nwgpu_ppr_run (one-hot).
int solve_single(nwgpu_graph* g, const uint32_t* out_degree, float* ranks, float damping, float threshold,
                 uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats, int teleport,
                 uint32_t seed_in) {
  clear_error();
  if (!g) return fail(NWGPU_ERR_INVALID_ARG, "graph is NULL");
  if (g->n && (!out_degree || !ranks)) return fail(NWGPU_ERR_INVALID_ARG, "out_degree / ranks is NULL");
  if (!(damping >= 0.0f && damping <= 1.0f)) return fail(NWGPU_ERR_INVALID_ARG, "damping %g outside [0, 1]", (double)damping);
  if (teleport == kTeleportSeed && seed_in >= g->n)
    return fail(NWGPU_ERR_INVALID_ARG, "seed %u >= n = %llu", seed_in, (unsigned long long)g->n);
  const nwgpu_pr_options opt = read_options(options);
  if (opt.mode != NWGPU_MODE_PARITY) return fail(NWGPU_ERR_UNSUPPORTED, "mode %u is not supported", opt.mode);
  if (opt.launch > NWGPU_LAUNCH_STREAM) return fail(NWGPU_ERR_INVALID_ARG, "launch %u unknown", opt.launch);
  const uint64_t n = g->n;
  if (stats) {
    double*  eb = stats->errors;
    uint64_t ec = stats->errors_cap;
    memset(stats, 0, sizeof(*stats));
    stats->errors = eb;
    stats->errors_cap = ec;
    stats->bytes_per_iter = 4.0 * (double)g->nnz + 4.0 * (double)(n + 1) + 20.0 * (double)n;
  }
  // page_rank.hpp:92-94: N = graph.size(); constants in double, stored as Real.
  const float init = (float)(1.0 / (double)n);
  const float base = (teleport == kTeleportSeed) ? (float)(1.0 - (double)damping)
                                                 : (float)((1.0 - (double)damping) / (double)n);
  if (n == 0) {
    // The reference's sweep reduces over an empty range: error 0.
    const uint64_t its = (max_iters == 0) ? 0 : ((0.0 < (double)threshold) ? 1 : max_iters);
    if (stats) {
      stats->iterations = its;
      stats->converged = its > 0 && 0.0 < (double)threshold;
    }
    return NWGPU_OK;
  }
  cudaStream_t s = opt.stream ? (cudaStream_t)opt.stream : g->stream;
  PhaseTimer   trace(s);
  int          rc = ensure_solve_buffers(g);
  if (rc) return rc;
  *(volatile unsigned int*)g->h_abort = 0u;
  trace.mark("solve buffers");
  if ((rc = load_degrees(g, out_degree, opt.device_ptrs != 0, s))) return rc;
  uint32_t seed = seed_in;
  if (teleport == kTeleportSeed && g->relabelled)
    CK(cudaMemcpy(&seed, g->g.perm + seed_in, sizeof(uint32_t), cudaMemcpyDeviceToHost), "seed id");
  PrState h = {};
  h.max_iters = max_iters;
  h.chunk_end = kGraphChunk;
  h.threshold = (double)threshold;
  h.done = (max_iters == 0) ? 1u : 0u;
  *g->h_st = h;
  CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
  const BinPlan* plan = g->plan.ok ? &g->plan : nullptr;
  if (use_blocked(g, plan, kModePlain)) CK(launch_check_degrees(g->bplan, g->deg, g->st, g->sms, s), "check degrees");
  SweepArgs a = make_sweep_args(g, damping, base, teleport, seed);
  CK(launch_pr_init(a, n, init, g->sms, s), "pr_init");

  trace.mark("degrees + init");
  CK(cudaEventRecord(g->ev0, s), "cudaEventRecord");
  PrState fin{};
  rc = run_sweeps(g, a, opt.launch, max_iters, s, &fin, plan, kModePlain);
  if (rc == kRetryBinned) {
    // out-degrees below the entry counts: the binned sweep, whose FP32 sums follow the reference for any degrees
    g->blocked_off = true;
    *g->h_st = h;
    CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
    CK(launch_pr_init(a, n, init, g->sms, s), "pr_init");
    CK(cudaEventRecord(g->ev0, s), "cudaEventRecord");
    rc = run_sweeps(g, a, opt.launch, max_iters, s, &fin, plan, kModePlain);
    g->blocked_off = false;
  }
  if (rc) return rc;
  CK(cudaEventRecord(g->ev1, s), "cudaEventRecord");
  trace.mark("sweeps");
  if (g->relabelled) {
    float* dst = opt.device_ptrs ? ranks : reinterpret_cast<float*>(g->stage_u32);
    CK(launch_gather_f32(g->rank, g->g.perm, dst, n, g->sms, s), "permute ranks");
    if (!opt.device_ptrs) CK(cudaMemcpyAsync(ranks, dst, n * sizeof(float), cudaMemcpyDeviceToHost, s), "copy ranks");
  } else {
    CK(cudaMemcpyAsync(ranks, g->rank, n * sizeof(float), opt.device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       s),
       "copy ranks");
  }
  CK(cudaStreamSynchronize(s), "copy ranks");
  trace.mark("ranks out");
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->iterations = fin.iter;
    stats->final_error = fin.last_error;
    stats->converged = (int32_t)fin.converged;
    stats->device_ms = ms;
    stats->ms_per_iter = fin.iter ? ms / (double)fin.iter : 0.0;
    stats->gteps = ms > 0 ? (double)g->nnz * (double)fin.iter / (ms * 1e6) : 0.0;
    if (stats->errors && stats->errors_cap) {
      uint64_t m = fin.iter < stats->errors_cap ? fin.iter : stats->errors_cap;
      if (m > g->err_cap) m = g->err_cap;
      if (m) {
        CK(cudaMemcpyAsync(stats->errors, g->err_hist, m * sizeof(double), cudaMemcpyDeviceToHost, s), "copy errors");
        CK(cudaStreamSynchronize(s), "copy errors");
      }
    }
  }
  if (fin.aborted) return fail(NWGPU_ERR_ABORTED, "solve aborted after %llu sweeps", (unsigned long long)fin.iter);
  return NWGPU_OK;
}

}  // namespace nwgpu

namespace nwgpu {
int pr_solve_queue(nwgpu_graph* g, const uint32_t* d_degree, float* d_ranks, float damping, float threshold,
                   uint64_t max_iters, cudaStream_t s, bool* queued) {
  *queued = false;
  if (!g || g->n == 0 || !g->relabelled || !g->plan.ok || max_iters == 0) return NWGPU_OK;
  const uint64_t n = g->n;
  const float    init = (float)(1.0 / (double)n);  // page_rank.hpp:92-94
  const float    base = (float)((1.0 - (double)damping) / (double)n);
  int            rc = ensure_solve_buffers(g);
  if (rc) return rc;
  *(volatile unsigned int*)g->h_abort = 0u;
  if ((rc = load_degrees(g, d_degree, true, s))) return rc;
  PrState h = {};
  h.max_iters = max_iters;
  h.chunk_end = kGraphChunk;
  h.threshold = (double)threshold;
  *g->h_st = h;
  CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
  if (use_blocked(g, &g->plan, kModePlain)) CK(launch_check_degrees(g->bplan, g->deg, g->st, g->sms, s), "check degrees");
  const SweepArgs a = make_sweep_args(g, damping, base, kTeleportUniform, 0u);
  CK(launch_pr_init(a, n, init, g->sms, s), "pr_init");
  if (!g->cg_exec || !same_loop(g, a, &g->plan, kModePlain)) {
    if ((rc = build_loop_graph(g, a, &g->plan, kModePlain))) return rc;
  }
  CK(cudaGraphLaunch(g->cg_exec, s), "cudaGraphLaunch");
  CK(cudaMemcpyAsync(g->h_st, g->st, sizeof(PrState), cudaMemcpyDeviceToHost, s), "copy state");
  CK(launch_gather_f32(g->rank, g->g.perm, d_ranks, n, g->sms, s), "permute ranks");
  *queued = true;
  return NWGPU_OK;
}

int pr_solve_finish(nwgpu_graph* g, float* d_ranks, float damping, float threshold, uint64_t max_iters, cudaStream_t s,
                    nwgpu_pr_stats* stats) {
  PrState fin = *g->h_st;
  if (fin.fault == kFaultDegrees && use_blocked(g, &g->plan, kModePlain)) {
    // out-degrees below the entry counts: solve again with the binned sweep
    const float init = (float)(1.0 / (double)g->n);
    PrState     h = {};
    h.max_iters = max_iters;
    h.chunk_end = kGraphChunk;
    h.threshold = (double)threshold;
    g->blocked_off = true;
    *g->h_st = h;
    CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
    const SweepArgs a = make_sweep_args(g, damping, (float)((1.0 - (double)damping) / (double)g->n), kTeleportUniform, 0u);
    CK(launch_pr_init(a, g->n, init, g->sms, s), "pr_init");
    int rc = run_sweeps(g, a, NWGPU_LAUNCH_GRAPH, max_iters, s, &fin, &g->plan, kModePlain);
    g->blocked_off = false;
    if (rc) return rc;
    CK(launch_gather_f32(g->rank, g->g.perm, d_ranks, g->n, g->sms, s), "permute ranks");
    CK(cudaStreamSynchronize(s), "permute ranks");
  }
  if (fin.fault) return fail(NWGPU_ERR_CUDA, "a bounded device wait gave up (fault word %u)", fin.fault);
  if (!fin.done) {  // more sweeps than one graph launch runs: the loop goes on as nwgpu_pr_run's does
    const SweepArgs a = make_sweep_args(g, damping, (float)((1.0 - (double)damping) / (double)g->n), kTeleportUniform, 0u);
    int             rc = run_sweeps(g, a, NWGPU_LAUNCH_GRAPH, max_iters, s, &fin, &g->plan, kModePlain);
    if (rc) return rc;
    CK(launch_gather_f32(g->rank, g->g.perm, d_ranks, g->n, g->sms, s), "permute ranks");
    CK(cudaStreamSynchronize(s), "permute ranks");
  }
  (void)threshold;
  if (stats) {
    stats->iterations = fin.iter;
    stats->final_error = fin.last_error;
    stats->converged = (int32_t)fin.converged;
  }
  if (fin.aborted) return fail(NWGPU_ERR_ABORTED, "solve aborted after %llu sweeps", (unsigned long long)fin.iter);
  return NWGPU_OK;
}
}  // namespace nwgpu

extern "C" {

int nwgpu_abi_version(void) { return NWGPU_ABI_VERSION; }

int nwgpu_selftest_bounded_wait(uint32_t polls, uint32_t* gave_up, double* ms) {
  clear_error();
  if (!gave_up || !ms) return fail(NWGPU_ERR_INVALID_ARG, "NULL argument");
  if (polls == 0 || polls > (1u << 20)) return fail(NWGPU_ERR_INVALID_ARG, "polls = %u outside [1, 2^20]", polls);
  int dev, sms;
  int rc = check_device(&dev, &sms);
  if (rc) return rc;
  unsigned int flag = 0;
  float        t = 0.f;
  CK(run_wait_selftest(polls, &flag, &t), "bounded-wait self-test");
  *gave_up = flag;
  *ms = t;
  return NWGPU_OK;
}

int nwgpu_last_error(char* buf, size_t len) {
  const std::string& e = last_error_text();
  if (buf && len) {
    size_t m = e.size() < len - 1 ? e.size() : len - 1;
    memcpy(buf, e.data(), m);
    buf[m] = '\0';
  }
  return (int)e.size();
}

namespace {
int upload_whole(nwgpu_graph* g, const uint32_t* row_ptr, const uint32_t* col, const float* weights, uint64_t n,
                 uint64_t nnz, uint32_t flags, cudaMemcpyKind kind, PhaseTimer& trace);
int finish_create(nwgpu_graph* g, const float* weights, uint32_t flags, nwgpu_graph** out, PhaseTimer& trace);
}  // namespace

int nwgpu_graph_create(const uint32_t* row_ptr, const uint32_t* col, const float* weights, uint64_t n, uint64_t nnz,
                       uint32_t flags, nwgpu_graph** out) {
  clear_error();
  if (!out) return fail(NWGPU_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!row_ptr) return fail(NWGPU_ERR_INVALID_ARG, "row_ptr is NULL");
  if (nnz && !col) return fail(NWGPU_ERR_INVALID_ARG, "col is NULL with nnz > 0");
  if (n >= 0xFFFFFFF0ull) return fail(NWGPU_ERR_INVALID_ARG, "n = %llu does not fit uint32 vertex ids", (unsigned long long)n);
  if (nnz > kMaxEntries)
    return fail(NWGPU_ERR_INVALID_ARG, "nnz = %llu is above the limit of %llu entries (uint32 row pointers and entry indices)",
                (unsigned long long)nnz, (unsigned long long)kMaxEntries);
  int dev, sms;
  int rc = check_device(&dev, &sms);
  if (rc) return rc;

  nwgpu_graph* g = new (std::nothrow) nwgpu_graph();
  if (!g) return fail(NWGPU_ERR_OUT_OF_MEMORY, "host allocation failed");
  g->device = dev;
  g->sms = sms;
  g->n = n;
  g->nnz = nnz;
  auto bail = [&](int code) {
    delete g;
    return code;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamCreate"));
  const cudaMemcpyKind kind = (flags & NWGPU_GRAPH_DEVICE_PTRS) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  PhaseTimer           trace(g->stream);
  const long           chunk_env = env_int("NWGPU_UPLOAD_CHUNK_ENTRIES", 0);
  const uint64_t       chunk = chunk_env > 0 ? (uint64_t)chunk_env : kUploadChunkEntries;
  if (kind == cudaMemcpyHostToDevice && !weights && !(flags & NWGPU_GRAPH_NO_RELABEL) && n > 1 && nnz > chunk) {
    rc = upload_streamed(g, row_ptr, col, n, nnz, chunk, trace);
    if (rc) return bail(rc);
  } else {
    rc = upload_whole(g, row_ptr, col, weights, n, nnz, flags, kind, trace);
    if (rc) return bail(rc);
  }
  rc = finish_create(g, weights, flags, out, trace);
  return rc ? bail(rc) : NWGPU_OK;
}

namespace {
// The CSR uploaded (or copied from device memory) in one piece, validated,
// then relabelled unless NWGPU_GRAPH_NO_RELABEL.
int upload_whole(nwgpu_graph* g, const uint32_t* row_ptr, const uint32_t* col, const float* weights, uint64_t n,
                 uint64_t nnz, uint32_t flags, cudaMemcpyKind kind, PhaseTimer& trace) {
  const int   sms = g->sms;
  cudaError_t e;
  auto        bail = [](int code) { return code; };
  // Upload into padded buffers.
  Relabelled in;
  auto       free_in = [&]() {
    pool_free(in.row_ptr, g->stream);
    pool_free(in.col, g->stream);
    pool_free(in.w, g->stream);
  };
  if ((e = dalloc(g, &in.row_ptr, n + 1)) != cudaSuccess || (e = dalloc(g, &in.col, nnz)) != cudaSuccess) {
    free_in();
    return bail(cuda_fail(e, "cudaMalloc(CSR)"));
  }
  if ((e = cudaMemcpyAsync(in.row_ptr, row_ptr, (n + 1) * sizeof(uint32_t), kind, g->stream)) != cudaSuccess ||
      (nnz && (e = cudaMemcpyAsync(in.col, col, nnz * sizeof(uint32_t), kind, g->stream)) != cudaSuccess)) {
    free_in();
    return bail(cuda_fail(e, "upload CSR"));
  }
  if (weights) {
    if ((e = dalloc(g, &in.w, nnz)) != cudaSuccess ||
        (nnz && (e = cudaMemcpyAsync(in.w, weights, nnz * sizeof(float), kind, g->stream)) != cudaSuccess)) {
      free_in();
      return bail(cuda_fail(e, "upload weights"));
    }
  }
  trace.mark("upload");
  // Validate on the device before any kernel indexes with these arrays.
  unsigned int* d_err = nullptr;
  unsigned int  h_err = 0;
  if ((e = pool_alloc_n(&d_err, 1, g->stream)) != cudaSuccess) {
    free_in();
    return bail(cuda_fail(e, "cudaMalloc(err)"));
  }
  cudaMemsetAsync(d_err, 0, sizeof(unsigned int), g->stream);
  e = validate_csr(in.row_ptr, in.col, n, nnz, d_err, sms, g->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  pool_free(d_err, g->stream);
  if (e != cudaSuccess) {
    free_in();
    return bail(cuda_fail(e, "validate"));
  }
  if (h_err) {
    free_in();
    char why[160];
    return bail(fail(NWGPU_ERR_INVALID_GRAPH, "invalid CSR:%s", csr_error_text(h_err, why, sizeof(why))));
  }
  trace.mark("validate");
  if (!(flags & NWGPU_GRAPH_NO_RELABEL) && n > 1) {
    e = build_relabelled(in.row_ptr, in.col, in.w, n, nnz, sms, &g->g, g->stream);
    free_in();
    if (e != cudaSuccess) return bail(cuda_fail(e, "relabel"));
    g->relabelled = true;
  } else {
    g->g.row_ptr = in.row_ptr;
    g->g.col = in.col;
    g->g.w = in.w;
  }
  trace.mark("relabel");
  return NWGPU_OK;
}

// Launch set-up of a handle whose CSR is in place: tiling, the bin plan, the
// tuner, the out-row CSR.
int finish_create(nwgpu_graph* g, const float* weights, uint32_t flags, nwgpu_graph** out, PhaseTimer& trace) {
  const uint64_t n = g->n, nnz = g->nnz;
  const int      sms = g->sms;
  cudaError_t    e;
  int            rc;
  auto           bail = [](int code) { return code; };
  // Merge-path sweep (graphs kept in input order, or NWGPU_SWEEP naming a
  // merge-path variant): 256-thread CTAs by default. NWGPU_SWEEP
  // (base|hot|hot512|hot1024x8), NWGPU_IPT, NWGPU_HOT_IDS, NWGPU_CTAS_PER_SM and
  // NWGPU_CARVEOUT override for tuning. Relabelled graphs use the degree-binned
  // sweep (set up below) unless NWGPU_SWEEP names a merge-path variant.
  SweepVariant v{256, kDefaultIpt, false};
  const char*  which = getenv("NWGPU_SWEEP");
  const bool   want_hot = which && strncmp(which, "hot", 3) == 0;
  if (want_hot) {
    v = SweepVariant{1024, 4, true};
    if (which && !strcmp(which, "hot512")) v = SweepVariant{512, 8, true};
    if (which && !strcmp(which, "hot1024x8")) v = SweepVariant{1024, 8, true};
  } else {
    v.ipt = env_int("NWGPU_IPT", kDefaultIpt);
    if (!sweep_variant_supported(v)) v.ipt = kDefaultIpt;
  }
  g->variant = v;
  const long hot_env = env_int("NWGPU_HOT_IDS", -1);
  if (v.hot_smem) {
    uint32_t cap = sweep_hot_capacity(v);
    if (hot_env >= 0 && (uint32_t)hot_env < cap) cap = (uint32_t)hot_env;
    g->hot_ids = (uint32_t)(n < cap ? n : cap) & ~3u;
  } else {
    g->hot_ids = hot_env >= 0 ? (uint32_t)hot_env : (g->relabelled ? kDefaultHotIds : 0xffffffffu);
  }
  const int carve = env_int("NWGPU_CARVEOUT", -1);
  if (carve >= 0) set_sweep_carveout(v, carve);
  if ((e = build_tiling(g->g.row_ptr, n, nnz, v.tile_items(), &g->tiling, g->stream)) != cudaSuccess)
    return bail(cuda_fail(e, "build_tiling"));
  int per_sm = sweep_blocks_per_sm(v, g->hot_ids);
  const int cap = env_int("NWGPU_CTAS_PER_SM", 0);
  if (cap > 0 && cap < per_sm) per_sm = cap;
  const uint64_t want = (uint64_t)sms * per_sm;
  g->grid = (int)(want < g->tiling.num_tiles ? want : (g->tiling.num_tiles ? g->tiling.num_tiles : 1));
  g->finish_grid = finish_grid_for(g->tiling.num_tiles);
  if ((e = cudaStreamSynchronize(g->stream)) != cudaSuccess) return bail(cuda_fail(e, "graph create"));
  trace.mark("tiling");
  const bool want_binned =
      which ? (!strcmp(which, "binned") || !strcmp(which, "binned_hot") || !strcmp(which, "blocked")) : true;
  const char* tune_env = getenv("NWGPU_AUTOTUNE");
  const bool  tune_all = ((flags & NWGPU_GRAPH_AUTOTUNE) || (tune_env && !strcmp(tune_env, "1"))) && !which &&
                        !getenv("NWGPU_HOT_IDS") && !getenv("NWGPU_HOT_L1_IDS") && !getenv("NWGPU_LONG_ROW") &&
                        !getenv("NWGPU_CHUNK_ENTRIES") && !getenv("NWGPU_BIN0_ROWS");
  if (g->relabelled && want_binned) {
    // NWGPU_SWEEP=binned keeps the hubs in L1 only (256-thread CTAs); NWGPU_LONG_ROW and
    // NWGPU_CHUNK_ENTRIES set the long-row cut-offs, NWGPU_BIN0_ROWS the bin-0 rows per warp
    // (the tuner's choice otherwise: the cached one for this graph's signature, if any, so the
    // plan is built once)
    uint32_t long_row = (uint32_t)env_int("NWGPU_LONG_ROW", (int)kLongRow);
    uint32_t chunk = (uint32_t)env_int("NWGPU_CHUNK_ENTRIES", (int)kChunk);
    uint32_t bin0_rows = (uint32_t)env_int("NWGPU_BIN0_ROWS", (int)kBin0Rows);
    if (tune_all && (rc = cached_cutoffs(g, &long_row, &chunk, &bin0_rows))) return bail(rc);
    rc = build_bin_plan(g, g->g.row_ptr, n, !which || strcmp(which, "binned") != 0, &g->plan, long_row, chunk,
                        bin0_rows);
    if (rc) return bail(rc);
  }
  trace.mark("bins");
  // The destination-blocked sweep of plain solves (NWGPU_SWEEP=blocked): relabelled unweighted graphs
  // (NWGPU_BLOCK_PIECE_ENTRIES sets the largest work item).
  if (g->relabelled && !weights && !(flags & kGraphNoBlockedPlan) && which && !strcmp(which, "blocked")) {
    const long piece = env_int("NWGPU_BLOCK_PIECE_ENTRIES", 0);
    const char* fmt = getenv("NWGPU_BLOCK_FORMAT");  // "wide": 6-byte entries instead of the packed 4-byte words
    if ((e = build_block_plan(g->g.row_ptr, g->g.col, n, nnz, n, sms, piece > 0 ? (uint64_t)piece : 0,
                              !(fmt && !strcmp(fmt, "wide")), &g->bplan, g->stream)) != cudaSuccess)
      return bail(cuda_fail(e, "blocked entry order"));
    g->device_bytes += g->bplan.bytes;
    const int loads = env_int("NWGPU_BLOCK_LOADS", 8);  // entries in flight per thread: 4, 8 or 16
    g->bplan.loads = loads <= 4 ? 4 : (loads >= 16 ? 16 : 8);
    trace.mark("blocked");
  }
  {
    // explicit launch settings in the environment take precedence over tuning
    const char* tune = getenv("NWGPU_AUTOTUNE");
    const bool  shapes_only = (flags & kGraphTuneShapes) && !(flags & NWGPU_GRAPH_AUTOTUNE);
    const bool  want_tune = (flags & (NWGPU_GRAPH_AUTOTUNE | kGraphTuneShapes)) || (tune && !strcmp(tune, "1"));
    if (want_tune && g->bplan.ok && !getenv("NWGPU_BLOCK_LOADS") && !getenv("NWGPU_BLOCK_PIECE_ENTRIES")) {
      rc = autotune_blocked(g);  // plain solves run the blocked sweep
      if (rc) return bail(rc);
      trace.mark("autotune");
    } else if (want_tune && g->plan.ok && !g->bplan.ok && !which && !getenv("NWGPU_HOT_IDS") &&
               !getenv("NWGPU_HOT_L1_IDS") && !getenv("NWGPU_LONG_ROW") && !getenv("NWGPU_CHUNK_ENTRIES") &&
               !getenv("NWGPU_BIN0_ROWS")) {
      rc = autotune_binned(g, shapes_only);
      if (rc) return bail(rc);
      trace.mark("autotune");
    }
  }
  if ((flags & NWGPU_GRAPH_TRANSPOSE) && weights && g->plan.ok) {
    rc = ensure_wpr(g);
    if (rc) return bail(rc);
    trace.mark("out-row CSR");
  }
  *out = g;
  return NWGPU_OK;
}
}  // namespace

int nwgpu_graph_destroy(nwgpu_graph* g) {
  clear_error();
  if (!g) return NWGPU_OK;
  if (g->stream) cudaStreamSynchronize(g->stream);
  PhaseTimer trace(nullptr);
  delete g;
  trace.mark("destroy");
  return NWGPU_OK;
}

int nwgpu_graph_get_info(const nwgpu_graph* g, nwgpu_graph_info* info) {
  if (!g || !info) return fail(NWGPU_ERR_INVALID_ARG, "NULL argument");
  memset(info, 0, sizeof(*info));
  info->n = g->n;
  info->nnz = g->nnz;
  info->num_tiles = g->tiling.num_tiles;
  info->tile_items = g->tiling.tile_items;
  info->grid = (uint32_t)g->grid;
  info->device_bytes = g->device_bytes;
  info->device = g->device;
  info->has_weights = g->g.w != nullptr;
  info->has_transpose = g->wpr.ready ? 1 : 0;
  info->binned = g->plan.ok ? 1 : 0;
  if (g->plan.ok) {
    info->sweep_threads = g->plan.hot ? kBinnedHotThreads : kBinnedThreads;
    info->sweep_grid = (uint32_t)g->plan.sweep_grid;
    info->hub_smem_ids = g->plan.bin.smem_ids;
    info->hub_l1_ids = g->plan.bin.l1_ids;
    info->long_row_entries = g->plan.bin.long_row;
    info->chunk_entries = g->plan.bin.chunk;
    info->bin0_rows_per_warp = g->plan.bin.bin0_rows;
  } else {
    info->sweep_threads = (uint32_t)g->variant.threads;
    info->sweep_grid = (uint32_t)g->grid;
  }
  info->tuned = g->tuned;
  info->tuned_us_per_sweep = g->tune_us;
  info->blocked = g->bplan.ok ? 1 : 0;
  info->block_count = g->bplan.num_blocks;
  info->block_items = g->bplan.num_items;
  info->block_loads = g->bplan.ok ? (uint32_t)g->bplan.loads : 0u;
  info->block_piece_entries = g->bplan.ok ? g->bplan.piece_entries : 0ull;
  return NWGPU_OK;
}

int nwgpu_abort(nwgpu_graph* g) {
  if (!g) return fail(NWGPU_ERR_INVALID_ARG, "NULL graph");
  if (g->h_abort) *(volatile unsigned int*)g->h_abort = 1u;
  return NWGPU_OK;
}

int nwgpu_pr_run(nwgpu_graph* g, const uint32_t* out_degree, float* ranks, float damping, float threshold,
                 uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats) {
  return solve_single(g, out_degree, ranks, damping, threshold, max_iters, options, stats, kTeleportUniform, 0u);
}

int nwgpu_pr_residual_run(nwgpu_graph* g, const uint32_t* out_degree, float* ranks, float damping, float threshold,
                          uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats) {
  clear_error();
  if (!g) return fail(NWGPU_ERR_INVALID_ARG, "graph is NULL");
  if (g->n && (!out_degree || !ranks)) return fail(NWGPU_ERR_INVALID_ARG, "out_degree / ranks is NULL");
  if (!(damping >= 0.0f && damping <= 1.0f)) return fail(NWGPU_ERR_INVALID_ARG, "damping %g outside [0, 1]", (double)damping);
  const nwgpu_pr_options opt = read_options(options);
  if (opt.launch > NWGPU_LAUNCH_STREAM) return fail(NWGPU_ERR_INVALID_ARG, "launch %u unknown", opt.launch);
  const uint64_t n = g->n;
  if (stats) {
    double*  eb = stats->errors;
    uint64_t ec = stats->errors_cap;
    memset(stats, 0, sizeof(*stats));
    stats->errors = eb;
    stats->errors_cap = ec;
    stats->bytes_per_iter = 4.0 * (double)g->nnz + 4.0 * (double)(n + 1) + 20.0 * (double)n;
  }
  if (n == 0) {  // no vertex pushes: the first iteration ends the loop
    if (stats) stats->iterations = max_iters ? 1 : 0;
    if (stats) stats->converged = max_iters ? 1 : 0;
    return NWGPU_OK;
  }
  if (!g->plan.ok) return fail(NWGPU_ERR_UNSUPPORTED, "the residual-push solve runs on the binned sweep: relabel the graph");
  cudaStream_t s = opt.stream ? (cudaStream_t)opt.stream : g->stream;
  int          rc = ensure_solve_buffers(g);
  if (rc) return rc;
  *(volatile unsigned int*)g->h_abort = 0u;
  if ((rc = load_degrees(g, out_degree, opt.device_ptrs != 0, s))) return rc;
  // page_rank_v13's first iteration, first phase: every residual is (float)(1 - d)
  const float r0 = (float)(1.0 - (double)damping);
  PrState     h = {};
  *g->h_st = h;
  CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
  CK(launch_residual_init(g->rank, g->contrib[0], g->deg, n, r0, damping, max_iters > 0 && r0 > threshold,
                          &g->st->pending, g->sms, s),
     "residual init");
  CK(cudaMemcpyAsync(g->h_st, g->st, sizeof(PrState), cudaMemcpyDeviceToHost, s), "copy state");
  CK(cudaStreamSynchronize(s), "residual init");
  const uint64_t first = g->h_st->pending;  // vertices that pushed in the first iteration
  CK(cudaEventRecord(g->ev0, s), "cudaEventRecord");
  PrState fin{};
  if (max_iters > 1 && first > 0) {
    // each sweep: the second phase of one iteration and the first of the next;
    // its "error" is the number of vertices that pushed, and no push ends the loop
    h = {};
    h.max_iters = max_iters - 1;
    h.chunk_end = kGraphChunk;
    h.threshold = 0.5;
    *g->h_st = h;
    CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
    SweepArgs a = make_sweep_args(g, damping, 0.f, kTeleportUniform, 0u);
    a.push_threshold = threshold;
    if ((rc = run_sweeps(g, a, opt.launch, max_iters - 1, s, &fin, &g->plan, kModeResidual))) return rc;
  }
  CK(cudaEventRecord(g->ev1, s), "cudaEventRecord");
  float* dst = opt.device_ptrs ? ranks : reinterpret_cast<float*>(g->stage_u32);
  CK(launch_gather_f32(g->rank, g->g.perm, dst, n, g->sms, s), "permute ranks");
  if (!opt.device_ptrs) CK(cudaMemcpyAsync(ranks, dst, n * sizeof(float), cudaMemcpyDeviceToHost, s), "copy ranks");
  CK(cudaStreamSynchronize(s), "copy ranks");
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    const uint64_t its = max_iters == 0 ? 0 : 1 + fin.iter;
    stats->iterations = its;
    stats->final_error = fin.iter ? fin.last_error : (double)first;
    stats->converged = max_iters > 0 && (fin.iter ? fin.converged != 0 : first == 0);
    stats->device_ms = ms;
    stats->ms_per_iter = fin.iter ? ms / (double)fin.iter : 0.0;
    stats->gteps = ms > 0 ? (double)g->nnz * (double)fin.iter / (ms * 1e6) : 0.0;
    if (stats->errors && stats->errors_cap && its) {
      stats->errors[0] = (double)first;
      uint64_t m = fin.iter < stats->errors_cap - 1 ? fin.iter : stats->errors_cap - 1;
      if (m > g->err_cap) m = g->err_cap;
      if (m) {
        CK(cudaMemcpyAsync(stats->errors + 1, g->err_hist, m * sizeof(double), cudaMemcpyDeviceToHost, s), "copy errors");
        CK(cudaStreamSynchronize(s), "copy errors");
      }
    }
  }
  if (fin.aborted) return fail(NWGPU_ERR_ABORTED, "solve aborted after %llu sweeps", (unsigned long long)fin.iter);
  return NWGPU_OK;
}

int nwgpu_ppr_run(nwgpu_graph* g, const uint32_t* out_degree, uint32_t seed, float* ranks, float damping,
                  float threshold, uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats) {
  return solve_single(g, out_degree, ranks, damping, threshold, max_iters, options, stats, kTeleportSeed, seed);
}

}  // extern "C"
