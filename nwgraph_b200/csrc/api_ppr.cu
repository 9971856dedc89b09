// C ABI: batched personalised PageRank (nwgpu_ppr_batched, include/nwgpu.h).
// No counterpart in the reference; the single-vector personalised solve is
// nwgpu_ppr_run in api.cu, and the looped baseline calls it k times.
#include "handle.h"

namespace nwgpu {

void PprBuffers::release(cudaStream_t s) {
  if (cg_exec) cudaGraphExecDestroy(cg_exec);
  if (cg) cudaGraphDestroy(cg);
  cg_exec = nullptr;
  cg = nullptr;
  void* ptrs[] = {tiling.tile_row, tiling.tile_nnz, rank, contrib[0], contrib[1], out, cpart, epart, res_part,
                  spans, seeds, seeds_in, col_done, col_conv, col_iters, col_err, st, vbase, slot_map, slot_orig};
  for (void* p : ptrs) pool_free(p, s);
  if (h_st) {
    cudaStreamSynchronize(s);  // no copy may still target the block when it is reused
    host_block_put(h_st);
  }
  *this = PprBuffers();
}

static int ensure_ppr(nwgpu_graph* g, int K) {
  PprBuffers& b = g->ppr;
  if (b.K == K) return NWGPU_OK;
  b.release(g->stream);
  const uint64_t n = g->n, nk = g->n * (uint64_t)K;
  CK(build_tiling(g->g.row_ptr, n, g->nnz, (uint32_t)kPprTileItems, &b.tiling, g->stream), "ppr tiling");
  const uint64_t T = b.tiling.num_tiles;
  b.sweep_grid = ppr_sweep_grid(K, g->sms);
  b.finish_grid = g->sms * 4;
  CK(dalloc(g, &b.rank, nk), "cudaMalloc(ppr rank)");
  CK(dalloc(g, &b.contrib[0], nk), "cudaMalloc(ppr contrib)");
  CK(dalloc(g, &b.contrib[1], nk), "cudaMalloc(ppr contrib)");
  CK(dalloc(g, &b.out, nk), "cudaMalloc(ppr out)");
  CK(dalloc(g, &b.cpart, (T + 1) * K), "cudaMalloc(ppr cpart)");
  CK(dalloc(g, &b.epart, (T + 1) * K), "cudaMalloc(ppr epart)");
  CK(dalloc(g, &b.res_part, (uint64_t)(b.sweep_grid + b.finish_grid) * K), "cudaMalloc(ppr res)");
  CK(dalloc(g, &b.seeds, (uint64_t)K), "cudaMalloc(seeds)");
  CK(dalloc(g, &b.seeds_in, (uint64_t)K), "cudaMalloc(seeds)");
  CK(dalloc(g, &b.col_done, (uint64_t)K), "cudaMalloc(col flags)");
  CK(dalloc(g, &b.col_conv, (uint64_t)K), "cudaMalloc(col flags)");
  CK(dalloc(g, &b.col_iters, (uint64_t)K), "cudaMalloc(col iters)");
  CK(dalloc(g, &b.col_err, (uint64_t)K), "cudaMalloc(col err)");
  CK(dalloc(g, &b.st, 1), "cudaMalloc(ppr state)");
  CK(dalloc(g, &b.slot_map, (uint64_t)K), "cudaMalloc(ppr slots)");
  CK(dalloc(g, &b.slot_orig, (uint64_t)K), "cudaMalloc(ppr slots)");
  // rows crossing warp tiles, once per graph (counted in the state's ticket word, reset below)
  CK(dalloc(g, &b.spans, T + 1), "cudaMalloc(ppr spans)");
  {
    unsigned int* cnt = &b.st->ticket;
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned int), g->stream), "ppr spans");
    CK(launch_ppr_spans(g->g.row_ptr, b.tiling.tile_row, b.tiling.tile_nnz, b.tiling.num_tiles, (uint32_t)kPprTileItems,
                        b.spans, cnt, g->sms, g->stream),
       "ppr spans");
    unsigned int h_cnt = 0;
    CK(cudaMemcpyAsync(&h_cnt, cnt, sizeof(h_cnt), cudaMemcpyDeviceToHost, g->stream), "ppr spans");
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned int), g->stream), "ppr spans");
    CK(cudaStreamSynchronize(g->stream), "ppr spans");
    b.num_spans = h_cnt;
  }
  static_assert(sizeof(PprState) <= kHostBlock, "state mirror fits a host block");
  CK(host_block_get((void**)&b.h_st), "cudaHostAlloc(ppr state)");
  CK(cudaStreamSynchronize(g->stream), "ppr buffers");
  b.K = K;
  return NWGPU_OK;
}

int ppr_loop(nwgpu_graph* g, const PprArgs& a, int K, uint32_t k, float* ranks_nxk, float damping, uint64_t max_iters,
             const nwgpu_pr_options& opt, nwgpu_ppr_stats* stats, cudaStream_t s);

static PprArgs make_ppr_args(nwgpu_graph* g, float damping) {
  PprBuffers& b = g->ppr;
  PprArgs     a = {};
  a.row_ptr = g->g.row_ptr;
  a.col = g->g.col;
  a.tile_row = b.tiling.tile_row;
  a.tile_nnz = b.tiling.tile_nnz;
  a.num_tiles = b.tiling.num_tiles;
  a.tile_items = (uint32_t)kPprTileItems;
  a.deg = g->deg;
  a.rank = b.rank;
  a.contrib0 = b.contrib[0];
  a.contrib1 = b.contrib[1];
  a.cpart = b.cpart;
  a.epart = b.epart;
  a.res_part = b.res_part;
  a.epi_grid = (uint32_t)b.finish_grid;
  a.n = g->n;
  a.K = (uint32_t)b.K;
  a.spans = b.spans;
  a.num_spans = b.num_spans;

  a.seeds = b.seeds;
  a.col_done = b.col_done;
  a.col_conv = b.col_conv;
  a.col_iters = b.col_iters;
  a.col_err = b.col_err;
  a.st = b.st;
  a.abort_word = g->d_abort;
  a.damping = damping;
  a.one_minus_d = (float)(1.0 - (double)damping);
  return a;
}

}  // namespace nwgpu

using namespace nwgpu;

extern "C" int nwgpu_ppr_batched(nwgpu_graph* g, const uint32_t* out_degree, const uint32_t* seeds, uint32_t k,
                                 float* ranks_nxk, float damping, float threshold, uint64_t max_iters,
                                 const nwgpu_pr_options* options, nwgpu_ppr_stats* stats) {
  clear_error();
  if (!g) return fail(NWGPU_ERR_INVALID_ARG, "graph is NULL");
  if (k == 0 || k > 128) return fail(NWGPU_ERR_INVALID_ARG, "k = %u outside [1, 128]", k);
  if (!seeds || (g->n && (!out_degree || !ranks_nxk))) return fail(NWGPU_ERR_INVALID_ARG, "NULL array argument");
  if (!(damping >= 0.0f && damping <= 1.0f)) return fail(NWGPU_ERR_INVALID_ARG, "damping %g outside [0, 1]", (double)damping);
  nwgpu_pr_options opt = {};
  if (options) memcpy(&opt, options, options->size && options->size < sizeof(opt) ? options->size : sizeof(opt));
  if (opt.launch > NWGPU_LAUNCH_STREAM) return fail(NWGPU_ERR_INVALID_ARG, "launch %u unknown", opt.launch);
  uint32_t h_seeds[128];
  if (opt.device_ptrs) {
    CK(cudaMemcpy(h_seeds, seeds, k * sizeof(uint32_t), cudaMemcpyDeviceToHost), "copy seeds");
  } else {
    memcpy(h_seeds, seeds, k * sizeof(uint32_t));
  }
  for (uint32_t c = 0; c < k; ++c)
    if (h_seeds[c] >= g->n) return fail(NWGPU_ERR_INVALID_ARG, "seeds[%u] = %u >= n", c, h_seeds[c]);
  const int      K = ppr_padded_k(k);
  const uint64_t n = g->n;
  if (stats) {
    uint32_t* ci = stats->col_iterations;
    double*   ce = stats->col_errors;
    int32_t*  cc = stats->col_converged;
    memset(stats, 0, sizeof(*stats));
    stats->col_iterations = ci;
    stats->col_errors = ce;
    stats->col_converged = cc;
    stats->bytes_per_iter = 4.0 * (double)g->nnz + 4.0 * (double)(n + 1) + 4.0 * (double)n + 16.0 * k * (double)n;
  }
  int rc = ensure_solve_buffers(g);
  if (rc) return rc;
  if ((rc = ensure_ppr(g, K))) return rc;
  PprBuffers&  b = g->ppr;
  cudaStream_t s = opt.stream ? (cudaStream_t)opt.stream : g->stream;
  *(volatile unsigned int*)g->h_abort = 0u;
  if ((rc = load_degrees(g, out_degree, opt.device_ptrs != 0, s))) return rc;
  PprArgs a = make_ppr_args(g, damping);
  CK(cudaMemcpyAsync(b.seeds_in, h_seeds, k * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "copy seeds");
  CK(launch_ppr_seeds(b.seeds_in, k, K, g->relabelled ? g->g.perm : nullptr, a, s), "ppr seeds");
  PprState h = {};
  h.max_iters = max_iters;
  h.chunk_end = kGraphChunk;
  h.threshold = (double)threshold;
  h.done = (max_iters == 0) ? 1u : 0u;
  h.narrow_at = K > 32 ? (unsigned int)(K / 2) : 0u;
  *b.h_st = h;
  CK(cudaMemcpyAsync(b.st, b.h_st, sizeof(PprState), cudaMemcpyHostToDevice, s), "copy ppr state");
  CK(launch_ppr_init(a, K, n, g->sms, s), "ppr init");
  return ppr_loop(g, a, K, k, ranks_nxk, damping, max_iters, opt, stats, s);
}

namespace nwgpu {
// The batched sweep loop from the state on the device, then the output and
// the per-column stats (both batched entry points).
//
// Narrowing (state narrow_at > 0): once at most narrow_at columns still run,
// the device loop stops; every column's current ranks go to the output, the
// running columns move into an n x K/2 layout (K' = 64 or 32), and the solve
// goes on with the narrower kernels, launched from the host a few sweeps at a
// time. The gather sums each column in the same order at every K, so the
// result is the one the wide layout would give, at a fraction of the gather
// traffic in the sweeps where most columns have stopped.
int ppr_loop(nwgpu_graph* g, const PprArgs& a0, int K0, uint32_t k, float* ranks_nxk, float damping, uint64_t max_iters,
             const nwgpu_pr_options& opt, nwgpu_ppr_stats* stats, cudaStream_t s) {
  PprBuffers&     b = g->ppr;
  const uint64_t  n = g->n;
  const int       mode = ppr_mode(a0);
  const uint32_t* perm = g->relabelled ? g->g.perm : nullptr;
  float*          dst = opt.device_ptrs ? ranks_nxk : b.out;
  PprArgs         a = a0;
  int             K = K0;
  bool            narrowed_any = false;
  // per slot: the caller's column it holds (>= k: padding); per caller's column: its stats
  uint32_t orig[128], h_iters[128] = {}, h_conv[128] = {};
  double   h_err[128] = {};
  for (int j = 0; j < K0; ++j) orig[j] = (uint32_t)j < k ? (uint32_t)j : 0xffffffffu;
  auto pull_stats = [&](uint32_t* done_out) -> int {
    uint32_t it[128], cv[128], dn[128];
    double   er[128];
    CK(cudaMemcpyAsync(it, a.col_iters, K * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy col iters");
    CK(cudaMemcpyAsync(cv, a.col_conv, K * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy col flags");
    CK(cudaMemcpyAsync(er, a.col_err, K * sizeof(double), cudaMemcpyDeviceToHost, s), "copy col err");
    CK(cudaMemcpyAsync(dn, a.col_done, K * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy col flags");
    CK(cudaStreamSynchronize(s), "copy col stats");
    for (int j = 0; j < K; ++j) {
      if (orig[j] < k) {
        h_iters[orig[j]] = it[j];
        h_conv[orig[j]] = cv[j];
        h_err[orig[j]] = er[j];
      }
      if (done_out) done_out[j] = dn[j];
    }
    return NWGPU_OK;
  };
  CK(cudaEventRecord(g->ev0, s), "cudaEventRecord");
  if (opt.launch == NWGPU_LAUNCH_GRAPH) {
    if (!b.cg_exec || b.cg_damping != damping || b.cg_mode != mode) {
      if (b.cg_exec) cudaGraphExecDestroy(b.cg_exec);
      if (b.cg) cudaGraphDestroy(b.cg);
      b.cg_exec = nullptr;
      CK(cudaGraphCreate(&b.cg, 0), "cudaGraphCreate");
      CK(build_ppr_graph(b.cg, a, K, b.sweep_grid, b.st, &b.cg_exec), "ppr graph");
      b.cg_damping = damping;
      b.cg_mode = mode;
    }
    const uint64_t max_launches = max_iters / kGraphChunk + 2;
    for (uint64_t l = 0;; ++l) {
      if (l == max_launches) return fail(NWGPU_ERR_CUDA, "ppr sweep loop did not finish");
      CK(cudaGraphLaunch(b.cg_exec, s), "cudaGraphLaunch");
      CK(cudaMemcpyAsync(b.h_st, b.st, sizeof(PprState), cudaMemcpyDeviceToHost, s), "copy ppr state");
      CK(cudaStreamSynchronize(s), "ppr sweep loop");
      if (b.h_st->done) break;
    }
  } else {
    uint64_t launched = 0;
    for (;;) {
      const uint64_t batch = (max_iters - launched) < kGraphChunk ? (max_iters - launched) : kGraphChunk;
      for (uint64_t i = 0; i < batch; ++i) CK(launch_ppr_sweep(a, K, b.sweep_grid, s), "ppr sweep");
      launched += batch;
      CK(cudaMemcpyAsync(b.h_st, b.st, sizeof(PprState), cudaMemcpyDeviceToHost, s), "copy ppr state");
      CK(cudaStreamSynchronize(s), "ppr sweep loop");
      if (b.h_st->done || launched >= max_iters) break;
    }
  }
  while (b.h_st->narrowed) {
    // the columns' current ranks to the output: the stopped ones are final
    uint32_t done[128], map[128], orig2[128];
    int      rc = pull_stats(done);
    if (rc) return rc;
    CK(cudaMemcpyAsync(b.slot_orig, orig, K * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "copy slots");
    CK(launch_ppr_output_slots(a.rank, perm, n, K, b.slot_orig, k, dst, g->sms, s), "ppr output");
    uint32_t nact = 0;
    for (int j = 0; j < K; ++j)
      if (!done[j]) map[nact++] = (uint32_t)j;
    const int K2 = ppr_padded_k(nact ? nact : 1);
    if (K2 >= K) return fail(NWGPU_ERR_CUDA, "narrowing found %u running columns of %d", nact, K);
    for (int j = 0; j < K2; ++j) orig2[j] = (uint32_t)j < nact ? orig[map[j]] : 0xffffffffu;
    CK(cudaMemcpyAsync(b.slot_map, map, nact * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "copy slots");
    // ranks through the idle contribution buffer, then the current contributions into it
    const uint64_t it = b.h_st->iter;
    float*         cur = (it & 1ull) ? a.contrib1 : a.contrib0;  // the next sweep's input
    float*         idle = (it & 1ull) ? a.contrib0 : a.contrib1;
    CK(launch_ppr_repack(a.rank, idle, n, K, K2, b.slot_map, nact, g->sms, s), "ppr repack");
    CK(cudaMemcpyAsync(a.rank, idle, n * (uint64_t)K2 * sizeof(float), cudaMemcpyDeviceToDevice, s), "ppr repack");
    if (a.vbase) {  // teleport vectors: their base terms move with their columns
      CK(launch_ppr_repack(a.vbase, idle, n, K, K2, b.slot_map, nact, g->sms, s), "ppr repack");
      CK(cudaMemcpyAsync(const_cast<float*>(a.vbase), idle, n * (uint64_t)K2 * sizeof(float), cudaMemcpyDeviceToDevice, s),
         "ppr repack");
    }
    CK(launch_ppr_repack(cur, idle, n, K, K2, b.slot_map, nact, g->sms, s), "ppr repack");
    CK(launch_ppr_repack_cols(a, K2, b.slot_map, nact, s), "ppr repack");
    if (it & 1ull) {
      a.contrib1 = idle;
      a.contrib0 = cur;
    } else {
      a.contrib0 = idle;
      a.contrib1 = cur;
    }
    a.K = (uint32_t)K2;
    K = K2;
    for (int j = 0; j < K; ++j) orig[j] = orig2[j];
    narrowed_any = true;
    PprState h = *b.h_st;
    h.done = 0u;
    h.narrowed = 0u;
    h.narrow_at = K > 32 ? (unsigned int)(K / 2) : 0u;
    *b.h_st = h;
    CK(cudaMemcpyAsync(b.st, b.h_st, sizeof(PprState), cudaMemcpyHostToDevice, s), "copy ppr state");
    const int grid = ppr_sweep_grid(K, g->sms);
    for (;;) {  // a few sweeps per check: the narrowed phases are short
      const uint64_t left = max_iters - b.h_st->iter, batch = left < 4 ? left : 4;
      for (uint64_t i = 0; i < batch; ++i) CK(launch_ppr_sweep(a, K, grid, s), "ppr sweep");
      CK(cudaMemcpyAsync(b.h_st, b.st, sizeof(PprState), cudaMemcpyDeviceToHost, s), "copy ppr state");
      CK(cudaStreamSynchronize(s), "ppr sweep loop");
      if (b.h_st->done || b.h_st->iter >= max_iters) break;
    }
  }
  CK(cudaEventRecord(g->ev1, s), "cudaEventRecord");
  if (narrowed_any) {
    CK(cudaMemcpyAsync(b.slot_orig, orig, K * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "copy slots");
    CK(launch_ppr_output_slots(a.rank, perm, n, K, b.slot_orig, k, dst, g->sms, s), "ppr output");
  } else {
    CK(launch_ppr_output(a.rank, perm, n, K, k, dst, g->sms, s), "ppr output");
  }
  if (!opt.device_ptrs)
    CK(cudaMemcpyAsync(ranks_nxk, dst, n * k * sizeof(float), cudaMemcpyDeviceToHost, s), "copy ranks");
  int rc = pull_stats(nullptr);  // synchronises the stream
  if (rc) return rc;
  const PprState fin = *b.h_st;
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->iterations = fin.iter;
    stats->device_ms = ms;
    stats->ms_per_iter = fin.iter ? ms / (double)fin.iter : 0.0;
    int all = 1;
    for (uint32_t c = 0; c < k; ++c) {
      all &= (h_conv[c] != 0);
      if (stats->col_iterations) stats->col_iterations[c] = h_iters[c];
      if (stats->col_errors) stats->col_errors[c] = h_err[c];
      if (stats->col_converged) stats->col_converged[c] = (int32_t)h_conv[c];
    }
    stats->all_converged = all;
  }
  if (fin.aborted) return fail(NWGPU_ERR_ABORTED, "batched solve aborted after %llu sweeps", (unsigned long long)fin.iter);
  return NWGPU_OK;
}
}  // namespace nwgpu

namespace nwgpu {
// Both teleport-matrix forms of the batched solve. Weighted: entry weights in
// the gather, out-weight sums as divisors. Unweighted: the caller's
// out-degrees as divisors. Column c starts at t_c with base terms
// (1 - d) t_c; the padding columns are stopped from the start.
static int teleport_batched(nwgpu_graph* g, bool weighted, const uint32_t* out_degree, const float* teleports,
                            uint32_t k, float* ranks_nxk, float damping, float threshold, uint64_t max_iters,
                            const nwgpu_pr_options* options, nwgpu_ppr_stats* stats) {
  if (!g) return fail(NWGPU_ERR_INVALID_ARG, "graph is NULL");
  if (k == 0 || k > 128) return fail(NWGPU_ERR_INVALID_ARG, "k = %u outside [1, 128]", k);
  if (g->n && (!teleports || !ranks_nxk || (!weighted && !out_degree)))
    return fail(NWGPU_ERR_INVALID_ARG, "NULL array argument");
  if (!(damping >= 0.0f && damping <= 1.0f)) return fail(NWGPU_ERR_INVALID_ARG, "damping %g outside [0, 1]", (double)damping);
  if (weighted && !g->g.w)
    return fail(NWGPU_ERR_UNSUPPORTED, "the graph has no edge weights (pass them to nwgpu_graph_create)");
  if (weighted && (!g->relabelled || !g->plan.ok))
    return fail(NWGPU_ERR_UNSUPPORTED, "weighted solves need a relabelled graph");
  nwgpu_pr_options opt = {};
  if (options) memcpy(&opt, options, options->size && options->size < sizeof(opt) ? options->size : sizeof(opt));
  if (opt.launch > NWGPU_LAUNCH_STREAM) return fail(NWGPU_ERR_INVALID_ARG, "launch %u unknown", opt.launch);
  const int      K = ppr_padded_k(k);
  const uint64_t n = g->n;
  if (stats) {
    uint32_t* ci = stats->col_iterations;
    double*   ce = stats->col_errors;
    int32_t*  cc = stats->col_converged;
    memset(stats, 0, sizeof(*stats));
    stats->col_iterations = ci;
    stats->col_errors = ce;
    stats->col_converged = cc;
    stats->bytes_per_iter =
        (weighted ? 8.0 : 4.0) * (double)g->nnz + 4.0 * (double)(n + 1) + 4.0 * (double)n + 20.0 * k * (double)n;
  }
  if (n == 0) return NWGPU_OK;
  int rc = ensure_solve_buffers(g);
  if (rc) return rc;
  if (weighted && (rc = ensure_wpr(g))) return rc;  // out-weight sums (internal order)
  if ((rc = ensure_ppr(g, K))) return rc;
  PprBuffers& b = g->ppr;
  if (!b.vbase) CK(dalloc(g, &b.vbase, n * (uint64_t)K), "cudaMalloc(ppr base terms)");
  cudaStream_t s = opt.stream ? (cudaStream_t)opt.stream : g->stream;
  *(volatile unsigned int*)g->h_abort = 0u;
  if (!weighted && (rc = load_degrees(g, out_degree, opt.device_ptrs != 0, s))) return rc;
  // teleports on the device (the output staging holds n x K >= n x k floats)
  const float* t = teleports;
  if (!opt.device_ptrs) {
    CK(cudaMemcpyAsync(b.out, teleports, n * k * sizeof(float), cudaMemcpyHostToDevice, s), "copy teleports");
    t = b.out;
  }
  PprArgs a = make_ppr_args(g, damping);
  a.vbase = b.vbase;
  if (weighted) {
    a.w = g->g.w;
    a.vaux = g->wpr.t.s;
  }
  CK(cudaMemsetAsync(b.seeds_in, 0, k * sizeof(uint32_t), s), "ppr columns");
  CK(launch_ppr_seeds(b.seeds_in, k, K, nullptr, a, s), "ppr columns");
  PprState h = {};
  h.max_iters = max_iters;
  h.chunk_end = kGraphChunk;
  h.threshold = (double)threshold;
  h.done = (max_iters == 0) ? 1u : 0u;
  h.narrow_at = K > 32 ? (unsigned int)(K / 2) : 0u;
  *b.h_st = h;
  CK(cudaMemcpyAsync(b.st, b.h_st, sizeof(PprState), cudaMemcpyHostToDevice, s), "copy ppr state");
  CK(launch_ppr_winit(a, K, t, k, g->relabelled ? g->g.inv : nullptr, n, b.vbase, g->sms, s), "ppr teleports init");
  return ppr_loop(g, a, K, k, ranks_nxk, damping, max_iters, opt, stats, s);
}
}  // namespace nwgpu

extern "C" int nwgpu_wppr_batched(nwgpu_graph* g, const float* teleports, uint32_t k, float* ranks_nxk, float damping,
                                  float threshold, uint64_t max_iters, const nwgpu_pr_options* options,
                                  nwgpu_ppr_stats* stats) {
  clear_error();
  return teleport_batched(g, true, nullptr, teleports, k, ranks_nxk, damping, threshold, max_iters, options, stats);
}

extern "C" int nwgpu_ppr_batched_teleports(nwgpu_graph* g, const uint32_t* out_degree, const float* teleports,
                                           uint32_t k, float* ranks_nxk, float damping, float threshold,
                                           uint64_t max_iters, const nwgpu_pr_options* options,
                                           nwgpu_ppr_stats* stats) {
  clear_error();
  return teleport_batched(g, false, out_degree, teleports, k, ranks_nxk, damping, threshold, max_iters, options, stats);
}
