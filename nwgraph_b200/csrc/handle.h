// Internal: the graph handle and host helpers shared by the C ABI files.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/nwgpu.h"
#include "engine.h"
#include "ppr.h"
#include "binned.h"
#include "blocked.h"

namespace nwgpu {

int  fail(int code, const char* fmt, ...);
int  cuda_fail(cudaError_t e, const char* what);
void clear_error();
const std::string& last_error_text();
// Current device (must be compute capability 10.x) and its SM count; configures
// the sweep kernels once per process.
int  check_device(int* dev_out, int* sms_out);

#define CK(call, what)                                         \
  do {                                                         \
    cudaError_t _e = (call);                                   \
    if (_e != cudaSuccess) return ::nwgpu::cuda_fail(_e, what); \
  } while (0)

// Bin tables of one CSR for the degree-binned sweep.
struct BinPlan {
  bool       ok = false;        // the rows are in non-increasing length order and the tables exist
  bool       hot = false;       // hub contributions staged in shared memory
  BinnedArgs bin{};             // tables; the SweepArgs part is filled per solve
  uint32_t*  first = nullptr;   // row_first_chunk
  uint32_t*  chunk_row = nullptr;
  float*     chunk_part = nullptr;
  int        sweep_grid = 0, finish_grid = 1;
  uint64_t   bytes = 0;                 // device memory of the chunk tables
  void       release(cudaStream_t s);
};

// Buffers of the weighted solve and its adjoint (created on first use).
struct WprBuffers {
  bool       ready = false;
  Transposed t{};                // out-row CSR, out-weight sums
  BinPlan    tplan;              // bins of the out-row CSR (adjoint sweeps)
  float*     vbase = nullptr;    // n: (1-d) t (forward) or c (adjoint), internal order
  float*     vaux = nullptr;     // n: d / s (adjoint)
  float*     r_int = nullptr;    // n: forward ranks, internal order
  float*     stage = nullptr;    // n: input-order staging
  float*     stage2 = nullptr;   // n: input-order staging
  double*    res = nullptr;      // residual partials of the adjoint sweep
  float*     gw = nullptr;       // nnz: dL/dw staging for host outputs
  // GMRES adjoint: Krylov basis (kGmresRestart + 1 vectors of stride ld),
  // operator output, -d/s, per-block reduction partials, reduction results
  float*     basis = nullptr;
  uint64_t   ld = 0;
  float*     w = nullptr;
  float*     vneg = nullptr;
  double*    part = nullptr;
  double*    dout = nullptr;
  float*     f = nullptr;        // n: dL/dw factors d r_j / s_j
  float*     q = nullptr;        // n: dL/dw offsets q_j
  void       release(cudaStream_t s);
};

// Buffers of the batched personalised solve (K padded columns).
struct PprBuffers {
  int             K = 0;
  Tiling          tiling{};  // warp tiles of kPprTileItems
  int             sweep_grid = 0, finish_grid = 0;
  float*          rank = nullptr;
  float*          contrib[2] = {nullptr, nullptr};
  float*          out = nullptr;  // n x K staging for the output
  float*          cpart = nullptr;
  float*          epart = nullptr;
  double*         res_part = nullptr;
  uint4*          spans = nullptr;  // rows crossing warp tiles
  uint32_t        num_spans = 0;
  uint32_t*       seeds = nullptr;
  uint32_t*       seeds_in = nullptr;
  uint32_t*       col_done = nullptr;
  uint32_t*       col_conv = nullptr;
  uint32_t*       col_iters = nullptr;
  double*         col_err = nullptr;
  PprState*       st = nullptr;
  PprState*       h_st = nullptr;
  cudaGraph_t     cg = nullptr;
  cudaGraphExec_t cg_exec = nullptr;
  float           cg_damping = -1.f;
  int             cg_mode = -1;  // ppr_mode of the solve baked into cg_exec
  float*          vbase = nullptr;  // weighted solves: n x K base terms (1 - d) t
  uint32_t*       slot_map = nullptr;   // narrowing: old slot of each new slot
  uint32_t*       slot_orig = nullptr;  // caller's column held by each slot (>= k: none)
  void            release(cudaStream_t s);  // returns the buffers to the pool on stream s
};

}  // namespace nwgpu

struct nwgpu_graph {
  int          device = 0;
  int          sms = 148;
  cudaStream_t stream = nullptr;
  uint64_t     n = 0, nnz = 0;
  bool         relabelled = false;
  nwgpu::Relabelled g;  // device CSR (relabelled, or the input order with perm/inv null)
  nwgpu::Tiling tiling{};
  int          grid = 0;         // persistent sweep CTAs
  uint32_t     hot_ids = 0;      // internal ids below this are gathered from shared memory / L1
  nwgpu::SweepVariant variant{256, 8, false};
  int          tuned = 0;        // binned launch parameters: 0 defaults, 1 timed at creation, 2 from the tuning cache
  float        tune_us = 0.f;    // the chosen parameters' time per sweep when tuned
  // Degree-binned sweep (relabelled graphs with non-increasing row lengths).
  nwgpu::BinPlan plan;
  // Destination-blocked sweep (plain and single-seed solves), built at creation with NWGPU_SWEEP=blocked.
  nwgpu::BlockPlan bplan;
  bool             blocked_off = false;  // this solve's degrees failed the blocked sweep's check: binned sweep
  bool             cg_blocked = false;   // the cached loop graph runs the blocked sweep
  int          finish_grid = 1;  // finishing-kernel CTAs
  uint64_t     device_bytes = 0;

  // Plain-solve buffers, allocated on first use and kept.
  bool          solve_ready = false;
  float*        rank = nullptr;
  float*        contrib[2] = {nullptr, nullptr};
  uint32_t*     deg = nullptr;
  uint32_t*     stage_u32 = nullptr;  // host <-> device staging in input order
  float*        cpart = nullptr;
  float*        epart = nullptr;
  double*       res_part = nullptr;
  uint64_t      res_parts = 0;          // entries of res_part
  nwgpu::PrState* st = nullptr;
  double*       err_hist = nullptr;
  uint32_t      err_cap = 4096;
  nwgpu::PrState* h_st = nullptr;     // pinned mirror of *st
  unsigned int* h_abort = nullptr;  // mapped pinned abort word
  unsigned int* d_abort = nullptr;
  cudaEvent_t   ev0 = nullptr, ev1 = nullptr;

  // CUDA graph of the sweep loop (arm node -> while node { sweep; finish }).
  cudaGraph_t     cg = nullptr;
  cudaGraphExec_t cg_exec = nullptr;
  nwgpu::SweepArgs cg_args{};  // arguments baked into cg_exec
  const nwgpu::BinPlan* cg_plan = nullptr;
  int             cg_mode = 0;

  nwgpu::PprBuffers ppr;
  nwgpu::WprBuffers wpr;
  float*        unit = nullptr;  // n ones (nwgpu_spmv: out-weight sums of 1)
  float*        zero = nullptr;  // n zeros (nwgpu_spmv: base terms of 0)

  ~nwgpu_graph() {
    ppr.release(stream);
    wpr.release(stream);
    plan.release(stream);
    bplan.release(stream);
    if (cg_exec) cudaGraphExecDestroy(cg_exec);
    if (cg) cudaGraphDestroy(cg);
    void* dev_ptrs[] = {g.row_ptr, g.col, g.w, g.perm, g.inv, g.emap, tiling.tile_row, tiling.tile_nnz, rank, contrib[0],
                        contrib[1], deg, stage_u32, cpart, epart, res_part, st, err_hist, unit, zero};
    for (void* p : dev_ptrs) nwgpu::pool_free(p, stream);
    cudaStreamSynchronize(stream);  // the blocks are free for the next handle at once
    nwgpu::host_block_put(h_st);  // the stream is idle: no copy still targets them
    nwgpu::host_block_put(h_abort);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace nwgpu {
template <class T>
cudaError_t dalloc(nwgpu_graph* g, T** p, uint64_t count) {
  const uint64_t bytes = (count + kPad) * sizeof(T);
  cudaError_t    e = pool_alloc((void**)p, bytes, g->stream);
  if (e == cudaSuccess) {
    g->device_bytes += bytes;
    e = cudaMemsetAsync(*p, 0, bytes, g->stream);
  }
  return e;
}
int ensure_solve_buffers(nwgpu_graph* g);
int build_bin_plan(nwgpu_graph* g, const uint32_t* row_ptr, uint64_t n, bool hot, BinPlan* p,
                   uint32_t long_row = kLongRow, uint32_t chunk = kChunk, uint32_t bin0_rows = kBin0Rows);
// g->plan rebuilt with other long-row cut-offs or bin-0 rows per warp, keeping
// its launch shape and hub tiers.
int rebuild_bin_plan(nwgpu_graph* g, uint32_t long_row, uint32_t chunk, uint32_t bin0_rows);
// Residual partials the handle's sweeps write: the merge-path sweep's, or the
// binned plan's in its larger launch shape (the tuner may switch shapes).
uint64_t residual_parts(const nwgpu_graph* g);
// Sweep grid of a binned solve (the weighted and adjoint sweeps always use the
// hot launch shape) and the kernel arguments of one.
int        binned_grid(nwgpu_graph* g, const BinPlan& p, int mode);
BinnedArgs make_binned_args(nwgpu_graph* g, const BinPlan& p, const SweepArgs& sw, int mode);
// Sweep arguments over the handle's forward CSR and solve buffers.
SweepArgs make_sweep_args(nwgpu_graph* g, float damping, float base, int teleport, uint32_t seed);
// Runs the sweep loop from the state already on the device (CUDA graph or one
// launch per sweep); plan: the binned sweep's tables (null: merge-path sweep).
int run_sweeps(nwgpu_graph* g, const SweepArgs& a, uint32_t launch, uint64_t max_iters, cudaStream_t s, PrState* fin,
               const BinPlan* plan, int mode);
nwgpu_pr_options read_options(const nwgpu_pr_options* options);
// Graph-creation flag for internal callers: no blocked plan (a whole graph that
// is only relabelled and then cut into shards).
constexpr uint32_t kGraphNoBlockedPlan = 0x80000000u;
// Graph-creation flag for internal callers: tune the binned sweep's launch
// shape and hub tiers only, keeping the default long-row cut-offs, so the
// ranks equal an untuned handle's bit for bit (the graphs a ragged batch
// solves alone).
constexpr uint32_t kGraphTuneShapes = 0x40000000u;
// Whether a solve in `mode` over `plan` (the handle's forward plan or none) runs the blocked sweep.
bool use_blocked(const nwgpu_graph* g, const BinPlan* plan, int mode);
// run_sweeps' result when the degree check stopped a blocked solve before its first sweep (internal).
constexpr int kRetryBinned = 1000;
// Out-row CSR, its bins and the buffers of the weighted solve and its adjoint.
int ensure_wpr(nwgpu_graph* g);
// api_tune.cu: picks the binned sweep's long-row cut-offs (unless
// shapes_only), launch shape and hub tiers for g (timed, or from the
// per-signature cache) and sets g->plan accordingly.
int autotune_binned(nwgpu_graph* g, bool shapes_only = false);
// api_tune.cu: the long-row cut-offs and bin-0 rows per warp cached for g's
// signature, if any (else the arguments are left as they are), so a tuned
// graph like one already tuned builds its bin plan once.
int cached_cutoffs(nwgpu_graph* g, uint32_t* long_row, uint32_t* chunk, uint32_t* bin0_rows);
// api_tune.cu: picks the blocked sweep's entries in flight and piece size (timed, or cached per signature).
int autotune_blocked(nwgpu_graph* g);
// degrees (input order, host or device) -> g->deg (internal order)
int load_degrees(nwgpu_graph* g, const uint32_t* out_degree, bool device_ptrs, cudaStream_t s);
// nwgpu_pr_run's solve in two halves, for callers that run many graphs back to
// back on one stream (ragged batches). pr_solve_queue puts everything on s
// without waiting: the degrees (device pointer), the start, the first launch
// of the device-side sweep loop (a CUDA graph), the state copy and the ranks
// permuted into d_ranks (device pointer, input order). *queued is false, with
// nothing put on s, for the graphs that need the full call (no vertices, no
// binned sweep); the caller uses nwgpu_pr_run for them. After s has been
// synchronized, pr_solve_finish reads the state, runs the rest of a loop
// longer than one graph launch, and fills stats.
int pr_solve_queue(nwgpu_graph* g, const uint32_t* d_degree, float* d_ranks, float damping, float threshold,
                   uint64_t max_iters, cudaStream_t s, bool* queued);
int pr_solve_finish(nwgpu_graph* g, float* d_ranks, float damping, float threshold, uint64_t max_iters, cudaStream_t s,
                    nwgpu_pr_stats* stats);
}  // namespace nwgpu
