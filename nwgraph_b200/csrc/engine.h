// Internal interface between the C ABI (api.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nwgpu {

// Every device array is allocated with kPad spare elements so that 16-byte
// aligned bulk copies that round a slice outward stay inside the allocation.
constexpr uint64_t kPad = 16;
// Largest entry count of a graph (and of a ragged union). Row pointers and
// entry indices are uint32, and a sweep step forms indices up to 255 past a
// row's last entry (a 256-entry window), so those must stay below 2^32.
constexpr uint64_t kMaxEntries = 0xFFFFFE00ull;
constexpr int      kSweepThreads = 256;
constexpr unsigned long long kGraphChunk = 4096;  // sweeps per graph launch, at most

// Device-resident solve state; one per graph handle. Written by the host
// before a solve and by the last CTA of each sweep's finishing kernel.
struct PrState {
  unsigned long long iter;       // sweeps completed
  unsigned long long max_iters;  // sweep limit of this solve
  unsigned long long chunk_end;  // the graph loop stops after this sweep count (bounds one launch)
  double             threshold;  // stop when the sweep's L1 change < threshold
  double             last_error; // L1 change of the last sweep
  unsigned int       ticket;     // CTA arrivals of the finishing kernel in the current sweep
  unsigned int       done;       // 1 once converged, at max_iters, aborted or failed
  unsigned int       converged;
  unsigned int       aborted;
  unsigned int       fault;      // nonzero: a bounded device wait gave up (bit pattern = where)
  unsigned int       pending;    // ragged batches: graphs still running after the current sweep
};

struct Tiling {
  uint32_t  tile_items = 0;        // D: rows + entries per tile
  uint32_t  num_tiles = 0;
  uint32_t* tile_row = nullptr;    // num_tiles + 1 merge-path row coordinates
  uint32_t* tile_nnz = nullptr;    // num_tiles + 1 merge-path entry coordinates
};

// The relabelled CSR (vertices in descending out-degree order).
struct Relabelled {
  uint32_t* row_ptr = nullptr;  // n + 1 (+ kPad)
  uint32_t* col = nullptr;      // nnz (+ kPad)
  float*    w = nullptr;        // nnz (+ kPad) or null
  uint32_t* perm = nullptr;     // input id -> internal id
  uint32_t* inv = nullptr;      // internal id -> input id
  uint32_t* emap = nullptr;     // nnz: internal entry -> input entry (weighted graphs; null = identity)
};

// The out-row CSR (adjacency<0>) of the internal graph, for the adjoint:
// row j lists the entries whose column is j, in internal entry order.
struct Transposed {
  uint32_t* row_ptr = nullptr;  // n + 1
  uint32_t* col = nullptr;      // nnz: row (destination) of the forward entry
  float*    w = nullptr;        // nnz: weight of the forward entry
  uint32_t* fwd = nullptr;      // nnz: the forward entry
  float*    s = nullptr;        // n: out-weight sums, FP64 row sums of w rounded to FP32
  uint32_t* erow = nullptr;     // nnz: row of each forward entry
};

// One graph of a ragged batch: where its slices of the batch arrays start.
// Graph g has n local vertices and nnz entries; its row pointers (n + 1,
// local entry offsets) start at p0 = v0 + g, its column ids (local vertex
// ids) at e0, its ranks / contributions / degrees at v0, and its merge-path
// tiles (local diagonals, D items each, the last one partial) are tiles
// [tile0, tile0 + tiles) of the batch. Tile t's coordinates sit at index
// t + g of the tile tables, its end at t + g + 1.
struct RaggedGraph {
  uint64_t v0;
  uint64_t e0;
  uint64_t p0;
  uint32_t n;
  uint32_t nnz;
  uint32_t tile0;
  uint32_t tiles;
};

// Teleport term of the update r_i' = base_i + d * z_i.
enum TeleportMode : int {
  kTeleportUniform = 0,  // base_i = (1 - d) / n, page_rank.hpp:94
  kTeleportSeed = 1,     // personalised, one-hot: base_i = (1 - d) if i == seed else 0
};

// Update the binned sweep applies (page_rank.hpp:133-135 for kModePlain).
enum SweepMode : int {
  kModePlain = 0,     // z = sum contrib;      r = base + d z;          contrib' = r / deg
  kModeWeighted = 1,  // z = sum w * contrib;  r = vbase + d z;         contrib' = r / vaux  (vaux = out-weight sum)
  kModeAdjoint = 2,   // z = sum w * lambda;   l = vbase + vaux * z;    contrib' = l         (vaux = d / out-weight sum)
  kModeResidual = 3,  // residual push (page_rank_v13): z = sum delta; if z > push_threshold: r += z and
                      // delta' = z d / deg (deg > 0), else delta' = 0; the sweep "error" counts pushes
  kModeRagged = 4,    // the union of a ragged batch's graphs: as kModePlain with the row's graph's base term
                      // graph_base[row_graph[r]]; rows of stopped graphs (graph_done) are neither gathered nor
                      // updated; each updated row's FP64 |dr| goes to row_res[r] for the per-graph sums
};

struct SweepArgs {
  const uint32_t* row_ptr;
  const uint32_t* col;
  const uint32_t* tile_row;
  const uint32_t* tile_nnz;
  uint32_t        num_tiles;
  uint32_t        tile_items;  // D = kSweepThreads * IPT
  float*          contrib0;    // contribution vectors, ping-pong by sweep parity
  float*          contrib1;
  float*          rank;
  const uint32_t* deg;
  float*          cpart;       // per tile: partial sum of the row it carries out
  float*          epart;       // per tile: partial sum of the continued row it completes
  double*         res_part;    // residual partials: [0, sweep_grid) sweep kernel, then finishing kernel
  uint32_t        sweep_grid;
  PrState*        st;
  double*         err_hist;    // L1 errors of the first err_cap sweeps (later sweeps are not recorded)
  uint32_t        err_cap;
  const volatile unsigned int* abort_word;  // host-mapped; nonzero -> stop
  cudaGraphConditionalHandle   cond;
  int                          use_cond;
  float                        damping;
  float                        base;       // uniform teleport term (1 - d) / n
  int                          teleport;   // TeleportMode
  uint32_t                     seed;       // internal id of the one-hot teleport vertex
  uint32_t                     hot_ids;    // gathers of ids below this are cached in L1
  const float*                 w;          // kModeWeighted / kModeAdjoint: entry weights of the swept CSR
  const float*                 vbase;      // per-row base term (weighted: (1-d) t; adjoint: c)
  const float*                 vaux;       // per-row factor (weighted: out-weight sum; adjoint: d / out-weight sum)
  float                        push_threshold;  // kModeResidual: residuals above this are pushed
  // Nonzero: row_ptr, col, rank and deg are the caller's arrays of exactly
  // n_rows + 1, n_entries, n_rows and n_rows elements, with no spare elements
  // after them, so the merge-path sweep's tile copies read nothing past those
  // lengths (the no-alloc solve). Zero: the arrays carry kPad spare elements.
  int                          exact_ends;
  uint32_t                     n_rows;
  uint32_t                     n_entries;
  // Ragged batches only (the RAGGED sweep variant):
  const RaggedGraph*           graphs;
  const float*                 graph_base;  // per graph: (1 - d) / n
  double*                      res_tile;    // per tile: FP64 L1 change of the rows the tile completes
  // Tiles of the running graphs: running graph g's tiles are entries
  // [act_off[g], act_off[g + 1]) of the sweep's tile list act_list, as
  // (tile, graph) pairs (act_off[num_graphs] = their count); stopped graphs
  // have none.
  const uint32_t*              act_off;
  const uint2*                 act_list;
  uint32_t                     num_graphs;
  // kModeRagged (a union of graphs in one relabelled CSR): per internal row its graph, per graph whether it
  // stopped, per internal row the FP64 L1 change of the last sweep.
  const uint32_t*              row_graph;
  const uint32_t*              graph_done;
  double*                      row_res;
};

// Per-graph results of a ragged solve, written by the convergence kernel.
struct RaggedState {
  uint32_t* done;     // stopped (converged, at max_iters, aborted or failed)
  uint32_t* iters;    // sweeps run
  double*   err;      // L1 change of the last sweep
  uint32_t* conv;     // err < threshold
  uint32_t* act_off;  // num_graphs + 1: running graphs' tile-list offsets (SweepArgs::act_off)
  uint2*    act_list; // the tile list (SweepArgs::act_list)
};

// devmem.cu: the per-device stream-ordered pool that every handle allocation uses
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s);
void        pool_free(void* p, cudaStream_t s);
template <class T>
cudaError_t pool_alloc_n(T** p, uint64_t count, cudaStream_t s) {
  return pool_alloc(reinterpret_cast<void**>(p), (size_t)count * sizeof(T), s);
}

// devmem.cu: small mapped pinned blocks (kHostBlock bytes, zeroed) for the
// host mirrors of solve states and abort words, cached across handles: pinning
// and unpinning memory costs milliseconds per call. A block goes back with
// host_block_put only once no copy or kernel can still touch it.
constexpr size_t kHostBlock = 256;
cudaError_t host_block_get(void** p);
void        host_block_put(void* p);

// graph_build.cu
cudaError_t validate_csr(const uint32_t* d_row_ptr, const uint32_t* d_col, uint64_t n, uint64_t nnz,
                         unsigned int* d_err, int sms, cudaStream_t s);
cudaError_t build_tiling(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, uint32_t D, Tiling* t, cudaStream_t s);
// Merge-path coordinates into caller-owned tile_row / tile_nnz (num_tiles + 1 each).
cudaError_t fill_tiling(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, uint32_t D, uint32_t num_tiles,
                        uint32_t* tile_row, uint32_t* tile_nnz, cudaStream_t s);
cudaError_t validate_row_ptr(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, unsigned int* d_err, int sms,
                             cudaStream_t s);
cudaError_t build_relabelled(const uint32_t* d_row_ptr, const uint32_t* d_col, const float* d_w, uint64_t n,
                             uint64_t nnz, int sms, Relabelled* out, cudaStream_t s);
// The two halves of build_relabelled for a CSR whose column ids arrive in
// chunks: relabel_rows needs only the (validated) row pointers; scatter_entries
// places the entries of merge-path items [d0, d1) of the input CSR once they
// are on the device, setting bit 2 of *d_err for ids >= n.
cudaError_t relabel_rows(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, int sms, bool with_weights,
                         bool clear_entries, Relabelled* out, cudaStream_t s);
cudaError_t scatter_entries(const uint32_t* d_row_ptr, const uint32_t* d_col, uint64_t n, uint64_t nnz, uint64_t d0,
                            uint64_t d1, const Relabelled& out, unsigned int* d_err, int sms, cudaStream_t s);
cudaError_t build_transpose(const uint32_t* d_row_ptr, const uint32_t* d_col, const float* d_w, uint64_t n, uint64_t nnz,
                            int sms, Transposed* out, cudaStream_t s);

// pr_weighted.cu: set-up and gradient kernels of the weighted solve and its adjoint
cudaError_t launch_wpr_prepare(const float* t, const uint32_t* inv, const float* s, uint64_t n, float damping,
                               float* vbase, float* rank, float* contrib, int sms, cudaStream_t st);
cudaError_t launch_vjp_prepare(const float* r, const float* c, const uint32_t* inv, const float* s, uint64_t n,
                               float damping, float* r_int, float* vbase, float* vaux, float* lam, float* contrib, int sms,
                               cudaStream_t st);
// dL/dw over the forward entries (col: the forward CSR's columns); f, q: n-float scratch
cudaError_t launch_vjp_grad_w(const Transposed& t, const uint32_t* col, const uint32_t* emap, const float* r_int,
                              const float* lam, const float* c_int, uint64_t n, uint64_t nnz, float damping, float* f,
                              float* q, float* d_w, int sms, cudaStream_t st);
cudaError_t launch_vjp_grad_t(const float* lam, const uint32_t* perm, uint64_t n, float damping, float* d_t, int sms,
                              cudaStream_t st);

// Vector kernels of the GMRES adjoint solve (pr_weighted.cu). A VecGrid
// splits n into contiguous per-block ranges; reductions are FP64, fixed order.
constexpr int kGmresMaxBasis = 32;
struct VecGrid {
  int      blocks;
  uint64_t chunk;
};
VecGrid     vec_grid(uint64_t n, int sms);
// out[0..nv) = V_i . x for the nv (1..kGmresMaxBasis) vectors of V (stride
// ld), out[nv] = x . x; part: blocks * (nv + 1) doubles
cudaError_t launch_vec_dots(const float* V, uint64_t ld, int nv, const float* x, uint64_t n, const VecGrid& vg,
                            double* part, double* out, cudaStream_t st);
// y = scale * (x - sum_i coef[i] V_i) (x and y may alias); with out: the dots
// of the V_i with y, and y . y, as launch_vec_dots writes them
cudaError_t launch_vec_update(const float* x, float* y, const float* V, uint64_t ld, int nv, const float* coef, float scale,
                              uint64_t n, const VecGrid& vg, double* part, double* out, cudaStream_t st);
// y = alpha x + beta y; with l1_out: ||y||_1 after the update
cudaError_t launch_vec_axpby(float alpha, const float* x, float beta, float* y, uint64_t n, const VecGrid& vg,
                             double* part, double* l1_out, cudaStream_t st);
cudaError_t launch_neg_dinv(const float* s, uint64_t n, float damping, float* vaux, int sms, cudaStream_t st);
cudaError_t launch_op_state(PrState* st, cudaStream_t s);

// pr_plain.cu
cudaError_t launch_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint64_t n, int sms,
                              cudaStream_t s);
cudaError_t launch_gather_f32(const float* src, const uint32_t* idx, float* dst, uint64_t n, int sms, cudaStream_t s);
// One thread waits, with the sweeps' bounded mbarrier wait and `polls` polls,
// on a barrier that nothing completes; *gave_up = 1 when the wait gave up.
cudaError_t run_wait_selftest(uint32_t polls, unsigned int* gave_up, float* ms);
cudaError_t launch_pr_init(const SweepArgs& a, uint64_t n, float init, int sms, cudaStream_t s);
// Residual push, first phase of the first iteration: rank = push ? r0 : 0,
// delta = (push, deg > 0) ? r0 d / deg : 0, *pushed += vertices with both.
cudaError_t launch_residual_init(float* rank, float* delta, const uint32_t* deg, uint64_t n, float r0, float damping,
                                 bool push, unsigned int* pushed, int sms, cudaStream_t s);
// Sweep kernel variants: threads per CTA, items per thread, and whether the
// hottest ids are kept in shared memory (one large CTA per SM) or left to L1.
struct SweepVariant {
  int  threads;
  int  ipt;
  bool hot_smem;
  uint32_t tile_items() const { return (uint32_t)(threads * ipt); }
};
bool        sweep_variant_supported(const SweepVariant& v);
cudaError_t launch_pr_sweep(const SweepArgs& a, const SweepVariant& v, int grid, cudaStream_t s);
cudaError_t launch_pr_finish(const SweepArgs& a, int grid, cudaStream_t s);
cudaError_t add_pr_sweep_nodes(cudaGraph_t body, const SweepArgs& a, const SweepVariant& v, int sweep_grid,
                               int finish_grid);
cudaError_t add_pr_arm_node(cudaGraph_t g, PrState* st, cudaGraphNode_t* node);
cudaError_t configure_sweep_kernels();
cudaError_t set_sweep_carveout(const SweepVariant& v, int percent);
size_t      sweep_smem_bytes(const SweepVariant& v, uint32_t hot_ids);
// Ragged batches (pr_plain.cu): the merge-path sweep over per-graph tiles,
// the rows crossing tiles, then per-graph convergence and the loop condition.
constexpr uint32_t kRaggedTileItems = 2048;  // D of the ragged sweep (256 threads x 8 items)
cudaError_t launch_ragged_sweep(const SweepArgs& a, int sweep_grid, int finish_grid, uint32_t num_graphs,
                                const RaggedState& rs, int conv_grid, cudaStream_t s);
cudaError_t add_ragged_nodes(cudaGraph_t body, const SweepArgs& a, int sweep_grid, int finish_grid, uint32_t num_graphs,
                             const RaggedState& rs, int conv_grid);
// The running graphs' (tile, graph) list from act_off and the done flags
cudaError_t launch_ragged_list(const SweepArgs& a, const RaggedState& rs, int sms, cudaStream_t s);
// rank = 1/n_g, contrib = rank / deg over the batch's vertices; per-graph base
// terms and state reset
cudaError_t launch_ragged_init(const SweepArgs& a, const RaggedState& rs, uint32_t num_graphs, uint64_t num_vertices,
                               float damping, uint32_t stopped, int sms, cudaStream_t s);
// graph_build.cu: merge-path coordinates of every graph's tiles (num_tiles +
// num_graphs entries)
cudaError_t fill_ragged_tiling(const RaggedGraph* graphs, uint32_t num_graphs, const uint32_t* row_ptr,
                               uint32_t num_tiles, uint32_t* tile_row, uint32_t* tile_nnz, int sms, cudaStream_t s);
// Checks every graph's row pointers (first 0, last nnz, non-decreasing) and
// column ids (< n); sets the bits validate_csr sets.
cudaError_t validate_ragged(const RaggedGraph* graphs, uint32_t num_graphs, const uint32_t* row_ptr, const uint32_t* col,
                            uint64_t num_row_ptrs, uint64_t num_entries, unsigned int* err, int sms, cudaStream_t s);
uint32_t    sweep_hot_capacity(const SweepVariant& v);  // ids that fit in shared memory (hot_smem variants)
int         sweep_blocks_per_sm(const SweepVariant& v, uint32_t hot_ids);
int         finish_grid_for(uint32_t num_tiles);

}  // namespace nwgpu
