// Internal interface of the batched personalised PageRank kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nwgpu {

constexpr int kPprTileItems = 512;  // merge items per warp tile
// What a batched solve's columns are: one-hot teleports at seeds; teleport
// vectors on a weighted graph; teleport vectors on an unweighted graph.
constexpr int kPprSeeds = 0, kPprWeighted = 1, kPprTeleports = 2;

struct PprState {
  unsigned long long iter;
  unsigned long long max_iters;
  unsigned long long chunk_end;
  double             threshold;
  unsigned int       ticket;
  unsigned int       done;
  unsigned int       aborted;
  unsigned int       narrow_at;  // stop once at most this many columns still run (0: never), to narrow K
  unsigned int       narrowed;   // the loop stopped for narrowing, not at the end of the solve
  unsigned int       pad_;
};

struct PprArgs {
  const uint32_t* row_ptr;
  const uint32_t* col;
  const uint32_t* tile_row;  // warp tiles of kPprTileItems
  const uint32_t* tile_nnz;
  uint32_t        num_tiles;
  uint32_t        tile_items;
  const uint32_t* deg;
  float*          rank;      // n x K
  float*          contrib0;  // n x K, ping-pong
  float*          contrib1;
  float*          cpart;     // num_tiles x K
  float*          epart;
  double*         res_part;  // epi_grid x K: the epilogue's per-CTA column residuals
  uint32_t        epi_grid;
  uint64_t        n;
  uint32_t        K;          // padded column count
  const uint4*    spans;      // rows crossing warp tiles: (row, first tile, last tile)
  uint32_t        num_spans;
  const uint32_t* seeds;     // K internal seed ids (0xffffffff: padding column)
  uint32_t*       col_done;  // K flags
  uint32_t*       col_conv;  // K flags
  uint32_t*       col_iters; // K sweep counts
  double*         col_err;   // K last L1 changes
  PprState*       st;
  const volatile unsigned int* abort_word;
  cudaGraphConditionalHandle   cond;
  int                          use_cond;
  float                        damping;
  float                        one_minus_d;
  // Teleport vectors: base terms (1 - d) t (n x K); weighted solves (w != null)
  // also entry weights and out-weight sums (n), all in internal order.
  const float*                 w;
  const float*                 vbase;
  const float*                 vaux;
};

int         ppr_padded_k(uint32_t k);
int         ppr_mode(const PprArgs& a);  // kPprSeeds, kPprWeighted or kPprTeleports
// Rows crossing warp tiles (spans[count] = (row, first tile, last tile), any order).
cudaError_t launch_ppr_spans(const uint32_t* row_ptr, const uint32_t* tile_row, const uint32_t* tile_nnz, uint32_t T,
                             uint32_t D, uint4* spans, unsigned int* count, int sms, cudaStream_t s);
int         ppr_sweep_grid(int K, int sms);
cudaError_t launch_ppr_seeds(const uint32_t* seeds_in, uint32_t k, int K, const uint32_t* perm, const PprArgs& a,
                             cudaStream_t s);
cudaError_t launch_ppr_init(const PprArgs& a, int K, uint64_t n, int sms, cudaStream_t s);
// Start from teleports t_in (n x k row-major, input order; inv: internal ->
// input id): vbase = (1 - d) t, rank = t, contrib = t / s per column, s the
// out-weight sums a.vaux, or the out-degrees a.deg when a.vaux is null.
cudaError_t launch_ppr_winit(const PprArgs& a, int K, const float* t_in, uint32_t k, const uint32_t* inv, uint64_t n,
                             float* vbase, int sms, cudaStream_t s);
cudaError_t launch_ppr_output(const float* rank, const uint32_t* perm, uint64_t n, int K, uint32_t k, float* out,
                              int sms, cudaStream_t s);
cudaError_t launch_ppr_sweep(const PprArgs& a, int K, int sweep_grid, cudaStream_t s);
// Narrowing: dst (n x K_to) = the columns map[0, nact) of src (n x K_from), zeros after them.
cudaError_t launch_ppr_repack(const float* src, float* dst, uint64_t n, int K_from, int K_to, const uint32_t* map,
                              uint32_t nact, int sms, cudaStream_t s);
// The per-column state (seeds, flags, sweep counts, errors) of slots map[0, nact) moved to slots [0, nact);
// slots [nact, K_to) become stopped padding.
cudaError_t launch_ppr_repack_cols(const PprArgs& a, int K_to, const uint32_t* map, uint32_t nact, cudaStream_t s);
// out[i * k + slot_orig[j]] = rank[perm[i] * K + j] for the slots j < K whose column is < k.
cudaError_t launch_ppr_output_slots(const float* rank, const uint32_t* perm, uint64_t n, int K, const uint32_t* slot_orig,
                                    uint32_t k, float* out, int sms, cudaStream_t s);
cudaError_t build_ppr_graph(cudaGraph_t g, const PprArgs& proto, int K, int sweep_grid, PprState* st,
                            cudaGraphExec_t* exec);

}  // namespace nwgpu
