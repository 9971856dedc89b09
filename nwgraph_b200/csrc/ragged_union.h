// Internal interface of the union solve of a ragged batch (ragged_union.cu).
#pragma once

#include "binned.h"
#include "engine.h"

namespace nwgpu {

// The graphs of a union, in batch order: part j is batch graph ids[j], its
// union vertices [voff[j], voff[j + 1]) and entries [eoff[j], eoff[j + 1]).
// Each part's vertices are cut into chunks of kUnionChunk for the per-graph
// sums of the sweep's changes: part j's chunks are [coff[j], coff[j + 1]).
constexpr uint32_t kUnionChunk = 4096;
struct UnionParts {
  const uint32_t* ids;   // m batch graph indices
  const uint64_t* voff;  // m + 1
  const uint64_t* eoff;  // m + 1
  const uint32_t* coff;  // m + 1
  double*         chunk_part;  // coff[m] chunk sums of the last sweep's changes
  uint32_t        m;
  uint32_t        chunks;      // coff[m]
  uint64_t        n, nnz;  // union vertices and entries (both below 2^32)
};

// The union CSR (n + 1 row pointers, nnz column ids) from the batch's per-graph local CSRs.
cudaError_t launch_union_build(const RaggedGraph* graphs, const uint32_t* batch_row_ptr, const uint32_t* batch_col,
                               const UnionParts& p, uint32_t* rp, uint32_t* col, int sms, cudaStream_t s);
// row_graph[r] = the batch graph of the relabelled union's internal row r (inv: internal -> union id).
cudaError_t launch_union_row_graph(const uint32_t* inv, const UnionParts& p, uint32_t* row_graph, int sms,
                                   cudaStream_t s);
// Start of a solve: base terms and fresh states of the union's graphs (stopped = max_iters == 0); degrees, ranks
// and contributions of its internal rows.
cudaError_t launch_union_start(const RaggedGraph* graphs, const UnionParts& p, const uint32_t* inv,
                               const uint32_t* row_graph, const uint32_t* batch_deg, float damping, uint32_t stopped,
                               float* base, const RaggedState& rs, uint32_t* deg, float* rank, float* contrib, int sms,
                               cudaStream_t s);
// Per-graph stopping tests after a sweep (perm: union id -> internal row).
cudaError_t launch_union_converge(const UnionParts& p, const uint32_t* perm, const double* row_res,
                                  const RaggedState& rs, PrState* st, double threshold,
                                  const volatile unsigned int* abort_word, int sms, cudaStream_t s);
// The union's ranks into the batch's rank array.
cudaError_t launch_union_output(const RaggedGraph* graphs, const UnionParts& p, const uint32_t* perm, const float* rank,
                                float* out, int sms, cudaStream_t s);
// The solve loop as a CUDA graph: a while node over sweep, finishing and convergence kernels.
cudaError_t build_union_graph(cudaGraph_t cg, const BinnedArgs& proto, int sweep_grid, int finish_grid,
                              const UnionParts& p, const uint32_t* perm, const double* row_res, const RaggedState& rs,
                              PrState* st, double threshold, const volatile unsigned int* abort_word, int sms,
                              cudaGraphExec_t* exec);

}  // namespace nwgpu
