// Internal interface between the C ABI (api.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nwgpu {

// Device-resident solve state; one per graph handle. Written by the host
// before a solve and by the last CTA of each sweep.
struct PrState {
  unsigned long long iter;       // sweeps completed
  unsigned long long max_iters;  // sweep limit of this solve
  unsigned long long chunk_end;  // the graph loop stops after this sweep count (bounds one launch)
  double             threshold;  // stop when the sweep's L1 change < threshold
  double             last_error; // L1 change of the last sweep
  unsigned int       ticket;     // CTA arrivals in the current sweep
  unsigned int       done;       // 1 once converged, at max_iters, or aborted
  unsigned int       converged;
  unsigned int       aborted;
};

struct Tiling {
  int       items_per_thread;  // IPT; a tile holds NT * IPT rows + entries
  uint32_t  num_tiles;
  uint32_t* tile_row;  // num_tiles + 1 merge-path row coordinates
  uint32_t* tile_nnz;  // num_tiles + 1 merge-path entry coordinates
};

struct SweepArgs {
  const uint32_t* row_ptr;
  const uint32_t* col;
  const uint32_t* tile_row;
  const uint32_t* tile_nnz;
  uint32_t        num_tiles;
  float*          contrib0;  // contribution vectors, ping-pong by sweep parity
  float*          contrib1;
  float*          rank;
  const uint32_t* deg;
  float*          cpart;     // per tile: partial sum of the row it carries out
  float*          epart;     // per tile: partial sum of the continued row it completes
  uint32_t*       cnt;       // per tile: arrivals for the spanning row that starts there
  double*         res_part;  // per CTA residual partials
  PrState*        st;
  double*         err_hist;  // per-sweep L1 errors (ring of err_cap)
  uint32_t        err_cap;
  const volatile unsigned int* abort_word;  // host-mapped; nonzero -> stop
  cudaGraphConditionalHandle   cond;
  int                          use_cond;
  float                        damping;
  float                        base;
};

constexpr int kSweepThreads = 256;
constexpr unsigned long long kGraphChunk = 4096;  // sweeps per graph launch, at most

// pr_plain.cu
cudaError_t build_tiling(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, int ipt, Tiling* t, cudaStream_t s);
cudaError_t validate_csr(const uint32_t* d_row_ptr, const uint32_t* d_col, uint64_t n, uint64_t nnz,
                         unsigned int* d_err, cudaStream_t s);
cudaError_t launch_pr_init(const SweepArgs& a, uint64_t n, float init, cudaStream_t s);
cudaError_t launch_pr_sweep(const SweepArgs& a, int ipt, int grid, cudaStream_t s);
cudaError_t add_pr_sweep_node(cudaGraph_t body, const SweepArgs& a, int ipt, int grid);
cudaError_t add_pr_arm_node(cudaGraph_t g, PrState* st, cudaGraphNode_t* node);
int         sweep_blocks_per_sm(int ipt);
bool        ipt_supported(int ipt);

}  // namespace nwgpu
