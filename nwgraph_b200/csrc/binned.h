// Internal interface of the degree-binned sweep (pr_binned.cu).
#pragma once

#include "engine.h"

namespace nwgpu {

// Defaults of the plan's two runtime cut-offs (the tuner searches both):
constexpr uint32_t kLongRow = 2048;  // rows longer than this are split into chunks
constexpr uint32_t kChunk = 1024;    // entries per long-row chunk (one warp)
constexpr uint32_t kBin0Rows = 2;    // bin-0 rows per warp: 2 (half a warp each) or 1 (a whole warp)
constexpr int      kNumBins = 8;     // warp per row, then G = 32, 16, 8, 4, 2, 1, empty

struct BinnedArgs {
  SweepArgs       sw;                     // row_ptr / col / vectors / state / loop control
  uint32_t        long_row;               // rows longer than this are chunked (> 128)
  uint32_t        chunk;                  // entries per long-row chunk (a multiple of 256)
  uint32_t        bin0_rows;              // bin-0 rows per warp (kBin0Rows unless tuned or set): 2 or 1
  uint32_t        num_long_rows;          // rows [0, num_long_rows) are chunked
  uint32_t        num_big_rows;           // rows [0, num_big_rows) have more than 32 chunks
  uint32_t        num_chunks;
  const uint32_t* row_first_chunk;        // num_long_rows + 1
  const uint32_t* chunk_row;              // num_chunks
  float*          chunk_part;             // num_chunks partial sums
  uint32_t        bin_row_begin[kNumBins];
  uint32_t        bin_row_end[kNumBins];
  uint32_t        bin_warp_end[kNumBins]; // cumulative warps over the bins
  // bin 0: 129..long_row entries, half a warp or a warp per row; bins 1-6: G = 32..1 lanes
  // per row, two rows per lane group, rows of (2G, 4G] entries (G = 1: 1..4);
  // bin 7: empty rows
  uint32_t        smem_ids;               // hot variant: contrib[0, smem_ids) is staged in shared memory
  uint32_t        l1_ids;                 // ids in [smem_ids, l1_ids) are gathered through L1 (evict-last)
};

// Launch shapes of the binned sweep: 256-thread CTAs, four per SM, hub ids
// through L1; or one 1024-thread CTA per SM with the hub contributions staged
// in shared memory at the start of every sweep.
constexpr int kBinnedThreads = 256;
constexpr int kBinnedHotThreads = 1024;

cudaError_t launch_bin_bounds(const uint32_t* row_ptr, uint32_t n, uint32_t long_row, uint32_t chunk, uint32_t* d_out,
                              unsigned int* d_unsorted, int sms, cudaStream_t s);
cudaError_t launch_chunk_count(const uint32_t* row_ptr, uint32_t nlong, uint32_t chunk, uint32_t* cnt, int sms,
                               cudaStream_t s);
cudaError_t launch_chunk_fill(const uint32_t* first, uint32_t nlong, uint32_t* chunk_row, int sms, cudaStream_t s);
int         binned_sweep_grid(int sms, bool hot);
uint32_t    binned_hot_capacity();  // ids the hot variant can stage (a multiple of 4)
cudaError_t configure_binned_kernels();
int         binned_finish_grid(const BinnedArgs& a);
// mode: SweepMode. The weighted and adjoint sweeps always use the hot shape
// (sweep_grid = binned_sweep_grid(sms, true)).
cudaError_t launch_binned_sweep(const BinnedArgs& a, bool hot, int mode, int sweep_grid, int finish_grid, cudaStream_t s);
// finish_node (optional): the finishing kernel's node, the body's last.
cudaError_t add_binned_nodes(cudaGraph_t body, const BinnedArgs& a, bool hot, int mode, int sweep_grid, int finish_grid,
                             cudaGraphNode_t* finish_node = nullptr);

}  // namespace nwgpu
