// Internal interface of the destination-blocked sweep (pr_blocked.cu).
#pragma once

#include <vector>

#include "engine.h"

namespace nwgpu {

// Rows per destination block: the block's row sums live in shared memory as
// 64-bit fixed-point accumulators (28672 x 8 B = 224 KB, one 1024-thread CTA
// per SM).
constexpr uint32_t kBlockRows = 28672;
constexpr int      kBlockedThreads = 1024;
// PrState::fault bit set before a solve when some out_degree[j] is below the
// number of entries whose column is j: then row sums are no longer bounded by
// 1 and could overflow the fixed-point sums, so the solve runs the binned sweep.
constexpr unsigned int kFaultDegrees = 0x40000000u;

// One unit of work of a sweep: entries [e0, e1) of block `block` in the
// blocked entry order. A block of more than the piece size is cut into
// `pieces` items, whose partial sums meet in a global accumulator; the others
// are one item (pieces == 1) and finish in shared memory.
struct BlockItem {
  uint32_t block;
  uint32_t e0;
  uint32_t e1;
  uint32_t pieces;
};

// Packed entries: one 32-bit word per entry, (source - group base) << 15 |
// row within the block, for groups of 32 consecutive entries of a block. A
// group whose sources span 2^17 or more is "wide": its base word is
// kWideGroup | w, and its 32 sources are wide[32 w .. 32 w + 31].
constexpr uint32_t kPackRowBits = 15;  // kBlockRows <= 2^15
constexpr uint32_t kPackSpan = 1u << (32 - kPackRowBits);
constexpr uint32_t kWideGroup = 0x80000000u;

struct BlockedArgs {
  SweepArgs           sw;          // vectors, state, loop control, damping / teleport
  const uint32_t*     src;         // nnz: source (column id) of each entry, by (block, source); packed: the words
  const uint16_t*     dst;         // nnz: the entry's row within its block (unpacked only)
  const uint32_t*     gbase;       // packed: per group its base source, or kWideGroup | wide index
  const uint32_t*     wide;        // packed: sources of the wide groups
  const uint32_t*     blk_e0;      // packed: per block its first entry (num_blocks + 1)
  const uint32_t*     blk_g0;      // packed: per block its first group (num_blocks + 1)
  const BlockItem*    items;       // num_items, the largest first
  uint32_t            num_items;
  uint32_t            num_blocks;
  uint32_t            n;
  const uint32_t*     zoff;        // per block: its rows' first slot in zacc (blocks cut into pieces)
  unsigned long long* zacc;        // fixed-point row sums of the blocks cut into pieces; zero between sweeps
  uint32_t*           ticket;      // per block: pieces finished in this sweep
  double*             res_blk;     // per block: FP64 L1 change of its rows in the last sweep
  uint32_t*           next_item;   // the sweep's work counter; reset by the finishing kernel
};

// The blocked entry order of one CSR and its work list.
struct BlockPlan {
  bool                ok = false;
  uint32_t            num_blocks = 0;
  uint32_t*           src = nullptr;
  uint16_t*           dst = nullptr;
  bool                packed = false;  // src holds packed words; dst is empty
  uint32_t*           gbase = nullptr;
  uint32_t*           wide = nullptr;
  uint32_t*           blk_e0 = nullptr;
  uint32_t*           blk_g0 = nullptr;
  uint64_t            wide_groups = 0;
  uint32_t*           outcount = nullptr;  // n: entries whose column is j (the true out-degrees)
  BlockItem*          items = nullptr;
  uint32_t            num_items = 0;
  uint32_t*           zoff = nullptr;
  unsigned long long* zacc = nullptr;
  uint32_t*           ticket = nullptr;
  double*             res_blk = nullptr;
  uint32_t*           next_item = nullptr;
  uint64_t            bytes = 0;
  int                 sweep_grid = 0;
  int                 loads = 8;       // entries in flight per thread: 4, 8 or 16
  uint64_t            piece_entries = 0;
  uint64_t            n = 0, nnz = 0;
  std::vector<uint32_t> block_ptr;     // host: first entry of each block (num_blocks + 1)
  void                release(cudaStream_t s);
};

// Builds p from the CSR (rows in any order; the blocks are row ranges of
// kBlockRows rows); column ids are below id_bound. piece_entries: the largest
// item; 0 picks one from the SM count. packed: 4 bytes per entry (packed
// words) instead of 6 (source and row arrays); ignored when id_bound > 2^31.
cudaError_t build_block_plan(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, uint64_t nnz, uint64_t id_bound,
                             int sms, uint64_t piece_entries, bool packed, BlockPlan* p, cudaStream_t s);
// Rebuilds p's work list for another piece size (the entry order stays).
cudaError_t set_block_items(BlockPlan* p, int sms, uint64_t piece_entries, cudaStream_t s);
BlockedArgs make_blocked_args(const BlockPlan& p, const SweepArgs& sw, uint64_t n);
// Sets kFaultDegrees in st->fault when some deg[j] (internal order) < outcount[j].
cudaError_t launch_check_degrees(const BlockPlan& p, const uint32_t* deg, PrState* st, int sms, cudaStream_t s);
cudaError_t configure_blocked_kernels();
cudaError_t launch_blocked_sweep(const BlockedArgs& a, int sweep_grid, int loads, cudaStream_t s);
cudaError_t add_blocked_nodes(cudaGraph_t body, const BlockedArgs& a, int sweep_grid, int loads);

}  // namespace nwgpu
