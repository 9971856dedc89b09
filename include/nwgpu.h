/*
 * nwgpu.h -- C ABI of the B200 PageRank engine (libnwgpu.so).
 *
 * This is the drop-in boundary for NWGraph's PageRank hot path. It replaces
 *
 *   template <adjacency_list_graph Graph, typename Real>
 *   void nw::graph::page_rank(const Graph& graph,
 *                             const std::vector<vertex_id_type>& degrees,
 *                             std::vector<Real>& page_rank,
 *                             Real damping_factor, Real threshold,
 *                             size_t max_iters, size_t num_threads);
 *     include/nwgraph/algorithms/page_rank.hpp:89-91 (v11)
 *     include/nwgraph/experimental/algorithms/page_rank.hpp:377-379 (v10, same signature)
 *
 * with a graph handle (the CSR uploaded once) and a solve call carrying the
 * same parameters. The C++20 layer in include/nwgraph_gpu/page_rank.hpp keeps
 * the reference's exact call surface on top of these functions.
 *
 * Conventions
 *  - Every function returns an int status (NWGPU_OK == 0); none throws or
 *    aborts. nwgpu_last_error() returns the calling thread's last message.
 *  - The CSR is NWGraph's adjacency<1> (include/nwgraph/adjacency.hpp:86-195):
 *    row_ptr = indices_ (n+1 uint32), col = std::get<0>(to_be_indexed_)
 *    (nnz uint32); row i lists the in-neighbours j of i (edge j -> i).
 *    uint32 indices as default_index_t (include/nwgraph/util/defaults.hpp:23-24).
 *  - out_degree[j] is the out-degree of j, as the benchmark's build_degrees
 *    computes it (bench/gapbs/common.hpp:110-121).
 *  - A handle owns one CUDA stream; calls on one handle are serialised by the
 *    caller, calls on distinct handles may run concurrently.
 *  - Device memory of handles comes from one stream-ordered pool per device
 *    that keeps freed blocks mapped: creating and destroying handles again
 *    and again does not map and unmap pages each time.
 *    nwgpu_release_cached_memory() returns the unused blocks to the driver.
 *  - There is no CPU fallback: without a usable sm_100 device every call that
 *    needs one returns NWGPU_ERR_CUDA / NWGPU_ERR_NO_DEVICE.
 */
#ifndef NWGPU_H
#define NWGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NWGPU_ABI_VERSION 2

enum nwgpu_status {
  NWGPU_OK = 0,
  NWGPU_ERR_INVALID_ARG = 1,   /* null pointer, bad size, damping outside [0,1], ... */
  NWGPU_ERR_INVALID_GRAPH = 2, /* row_ptr not monotone, row_ptr[n] != nnz, col[k] >= n */
  NWGPU_ERR_CUDA = 3,          /* a CUDA runtime call failed (message has the CUDA error) */
  NWGPU_ERR_OUT_OF_MEMORY = 4,
  NWGPU_ERR_ABORTED = 5,       /* nwgpu_abort() was called while the solve ran */
  NWGPU_ERR_NO_DEVICE = 6,     /* no CUDA device, or not compute capability 10.x */
  NWGPU_ERR_UNSUPPORTED = 7
};

typedef struct nwgpu_graph nwgpu_graph;

/* nwgpu_graph_create flags */
#define NWGPU_GRAPH_DEVICE_PTRS 0x1u /* row_ptr / col / weights are device pointers (copied device-to-device) */
#define NWGPU_GRAPH_TRANSPOSE 0x2u   /* build the out-row CSR (adjacency<0>) of nwgpu_pr_vjp at creation, not on first use */
#define NWGPU_GRAPH_NO_RELABEL 0x4u  /* keep the input vertex order on the device (default: hubs first) */
#define NWGPU_GRAPH_AUTOTUNE 0x8u    /* pick the sweep's long-row cut-offs, launch shape and hub tiers by
                                        timing a few sweeps of each candidate (or reuse the choice cached for
                                        graphs of the same signature; NWGPU_TUNE_CACHE=<file> keeps the cache
                                        across processes). Launch shape and hub tiers give bitwise-equal ranks;
                                        the cut-offs and bin-0 rows per warp (reported by nwgpu_graph_get_info)
                                        set how rows are summed. Also set by NWGPU_AUTOTUNE=1 */

/* Upload a CSR once (replaces the per-call use of graph.indices_ /
 * to_be_indexed_ at page_rank.hpp:129). Validates it on the device
 * (monotone row_ptr, row_ptr[0] == 0, row_ptr[n] == nnz, every col < n),
 * renumbers vertices by descending out-degree unless NWGPU_GRAPH_NO_RELABEL
 * (each row keeps its entries in input order, so its sum has the same terms in
 * the same order; results are returned in input order) and partitions it into
 * equal-work merge-path tiles. weights may be NULL
 * (unweighted); with weights the graph can also run weighted PageRank and its
 * adjoint. Uses the current CUDA device. n must be below 2^32 - 16 and nnz at
 * most 2^32 - 512 (the reference's uint32 row pointers allow 2^32 - 1; the
 * sweep forms entry indices up to 255 past a row's end in 32 bits). */
int nwgpu_graph_create(const uint32_t* row_ptr, const uint32_t* col, const float* weights, uint64_t n, uint64_t nnz,
                       uint32_t flags, nwgpu_graph** out);
int nwgpu_graph_destroy(nwgpu_graph* g);

typedef struct nwgpu_graph_info {
  uint64_t n, nnz;
  uint64_t num_tiles;    /* merge-path tiles of one sweep */
  uint32_t tile_items;   /* rows + entries per tile */
  uint32_t grid;         /* persistent CTAs per sweep */
  uint64_t device_bytes; /* HBM held by the handle */
  int32_t  device;
  int32_t  has_weights, has_transpose;
  int32_t  binned;         /* 1: the degree-binned sweep (relabelled graphs); 0: merge-path tiles */
  uint32_t sweep_threads;  /* threads per CTA of the sweep */
  uint32_t sweep_grid;     /* CTAs of the sweep */
  uint32_t hub_smem_ids;   /* binned: contributions [0, hub_smem_ids) staged in shared memory each sweep */
  uint32_t hub_l1_ids;     /* binned: ids [hub_smem_ids, hub_l1_ids) gathered through L1 */
  int32_t  tuned;          /* 0 defaults, 1 timed at creation, 2 taken from the tuning cache */
  float    tuned_us_per_sweep;
  int32_t  blocked;        /* 1: plain solves run the destination-blocked sweep (exact fixed-point row sums) */
  uint32_t block_count;    /* blocked: destination blocks of 28,672 rows */
  uint32_t block_items;    /* blocked: work items per sweep (blocks, the large ones cut into pieces) */
  uint32_t block_loads;    /* blocked: entries in flight per thread */
  uint64_t block_piece_entries; /* blocked: the largest work item */
  uint32_t long_row_entries;    /* binned: rows longer than this are cut into chunks */
  uint32_t chunk_entries;       /* binned: entries per long-row chunk */
  uint32_t bin0_rows_per_warp;  /* binned: rows of 129 entries to the long-row cut-off per warp: 2 (half a warp
                                   each) or 1 (a whole warp); like the cut-offs it sets the rows' summation order */
} nwgpu_graph_info;
int nwgpu_graph_get_info(const nwgpu_graph* g, nwgpu_graph_info* info);

/* Solve modes */
#define NWGPU_MODE_PARITY 0u     /* page_rank_v10 semantics: Jacobi, leak (no dangling redistribution) */
/* Launch strategies */
#define NWGPU_LAUNCH_GRAPH 0u    /* CUDA graph; device-side while loop, convergence tested on the GPU */
#define NWGPU_LAUNCH_STREAM 1u   /* one kernel per sweep on the stream; sweeps after convergence exit at once */

typedef struct nwgpu_pr_options {
  uint32_t size;        /* sizeof(nwgpu_pr_options); 0 fields mean defaults */
  uint32_t mode;        /* NWGPU_MODE_* */
  uint32_t launch;      /* NWGPU_LAUNCH_* */
  uint32_t device_ptrs; /* 1: degrees / ranks / vectors are device pointers */
  uint32_t reserved0;
  void*    stream;      /* cudaStream_t to run the solve on; NULL = the handle's own stream */
  uint32_t reserved[2];
} nwgpu_pr_options;

typedef struct nwgpu_pr_stats {
  uint64_t iterations;     /* sweeps run, counting the one whose error fell below threshold */
  double   final_error;    /* L1 change of the last sweep (FP64, as page_rank.hpp:125-134) */
  int32_t  converged;      /* final_error < threshold */
  double   device_ms;      /* CUDA-event time of the sweep loop */
  double   ms_per_iter;
  double   bytes_per_iter; /* algorithmic bytes of one sweep: 4 nnz + 4 (n+1) + 20 n */
  double   gteps;          /* nnz * iterations / device time */
  double*  errors;         /* optional, caller-owned: errors[i] = L1 change of sweep i, for the first
                              min(iterations, errors_cap, 4096) sweeps (later sweeps are not recorded) */
  uint64_t errors_cap;     /* capacity of errors[] */
} nwgpu_pr_stats;

/* PageRank over the uploaded graph: the body of page_rank / page_rank_v10
 * (page_rank.hpp:92-147). ranks[n] is fully overwritten; damping, threshold
 * and max_iters mean what they mean there (stop after the first sweep whose
 * FP64 L1 change is < threshold, at most max_iters sweeps). out_degree[n] and
 * ranks[n] are host pointers unless options->device_ptrs. */
int nwgpu_pr_run(nwgpu_graph* g, const uint32_t* out_degree, float* ranks, float damping, float threshold,
                 uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats);

/* Residual-push PageRank: page_rank_v13 (experimental/algorithms/page_rank.hpp:
 * 552-625). Ranks start at 0 and every residual at (float)(1 - d). Each
 * iteration pushes every residual above `threshold` into its vertex's rank
 * and, for out-degree > 0, spreads residual * d / deg to the out-neighbours
 * (FP32); each vertex's next residual is the sum of what it received. It stops
 * after the first iteration in which no vertex with out-degree > 0 pushed, or
 * after max_iters. The ranks are the reference's: not normalised (they sum to
 * about n). stats->errors[i] / final_error count the vertices that pushed in
 * iteration i / the last one; converged = no push in the last iteration.
 * Needs a relabelled graph (the default). Sums run in the kernel's fixed
 * order, not the reference's serial one. */
int nwgpu_pr_residual_run(nwgpu_graph* g, const uint32_t* out_degree, float* ranks, float damping, float threshold,
                          uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats);

/* Personalised PageRank with a one-hot teleport at `seed` (input vertex id):
 *   r = (1 - d) e_seed + d A^T D^{-1} r,  r(0) = e_seed,
 * the plain update of page_rank.hpp:133 with base_i = (1 - d) [i == seed];
 * same stopping rule, leak semantics and argument conventions as nwgpu_pr_run.
 * No counterpart in the reference (personalised PageRank is an extension). */
int nwgpu_ppr_run(nwgpu_graph* g, const uint32_t* out_degree, uint32_t seed, float* ranks, float damping,
                  float threshold, uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats);

typedef struct nwgpu_ppr_stats {
  uint64_t  iterations;     /* sweeps run (the slowest column) */
  int32_t   all_converged;  /* every column met the threshold */
  double    device_ms;      /* CUDA-event time of the sweep loop */
  double    ms_per_iter;
  double    bytes_per_iter; /* 4 nnz + 4 (n+1) + 4 n + 16 k n */
  uint32_t* col_iterations; /* optional, caller-owned [k]: sweeps until column c stopped */
  double*   col_errors;     /* optional, caller-owned [k]: L1 change of column c's last sweep */
  int32_t*  col_converged;  /* optional, caller-owned [k] */
} nwgpu_ppr_stats;

/* k personalised vectors solved together (k <= 128): seeds[k] are input
 * vertex ids, ranks_nxk is an n x k row-major FP32 matrix in input vertex
 * order (column c = the vector of seeds[c]). Each column stops at its own
 * first sweep whose FP64 L1 change is < threshold (its values then stay
 * fixed) or at max_iters. One column-index load feeds all k gathers.
 * No counterpart in the reference. */
int nwgpu_ppr_batched(nwgpu_graph* g, const uint32_t* out_degree, const uint32_t* seeds, uint32_t k, float* ranks_nxk,
                      float damping, float threshold, uint64_t max_iters, const nwgpu_pr_options* options,
                      nwgpu_ppr_stats* stats);

/* Weighted personalised PageRank for k <= 128 teleport vectors at once (no
 * counterpart in the reference): column c solves nwgpu_wpr_run's problem
 *   r_c = (1 - d) t_c + d sum_k w_k r_c[col[k]] / s_{col[k]},  r_c(0) = t_c
 * with teleports[n x k] (row-major, input order) and writes ranks_nxk
 * (row-major, input order). One index and weight load feeds all k gathers;
 * each column stops at its own first sweep whose FP64 L1 change is below
 * threshold (its values then stay fixed) or at max_iters. The graph must carry
 * weights and be relabelled (the default). Arrays are host pointers unless
 * options->device_ptrs. */
int nwgpu_wppr_batched(nwgpu_graph* g, const float* teleports, uint32_t k, float* ranks_nxk, float damping,
                       float threshold, uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_ppr_stats* stats);

/* The teleport-matrix form of nwgpu_ppr_batched, for unweighted graphs (no
 * counterpart in the reference): column c solves
 *   r_c = (1 - d) t_c + d A^T D^{-1} r_c,  r_c(0) = t_c,
 * with teleports[n x k] (row-major, input order) and the caller's out-degrees
 * (D, as in nwgpu_pr_run), and writes ranks_nxk (row-major, input order). A
 * one-hot column t_c = e_s gives exactly nwgpu_ppr_batched's column for seed s.
 * Stopping rule, k <= 128 and argument conventions as nwgpu_ppr_batched. */
int nwgpu_ppr_batched_teleports(nwgpu_graph* g, const uint32_t* out_degree, const float* teleports, uint32_t k,
                                float* ranks_nxk, float damping, float threshold, uint64_t max_iters,
                                const nwgpu_pr_options* options, nwgpu_ppr_stats* stats);

/* PageRank without any allocation. No counterpart in the reference.
 *
 * For callers that must not allocate:
 *  - code running under a memory manager that owns the device's memory (an
 *    application pool, a process with a fixed memory cap), where a cudaMalloc
 *    from a library would fail or break the owner's accounting;
 *  - callers on a latency path, where cudaMalloc / cudaFree could synchronise
 *    the device.
 * The call allocates nothing on the device or the host. The caller passes the
 * CSR, the degrees and the output, all in device memory. The engine's own
 * working memory lives in one statically sized device array inside this
 * library (about 8.8 MB, present on every device once the library's kernels
 * are loaded). That array bounds the graph:
 *   n   <= NWGPU_NOALLOC_MAX_VERTICES,  nnz <= NWGPU_NOALLOC_MAX_ENTRIES.
 * Larger graphs, and pointers that are not 16-byte-aligned device memory, are
 * rejected with NWGPU_ERR_INVALID_ARG and a message naming the limit.
 *
 * Semantics are those of nwgpu_pr_run with NWGPU_GRAPH_NO_RELABEL and
 * NWGPU_LAUNCH_STREAM:
 *  - the same sweep, stopping rule and stats;
 *  - device_ms is host time around the sweep loop;
 *  - the CSR is validated on each call.
 * `stream` is a cudaStream_t (NULL = the default stream). The call returns
 * when the solve has finished.
 *
 * The arrays are read exactly within their lengths (row_ptr n + 1, col nnz,
 * out_degree and ranks n elements): an array may end at the very end of its
 * allocation.
 *
 * The first call on a device looks up that device's copy of the array. Make
 * that first call before any stream capture on the device. Under CUDA's lazy
 * module loading (the default), the library's kernels and this array are
 * loaded on a device at its first use: a caller whose memory manager will
 * take all of the device's memory should make one call (a warm-up solve on a
 * tiny graph) before that, so the array is already resident. The working array
 * is shared by every call on a device: calls whose GPU work overlaps (from two
 * host threads, or on two streams at once) race, and both results are
 * undefined. Serialise them. */
#define NWGPU_NOALLOC_MAX_VERTICES 1048576u
#define NWGPU_NOALLOC_MAX_ENTRIES 33554432u
int nwgpu_pr_run_noalloc(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, uint64_t nnz,
                         const uint32_t* out_degree, float* ranks, float damping, float threshold, uint64_t max_iters,
                         void* stream, nwgpu_pr_stats* stats);

/* Weighted PageRank (no counterpart in the reference, whose page_rank is
 * unweighted). g must carry edge weights (nwgpu_graph_create's `weights`,
 * w_k > 0 for the edge col[k] -> row of k) and be relabelled (the default).
 * With s_j the out-weight sum of j:
 *   r_i = (1 - d) t_i + d sum_{k in row i} w_k r_{col[k]} / s_{col[k]},  r(0) = t
 * teleport[n] (input order) is a distribution over the vertices; NULL means
 * uniform 1/n. The update, stopping rule (FP64 L1 change < threshold), leak
 * semantics and argument conventions are nwgpu_pr_run's. */
int nwgpu_wpr_run(nwgpu_graph* g, const float* teleport, float* ranks, float damping, float threshold, uint64_t max_iters,
                  const nwgpu_pr_options* options, nwgpu_pr_stats* stats);

/* Vector-Jacobian product of the weighted PageRank fixed point (no
 * counterpart in the reference). For L = sum_v dL_dr[v] r_v, with ranks[n]
 * the converged output of nwgpu_wpr_run (same damping), it solves the adjoint
 *   l_j = dL_dr_j + d sum_{k: col[k] = j} (w_k / s_j) l_{row(k)}
 * by implicit differentiation, with the same sweep over the out-row CSR (no
 * forward iterates are stored), to an FP64 L1 change < threshold, then writes
 *   dL_dt[v] = (1 - d) l_v                                (n, may be NULL)
 *   dL_dw[k] = d r_j / s_j (l_i - q_j),  q_j = (l_j - dL_dr_j) / d
 * for entry k of row i with col[k] = j, in the input entry order (nnz, may be
 * NULL). stats describe the adjoint solve. The out-rows must be in the
 * relabelled length order, which holds for symmetric graphs; otherwise
 * NWGPU_ERR_UNSUPPORTED. */
int nwgpu_pr_vjp(nwgpu_graph* g, const float* ranks, const float* dL_dr, float* dL_dw, float* dL_dt, float damping,
                 float threshold, uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats);

/* Weighted sparse matrix-vector product over the graph's rows:
 *   y[i] = sum over the entries k of row i of weights[k] * x[col[k]]
 * (bench/abstraction_penalty/spmv.cpp:52-62, the reference's SpMV kernel
 * `y[i] += x[idx[j]] * dat[j]` from y = 0), as one sweep of the weighted
 * PageRank kernel. x[n] and y[n] are in input order, host pointers unless
 * options->device_ptrs. The graph must carry weights and be relabelled (the
 * default); otherwise NWGPU_ERR_UNSUPPORTED. Row sums are FP32 in the
 * kernel's fixed order, not the reference's serial order. */
int nwgpu_spmv(nwgpu_graph* g, const float* x, float* y, const nwgpu_pr_options* options);

/* Ask a running solve on g to stop at its next sweep boundary; the solve
 * returns NWGPU_ERR_ABORTED. Safe to call from another host thread. */
int nwgpu_abort(nwgpu_graph* g);

/* Self-test of the engine's bounded device waits (no counterpart in the
 * reference). The sweeps wait on shared-memory barriers for their bulk copies
 * and give up after 2^20 polls, recording a fault that ends the solve with
 * NWGPU_ERR_CUDA instead of hanging. This runs that same wait loop, with
 * `polls` polls (1 .. 2^20), in one thread on a barrier that nothing ever
 * completes: *gave_up is 1 when the wait gave up as it should, and *ms is how
 * long that took. Nothing faults; the context stays usable. */
int nwgpu_selftest_bounded_wait(uint32_t polls, uint32_t* gave_up, double* ms);

/* ---- Graph construction on the device ------------------------------------
 * CSR from an edge list (src[e] -> dst[e], m edges over n vertices): the
 * reference's remove_self_loops (build.hpp:404-410), uniq (:394-402) and
 * fill_directed / fill_undirected (:209-272), in that order, as flags, on
 * the device. Rows
 * are indexed by target (adjacency<1>, row v lists the sources of edges into
 * v) unless NWGPU_EDGES_BY_SOURCE (adjacency<0>); entries of a row come out
 * sorted ascending, as with fill(..., sort_adjacency = true). Writes
 * row_ptr[n + 1], col[nnz] (col_capacity must be >= nnz; otherwise
 * NWGPU_ERR_INVALID_ARG with *nnz set) and, when degrees is not NULL,
 * degrees[n] = the number of entries whose column is v (the out-degree the
 * bench's build_degrees computes for an adjacency<1>, common.hpp:110-121).
 * Arrays are host pointers unless NWGPU_EDGES_DEVICE_PTRS. stream: a
 * cudaStream_t, NULL for the default stream; the call returns when done. */
#define NWGPU_EDGES_DEVICE_PTRS 0x1u       /* src, dst and the outputs are device pointers */
#define NWGPU_EDGES_BY_SOURCE 0x2u         /* rows indexed by source (adjacency<0>) */
#define NWGPU_EDGES_UNDIRECTED 0x4u        /* fill_undirected: every edge in both directions */
#define NWGPU_EDGES_REMOVE_SELF_LOOPS 0x8u /* remove_self_loops */
#define NWGPU_EDGES_UNIQUE 0x10u           /* uniq on the edge list: each (src, dst) pair once, before fill */
#define NWGPU_EDGES_UNIQUE_ENTRIES 0x20u   /* one entry per (row, col) of the result (simple graph; not a
                                              reference step: with UNDIRECTED, (u, v) and (v, u) both listed
                                              otherwise give two entries per row, as in fill_undirected) */
int nwgpu_csr_from_edges(const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n, uint32_t flags,
                         uint32_t* row_ptr, uint32_t* col, uint64_t col_capacity, uint64_t* nnz, uint32_t* degrees,
                         void* stream);

/* Graph files: the reference driver's load_graph (bench/gapbs/common.hpp:83-100)
 * reads a serialized NW edge list (edge_list.hpp:237-280) or a Matrix Market
 * coordinate file through read_mm<directed> (io/mmio.hpp:86-103, 171-208).
 * These read both on all host cores into the same edge list, in the same
 * order (Matrix Market: entry (i, j) gives edge (i-1, j-1), and symmetric
 * files add (j-1, i-1) for i != j; only general / symmetric coordinate files,
 * as read_mm). Build the CSR with nwgpu_csr_from_edges (no flags: the
 * reference driver's adjacency<1>). Host code only: no device is needed.
 * probe: the format, vertex count, an upper bound on the edges (capacity for
 * read) and whether the file holds values. read: src/dst[capacity] and, if
 * not NULL, values[capacity] (1.0 for pattern files); *m = edges read;
 * nthreads <= 0 uses every core. write_nw: the NW edge-list layout that
 * edge_list::deserialize reads (sources and targets, no attributes). */
#define NWGPU_FILE_MATRIX_MARKET 1
#define NWGPU_FILE_NW_EDGE_LIST 2
#define NWGPU_FILE_NW_ADJACENCY 3  /* a serialized adjacency<idx> (adjacency.hpp:176-191): a CSR; see below */
typedef struct nwgpu_edge_file {
  int32_t  format;     /* NWGPU_FILE_* */
  int32_t  directed;   /* NW: the directedness written in the file; Matrix Market: 1 */
  int32_t  has_values;
  uint64_t n;          /* vertices */
  uint64_t max_edges;  /* edges the file can yield (capacity for nwgpu_edge_file_read) */
} nwgpu_edge_file;
int nwgpu_edge_file_probe(const char* path, nwgpu_edge_file* info);
int nwgpu_edge_file_read(const char* path, uint32_t* src, uint32_t* dst, float* values, uint64_t capacity,
                         uint64_t* m, int nthreads);
int nwgpu_edge_file_write_nw(const char* path, const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n,
                             int directed);
/* A serialized adjacency<idx> (index_adjacency::serialize, adjacency.hpp:
 * 176-191 over compressed.hpp:377-413) read as its CSR: row_ptr[n + 1], col[nnz]
 * and, if not NULL, values[nnz] (its first attribute, 1.0 without one). With
 * row_ptr NULL only *n and *nnz are set. Host code only. */
int nwgpu_adjacency_file_read(const char* path, uint32_t* row_ptr, uint32_t* col, float* values, uint64_t n_cap,
                              uint64_t nnz_cap, uint64_t* n, uint64_t* nnz);

/* Seeded RMAT edge list on the device (no counterpart in the reference, which
 * ships no generator): m samples over 2^scale ids, each descending `scale`
 * levels with quadrant probabilities a, b, c (d = 1 - a - b - c) drawn from a
 * counter-based hash of (seed, sample, level); the same samples as the host
 * builder nwgen_rmat (include/nwgraph_gen.h). With 0 < n < 2^scale the ids
 * are taken modulo n. src[m], dst[m] are device pointers. Asynchronous on
 * stream. */
int nwgpu_rmat_edges(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed, uint64_t n, uint32_t* src,
                     uint32_t* dst, void* stream);

/* The side x side 4-neighbour grid as 2 side (side - 1) undirected edges
 * (horizontal (v, v+1) first, then vertical (v, v+side)); device pointers,
 * asynchronous on stream. Built with NWGPU_EDGES_UNDIRECTED it equals
 * nwgen_grid(side * side). */
int nwgpu_grid_edges(uint64_t side, uint32_t* src, uint32_t* dst, void* stream);

/* ---- Row-sharded PageRank across GPUs (one shard per rank) --------------
 * The sweep of page_rank.hpp:92-147 split by destination rows over `world`
 * ranks, one GPU each. Every rank passes the whole graph; it is relabelled
 * the same way on every rank (descending row length, stably) and rank q
 * keeps the internal rows [bounds[q], bounds[q+1]). Contributions live in a
 * padded layout of world * stride floats, rank q's rows at q * stride, so
 * one equal-count all-gather of the ranks' slices (stride floats each)
 * rebuilds the whole vector between sweeps. The caller runs that exchange and
 * the sum of the ranks' FP64 L1 changes (nwgraph_b200/shard.py does it over
 * NCCL through torch.distributed); nwgpu_shard_decide takes the stopping
 * decision from that sum on the device. bounds[world+1]
 * (host) must run from 0 to n, stride be a multiple of 4 and at least every
 * rank's row count; every rank passes the same bounds and stride.
 * All vectors below are device pointers; stream is a cudaStream_t, NULL
 * meaning the CUDA default stream (as torch's default stream is). */
typedef struct nwgpu_shard nwgpu_shard;
int nwgpu_shard_create(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, uint64_t nnz, uint32_t world,
                       uint32_t rank, const uint64_t* bounds, uint64_t stride, uint32_t flags, nwgpu_shard** out);
int nwgpu_shard_destroy(nwgpu_shard* s);
/* ranks of this rank's rows = 1/n; their contributions rank / out_degree into
 * contrib_slice[stride]. out_degree[n] is in input order (host unless
 * device_ptrs). */
int nwgpu_shard_start(nwgpu_shard* s, const uint32_t* out_degree, int device_ptrs, float* contrib_slice, void* stream);
/* One Jacobi sweep of this rank's rows from contrib_all[world * stride] (the
 * gathered slices): new ranks kept in the shard, new contributions into
 * contrib_slice, and the FP64 L1 change of these rows into *l1 (one double,
 * device; NaN if a bounded device wait gave up). */
int nwgpu_shard_sweep(nwgpu_shard* s, const float* contrib_all, float* contrib_slice, float damping, double* l1,
                      void* stream);
/* The stopping decision of the sweep just run, taken on the device from
 * *l1_total (the ranks' summed L1 changes, device; every rank passes the same
 * value) so the host need not read it back each sweep: stop after the first
 * sweep whose total is < threshold (page_rank.hpp:144), after max_iters
 * sweeps, or on a NaN total. Once stopped, the shard's later sweeps return
 * at once and change nothing (their *l1 repeats the last change), so a caller
 * may queue several sweeps, each with its exchange and decision, and read
 * state back once per batch. state[4] (device, zeroed by the caller before
 * the first sweep) = {sweeps decided, stopped, converged, failed};
 * errors[k] (device, may be NULL) receives the total of sweep k < errors_cap. */
int nwgpu_shard_decide(nwgpu_shard* s, const double* l1_total, double threshold, uint64_t max_iters, uint64_t* state,
                       double* errors, uint64_t errors_cap, void* stream);
/* This rank's ranks into rank_slice[stride]; after the caller gathers every
 * slice into ranks_all[world * stride], nwgpu_shard_unpermute writes the
 * ranks in input order into ranks[n]. */
int nwgpu_shard_rank_slice(nwgpu_shard* s, float* rank_slice, void* stream);
int nwgpu_shard_unpermute(nwgpu_shard* s, const float* ranks_all, float* ranks, void* stream);

/* ---- Ragged batches: many independent graphs in one solve ----------------
 * No counterpart in the reference: each graph's result is what page_rank
 * (page_rank.hpp:92-147) gives for that graph alone, and each graph stops at
 * its own first sweep whose FP64 L1 change is < threshold (or max_iters);
 * graphs that stopped are skipped by later sweeps.
 *
 * Graph g (0 <= g < num_graphs) has n_g = vertex_offsets[g+1] -
 * vertex_offsets[g] vertices and nnz_g = entry_offsets[g+1] - entry_offsets[g]
 * entries, as a CSR with local ids: its n_g + 1 row pointers (local entry
 * offsets, first 0, last nnz_g) are row_ptr[vertex_offsets[g] + g ...], its
 * column ids (local vertex ids < n_g) are col[entry_offsets[g] ...]. So
 * row_ptr holds vertex_offsets[num_graphs] + num_graphs words and col
 * entry_offsets[num_graphs]. vertex_offsets / entry_offsets are host arrays
 * of num_graphs + 1 non-decreasing values starting at 0; row_ptr / col are
 * host pointers unless flags has NWGPU_GRAPH_DEVICE_PTRS. Per graph n_g and
 * nnz_g must be below 2^32 - 16, and a graph solved alone (below) at most
 * 2^32 - 512 entries, as for nwgpu_graph_create; the batch totals are 64-bit.
 *
 * Graphs with at least 2^22 entries (the environment variable
 * NWGPU_RAGGED_SOLO_ENTRIES, read here, sets the bound; 0 keeps every graph in
 * the batch) get a single-graph handle of their own (as nwgpu_graph_create)
 * and are solved by it, beside the batch's sweep loop: for them that engine is
 * faster. A graph's result therefore depends only on the graph, not on the
 * batch it is in. */
typedef struct nwgpu_batch nwgpu_batch;
int nwgpu_batch_create(uint64_t num_graphs, const uint64_t* vertex_offsets, const uint64_t* entry_offsets,
                       const uint32_t* row_ptr, const uint32_t* col, uint32_t flags, nwgpu_batch** out);
int nwgpu_batch_destroy(nwgpu_batch* b);

typedef struct nwgpu_batch_stats {
  uint64_t  sweeps;           /* sweeps of the last graph to stop (graphs solved alone included) */
  uint64_t  converged_graphs; /* graphs whose last L1 change was < threshold */
  double    device_ms;        /* CUDA-event time of the sweep loop and the graphs solved alone */
  double    entries_swept;    /* sum over graphs of nnz_g x the graph's sweeps */
  double    gteps;            /* entries_swept / device time */
  uint32_t* graph_iterations; /* optional, caller-owned [num_graphs]: sweeps until graph g stopped */
  double*   graph_errors;     /* optional [num_graphs]: L1 change of graph g's last sweep */
  int32_t*  graph_converged;  /* optional [num_graphs] */
} nwgpu_batch_stats;

/* PageRank of every graph of the batch. out_degree and ranks hold
 * vertex_offsets[num_graphs] values, graph g's at vertex_offsets[g] (local
 * vertex order); host pointers unless options->device_ptrs. damping,
 * threshold and max_iters apply to every graph, with nwgpu_pr_run's meaning
 * and update. A graph with no vertices has error 0 at every sweep. */
int nwgpu_pr_ragged(nwgpu_batch* b, const uint32_t* out_degree, float* ranks, float damping, float threshold,
                    uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_batch_stats* stats);

/* Return the device memory that destroyed handles left in the pool to the
 * driver (all devices), and unpin the small host blocks they cached for their
 * solve states. Handles still alive keep theirs. */
int nwgpu_release_cached_memory(void);

/* Thread-local message for the last failing call (empty if none). Returns
 * the message length. */
int nwgpu_last_error(char* buf, size_t len);

int nwgpu_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NWGPU_H */
