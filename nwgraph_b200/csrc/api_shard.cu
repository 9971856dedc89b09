// C ABI: one rank's shard of a row-sharded PageRank solve (nwgpu_shard_*,
// include/nwgpu.h).
//
// The reference solves on one host (page_rank.hpp:89-148). Across GPUs the
// sweep shards by destination rows: every rank relabels the whole graph the
// same way (descending row length, stably), owns the internal rows
// [bounds[rank], bounds[rank + 1]), and needs the whole contribution vector
// each sweep. The contributions live in a padded layout of world * stride
// floats, rank q's rows at [q * stride, q * stride + rows_q), so one
// equal-count all-gather of every rank's slice rebuilds the whole vector; the
// shard's column ids are remapped to that layout once, at creation. The hub
// rows (the smallest internal ids) belong to rank 0, so they keep positions
// [0, 32768) and the binned sweep still stages them in shared memory.
//
// This file holds the per-rank building blocks (start, one sweep, the rank
// slice, the final unpermute); the exchange between sweeps (the all-gather of
// the slices and the sum of the ranks' FP64 L1 changes) belongs to the caller,
// which runs it over NCCL through torch.distributed (nwgraph_b200/shard.py).
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "handle.h"

namespace nwgpu {
namespace {

// Position of internal id u in the padded layout.
__device__ __forceinline__ uint32_t padded_pos(uint32_t u, const uint64_t* __restrict__ bounds, uint32_t world,
                                               uint64_t stride) {
  uint32_t lo = 0, hi = world - 1;  // last rank whose first row is <= u
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (bounds[mid] <= u)
      lo = mid;
    else
      hi = mid - 1;
  }
  return (uint32_t)((uint64_t)lo * stride + (u - bounds[lo]));
}

// Local CSR of rows [r0, r1): row pointers rebased, column ids mapped to the padded layout.
__global__ void shard_rows_kernel(const uint32_t* __restrict__ rp, uint64_t r0, uint64_t r1,
                                  uint32_t* __restrict__ lrp) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t base = rp[r0];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= r1 - r0; i += stride) lrp[i] = rp[r0 + i] - base;
}
__global__ void shard_cols_kernel(const uint32_t* __restrict__ col, uint64_t k0, uint64_t m,
                                  const uint64_t* __restrict__ bounds, uint32_t world, uint64_t pstride,
                                  uint32_t* __restrict__ lcol) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride)
    lcol[k] = padded_pos(col[k0 + k], bounds, world, pstride);
}
// ranks[v] = all[pos(perm[v])] (input order from the padded layout)
__global__ void shard_unpermute_kernel(const float* __restrict__ all, const uint32_t* __restrict__ perm, uint64_t n,
                                       const uint64_t* __restrict__ bounds, uint32_t world, uint64_t pstride,
                                       float* __restrict__ ranks) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    ranks[v] = all[padded_pos(perm[v], bounds, world, pstride)];
}
// The sweep's L1 change of this rank's rows, or NaN after a failed bounded wait.
__global__ void shard_err_kernel(const PrState* __restrict__ st, double* __restrict__ out) {
  *out = st->fault ? __longlong_as_double(0x7ff8000000000000ll) : st->last_error;
}

// The stopping decision of one sweep, on the device, from the ranks' summed
// L1 change `total` (page_rank.hpp:144): after the first sweep whose total is
// below the threshold, or max_iters sweeps, or a NaN total (a rank's bounded
// wait gave up), the shard's state is marked done, so its later sweep
// launches return at once and leave ranks and contributions as they are.
// state[4] = {sweeps decided, done, converged, failed}; hist[k] = total of sweep k (k < hist_cap).
__global__ void shard_decide_kernel(PrState* __restrict__ st, const double* __restrict__ total, double threshold,
                                    unsigned long long max_iters, unsigned long long* __restrict__ state,
                                    double* __restrict__ hist, unsigned long long hist_cap) {
  if (state[1]) return;
  const double             e = *total;
  const unsigned long long k = state[0];
  if (hist && k < hist_cap) hist[k] = e;
  const bool failed = !(e == e);
  const bool conv = !failed && e < threshold;
  state[0] = k + 1;
  if (conv || failed || k + 1 >= max_iters) {
    state[1] = 1ull;
    state[2] = conv ? 1ull : 0ull;
    state[3] = failed ? 1ull : 0ull;
    st->done = 1u;
  }
}

}  // namespace
}  // namespace nwgpu

struct nwgpu_shard {
  nwgpu_graph*          inner = nullptr;  // the local rows as a graph (binned plan, solve buffers)
  uint64_t              n = 0, nnz = 0;   // the whole graph
  uint32_t              world = 1, rank = 0;
  uint64_t              row0 = 0, rows = 0, stride = 0;
  std::vector<uint64_t> bounds;
  uint64_t*             d_bounds = nullptr;
  uint32_t*             perm = nullptr;      // input id -> internal id (whole graph)
  uint32_t*             inv_local = nullptr; // local row -> input id
  uint32_t*             deg_stage = nullptr; // out-degrees staged from host
  uint64_t              sweeps = 0;
  ~nwgpu_shard() {
    if (inner) {
      cudaStream_t s = inner->stream;
      nwgpu::pool_free(d_bounds, s);
      nwgpu::pool_free(perm, s);
      nwgpu::pool_free(inv_local, s);
      nwgpu::pool_free(deg_stage, s);
      cudaStreamSynchronize(s);
      delete inner;
    }
  }
};

using namespace nwgpu;

extern "C" {

int nwgpu_shard_create(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, uint64_t nnz, uint32_t world,
                       uint32_t rank, const uint64_t* bounds, uint64_t stride, uint32_t flags, nwgpu_shard** out) {
  clear_error();
  if (!out) return fail(NWGPU_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!row_ptr || (nnz && !col) || !bounds) return fail(NWGPU_ERR_INVALID_ARG, "row_ptr / col / bounds is NULL");
  if (world == 0 || rank >= world) return fail(NWGPU_ERR_INVALID_ARG, "rank %u of world %u", rank, world);
  if (n < 2 || n >= 0xFFFFFFF0ull || nnz > kMaxEntries)
    return fail(NWGPU_ERR_INVALID_ARG, "n = %llu, nnz = %llu: a shard needs 2 <= n < 2^32 - 16 and nnz <= 2^32 - 512",
                (unsigned long long)n, (unsigned long long)nnz);
  if (bounds[0] != 0 || bounds[world] != n)
    return fail(NWGPU_ERR_INVALID_ARG, "bounds must run from 0 to n = %llu", (unsigned long long)n);
  for (uint32_t q = 0; q < world; ++q) {
    if (bounds[q + 1] < bounds[q]) return fail(NWGPU_ERR_INVALID_ARG, "bounds decrease at rank %u", q);
    if (bounds[q + 1] - bounds[q] > stride)
      return fail(NWGPU_ERR_INVALID_ARG, "rank %u has %llu rows, more than the stride %llu", q,
                  (unsigned long long)(bounds[q + 1] - bounds[q]), (unsigned long long)stride);
  }
  if (stride % 4 || (uint64_t)world * stride >= 0xFFFFFFF0ull)
    return fail(NWGPU_ERR_INVALID_ARG, "stride %llu: must be a multiple of 4 with world * stride < 2^32 - 16",
                (unsigned long long)stride);
  if (flags & ~NWGPU_GRAPH_DEVICE_PTRS) return fail(NWGPU_ERR_UNSUPPORTED, "flags 0x%x", flags);
  // The whole graph, validated and relabelled exactly as nwgpu_graph_create does.
  nwgpu_graph* whole = nullptr;
  int          rc = nwgpu_graph_create(row_ptr, col, nullptr, n, nnz,
                                       (flags & NWGPU_GRAPH_DEVICE_PTRS) | kGraphNoBlockedPlan, &whole);
  if (rc) return rc;
  if (!whole->relabelled) {
    nwgpu_graph_destroy(whole);
    return fail(NWGPU_ERR_UNSUPPORTED, "the whole graph was not relabelled");
  }
  nwgpu_shard* sh = new (std::nothrow) nwgpu_shard();
  if (!sh) {
    nwgpu_graph_destroy(whole);
    return fail(NWGPU_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  nwgpu_graph* g = new (std::nothrow) nwgpu_graph();
  if (!g) {
    delete sh;
    nwgpu_graph_destroy(whole);
    return fail(NWGPU_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  sh->inner = g;
  auto bail = [&](int code) {
    delete sh;
    nwgpu_graph_destroy(whole);
    return code;
  };
  g->device = whole->device;
  g->sms = whole->sms;
  // nwgpu_graph_create returned with the whole graph's work complete
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamCreate"));
  sh->n = n;
  sh->nnz = nnz;
  sh->world = world;
  sh->rank = rank;
  sh->bounds.assign(bounds, bounds + world + 1);
  sh->row0 = bounds[rank];
  sh->rows = bounds[rank + 1] - bounds[rank];
  sh->stride = stride;
  cudaStream_t s = g->stream;
  // Row range of this rank in the relabelled CSR.
  uint32_t ends[2] = {0, 0};
  if (cudaMemcpyAsync(&ends[0], whole->g.row_ptr + sh->row0, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&ends[1], whole->g.row_ptr + sh->row0 + sh->rows, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return bail(cuda_fail(cudaGetLastError(), "shard row range"));
  const uint64_t m = ends[1] - ends[0];
  g->n = sh->rows;
  g->nnz = m;
  if ((e = pool_alloc_n(&sh->d_bounds, world + 1, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(sh->d_bounds, bounds, (world + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      (e = dalloc(g, &g->g.row_ptr, sh->rows + 1)) != cudaSuccess || (e = dalloc(g, &g->g.col, m)) != cudaSuccess ||
      (e = pool_alloc_n(&sh->perm, n + kPad, s)) != cudaSuccess ||
      (e = pool_alloc_n(&sh->inv_local, sh->rows + kPad, s)) != cudaSuccess ||
      (e = pool_alloc_n(&sh->deg_stage, n + kPad, s)) != cudaSuccess)
    return bail(cuda_fail(e, "cudaMalloc(shard)"));
  shard_rows_kernel<<<g->sms * 4, 256, 0, s>>>(whole->g.row_ptr, sh->row0, sh->row0 + sh->rows, g->g.row_ptr);
  if (m)
    shard_cols_kernel<<<g->sms * 8, 256, 0, s>>>(whole->g.col, ends[0], m, sh->d_bounds, world, stride, g->g.col);
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(sh->perm, whole->g.perm, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s)) !=
          cudaSuccess ||
      (sh->rows && (e = cudaMemcpyAsync(sh->inv_local, whole->g.inv + sh->row0, sh->rows * sizeof(uint32_t),
                                        cudaMemcpyDeviceToDevice, s)) != cudaSuccess) ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return bail(cuda_fail(e, "shard rows"));
  nwgpu_graph_destroy(whole);
  whole = nullptr;
  // The local rows keep the non-increasing length order, so the binned sweep
  // applies; its hub tier counts positions of the padded layout (rank 0's rows).
  g->relabelled = false;
  g->hot_ids = 0;
  if (sh->rows) {
    rc = build_bin_plan(g, g->g.row_ptr, sh->rows, true, &g->plan);
    if (rc) {
      delete sh;
      return rc;
    }
  }
  if (!g->plan.ok && sh->rows) {
    delete sh;
    return fail(NWGPU_ERR_CUDA, "the shard's rows are not in non-increasing length order");
  }
  {
    const uint64_t lim = binned_hot_capacity();
    uint64_t       hub = 32768 < lim ? 32768 : lim;
    if (hub > n) hub = n & ~3ull;
    g->plan.bin.smem_ids = (uint32_t)hub;
    g->plan.bin.l1_ids = (uint32_t)(hub + 16384);
  }
  g->finish_grid = 1;
  // With NWGPU_SWEEP=blocked, the blocked sweep of the local rows, as the
  // single-GPU engine then runs it: row sums are exact fixed-point sums, so
  // each row's value does not depend on how the rows are cut into blocks or
  // shards, and the sharded ranks equal the single-GPU engine's bit for bit.
  const char* which = getenv("NWGPU_SWEEP");
  if (sh->rows && which && !strcmp(which, "blocked")) {
    const char* fmt = getenv("NWGPU_BLOCK_FORMAT");
    if ((e = build_block_plan(g->g.row_ptr, g->g.col, sh->rows, m, (uint64_t)world * stride, g->sms, 0,
                              !(fmt && !strcmp(fmt, "wide")), &g->bplan, s)) != cudaSuccess) {
      delete sh;
      return cuda_fail(e, "shard blocked entry order");
    }
  }
  rc = ensure_solve_buffers(g);
  if (rc) {
    delete sh;
    return rc;
  }
  *out = sh;
  return NWGPU_OK;
}

int nwgpu_shard_destroy(nwgpu_shard* sh) {
  clear_error();
  delete sh;
  return NWGPU_OK;
}

int nwgpu_shard_start(nwgpu_shard* sh, const uint32_t* out_degree, int device_ptrs, float* contrib_slice, void* stream) {
  clear_error();
  if (!sh || !out_degree || !contrib_slice) return fail(NWGPU_ERR_INVALID_ARG, "NULL argument");
  nwgpu_graph* g = sh->inner;
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the CUDA default stream
  const uint32_t* deg_in = out_degree;
  if (!device_ptrs) {
    CK(cudaMemcpyAsync(sh->deg_stage, out_degree, sh->n * sizeof(uint32_t), cudaMemcpyHostToDevice, s),
       "copy out_degree");
    deg_in = sh->deg_stage;
  }
  // local degrees in internal order, rank = 1/n, this rank's contributions into its slice
  CK(launch_gather_u32(deg_in, sh->inv_local, g->deg, sh->rows, g->sms, s), "shard degrees");
  PrState h = {};
  h.max_iters = ~0ull;  // the caller decides when to stop, from the summed L1 changes
  h.chunk_end = ~0ull;
  h.threshold = -1.0;
  *g->h_st = h;
  CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
  SweepArgs a = make_sweep_args(g, 0.85f, 0.f, kTeleportUniform, 0u);
  a.contrib0 = contrib_slice;
  CK(launch_pr_init(a, sh->rows, (float)(1.0 / (double)sh->n), g->sms, s), "shard init");
  sh->sweeps = 0;
  return NWGPU_OK;
}

int nwgpu_shard_sweep(nwgpu_shard* sh, const float* contrib_all, float* contrib_slice, float damping, double* l1,
                      void* stream) {
  clear_error();
  if (!sh || !contrib_all || !contrib_slice || !l1) return fail(NWGPU_ERR_INVALID_ARG, "NULL argument");
  if (!(damping >= 0.0f && damping <= 1.0f)) return fail(NWGPU_ERR_INVALID_ARG, "damping %g outside [0, 1]", (double)damping);
  nwgpu_graph* g = sh->inner;
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the CUDA default stream
  if (sh->rows) {
    // page_rank.hpp:94: base = (1 - d) / N of the whole graph
    const float base = (float)((1.0 - (double)damping) / (double)sh->n);
    SweepArgs   a = make_sweep_args(g, damping, base, kTeleportUniform, 0u);
    // the kernels read contributions from contrib0 on even sweeps and contrib1 on odd ones
    float* all = const_cast<float*>(contrib_all);
    a.contrib0 = (sh->sweeps & 1) ? contrib_slice : all;
    a.contrib1 = (sh->sweeps & 1) ? all : contrib_slice;
    if (g->bplan.ok) {
      CK(launch_blocked_sweep(make_blocked_args(g->bplan, a, sh->rows), g->bplan.sweep_grid, g->bplan.loads, s), "shard sweep");
    } else {
      const BinnedArgs ba = make_binned_args(g, g->plan, a, kModePlain);
      CK(launch_binned_sweep(ba, g->plan.hot, kModePlain, g->plan.sweep_grid, g->plan.finish_grid, s), "shard sweep");
    }
    shard_err_kernel<<<1, 1, 0, s>>>(g->st, l1);
  } else {
    CK(cudaMemsetAsync(l1, 0, sizeof(double), s), "shard sweep");
  }
  CK(cudaGetLastError(), "shard sweep");
  ++sh->sweeps;
  return NWGPU_OK;
}

int nwgpu_shard_decide(nwgpu_shard* sh, const double* l1_total, double threshold, uint64_t max_iters,
                       uint64_t* state, double* errors, uint64_t errors_cap, void* stream) {
  clear_error();
  if (!sh || !l1_total || !state) return fail(NWGPU_ERR_INVALID_ARG, "NULL argument");
  nwgpu_graph* g = sh->inner;
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the CUDA default stream
  shard_decide_kernel<<<1, 1, 0, s>>>(g->st, l1_total, threshold, (unsigned long long)max_iters,
                                      reinterpret_cast<unsigned long long*>(state), errors,
                                      (unsigned long long)errors_cap);
  CK(cudaGetLastError(), "shard decide");
  return NWGPU_OK;
}

int nwgpu_shard_rank_slice(nwgpu_shard* sh, float* rank_slice, void* stream) {
  clear_error();
  if (!sh || !rank_slice) return fail(NWGPU_ERR_INVALID_ARG, "NULL argument");
  nwgpu_graph* g = sh->inner;
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the CUDA default stream
  if (sh->rows) CK(cudaMemcpyAsync(rank_slice, g->rank, sh->rows * sizeof(float), cudaMemcpyDeviceToDevice, s), "copy ranks");
  return NWGPU_OK;
}

int nwgpu_shard_unpermute(nwgpu_shard* sh, const float* ranks_all, float* ranks, void* stream) {
  clear_error();
  if (!sh || !ranks_all || !ranks) return fail(NWGPU_ERR_INVALID_ARG, "NULL argument");
  nwgpu_graph* g = sh->inner;
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the CUDA default stream
  shard_unpermute_kernel<<<g->sms * 4, 256, 0, s>>>(ranks_all, sh->perm, sh->n, sh->d_bounds, sh->world, sh->stride,
                                                    ranks);
  CK(cudaGetLastError(), "shard unpermute");
  return NWGPU_OK;
}

}  // extern "C"
