// Ragged batches as one union graph: every graph of a batch that is not
// solved alone becomes a diagonal block of one CSR (its vertices renumbered
// after the previous graphs'), which is relabelled and swept by the
// degree-binned kernel in its kModeRagged form. No counterpart in the
// reference (page_rank.hpp:92-147 solves one graph).
//
// A row's sum depends only on the row's own entries and its length (which
// bin, lanes and steps sum it), not on which rows share its warp, so every
// graph of the union gets, sweep for sweep, the ranks a single-graph handle
// gives it, bit for bit: init 1/n_g, base (1 - d)/n_g, contribution r / deg.
// Each graph stops at its own first sweep whose FP64 L1 change is below the
// threshold (page_rank.hpp:144): the sweep writes each updated row's |dr| to
// row_res, and one warp per graph sums its rows' changes in the graph's
// vertex order. Rows of stopped graphs are neither gathered nor updated.
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "ragged_union.h"

namespace nwgpu {

// Index j of the union part holding x: the last j with off[j] <= x (parts of
// zero length share an offset with the next one and are skipped).
__device__ __forceinline__ uint32_t part_of(const uint64_t* __restrict__ off, uint32_t m, uint64_t x) {
  uint32_t lo = 0, hi = m - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Union row pointers: row u of part j is row u - voff[j] of graph ids[j],
// whose local row pointers start at 0 in the batch's row_ptr at graphs[g].p0.
__global__ void union_rows_kernel(const RaggedGraph* __restrict__ graphs, const uint32_t* __restrict__ batch_row_ptr,
                                  UnionParts p, uint32_t* __restrict__ rp) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < p.n; u += stride) {
    const uint32_t j = part_of(p.voff, p.m, u);
    const uint32_t g = p.ids[j];
    rp[u] = (uint32_t)(p.eoff[j] + batch_row_ptr[graphs[g].p0 + (u - p.voff[j])]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) rp[p.n] = (uint32_t)p.nnz;
}

// Union column ids: entry e of part j is entry e - eoff[j] of graph ids[j]
// (local ids), shifted by the part's first union vertex.
__global__ void union_cols_kernel(const RaggedGraph* __restrict__ graphs, const uint32_t* __restrict__ batch_col,
                                  UnionParts p, uint32_t* __restrict__ col) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < p.nnz; e += stride) {
    const uint32_t j = part_of(p.eoff, p.m, e);
    const uint32_t g = p.ids[j];
    col[e] = batch_col[graphs[g].e0 + (e - p.eoff[j])] + (uint32_t)p.voff[j];
  }
}

// Per internal row of the relabelled union (inv: internal -> union id): its
// graph's batch index.
__global__ void union_row_graph_kernel(const uint32_t* __restrict__ inv, UnionParts p, uint32_t* __restrict__ row_graph) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < p.n; r += stride)
    row_graph[r] = p.ids[part_of(p.voff, p.m, inv[r])];
}

// Start of a solve: per graph of the union its base term (1 - d)/n_g (in
// double, stored as float: page_rank.hpp:93-94) and a fresh state; per
// internal row the degree from the batch's array, rank 1/n_g and
// contribution rank / deg (page_rank.hpp:100-104).
__global__ void union_start_kernel(const RaggedGraph* __restrict__ graphs, UnionParts p, const uint32_t* __restrict__ inv,
                                   const uint32_t* __restrict__ row_graph, const uint32_t* __restrict__ batch_deg,
                                   float damping, uint32_t stopped, float* __restrict__ base, RaggedState rs,
                                   uint32_t* __restrict__ deg, float* __restrict__ rank, float* __restrict__ contrib) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t j = tid; j < p.m; j += stride) {
    const uint32_t g = p.ids[j];
    const uint32_t n = graphs[g].n;
    base[g] = n ? (float)((1.0 - (double)damping) / (double)n) : 0.f;
    rs.done[g] = stopped;
    rs.iters[g] = 0u;
    rs.err[g] = 0.0;
    rs.conv[g] = 0u;
  }
  for (uint64_t r = tid; r < p.n; r += stride) {
    const uint64_t u = inv[r];
    const uint32_t j = part_of(p.voff, p.m, u);
    const uint32_t g = row_graph[r];
    const uint32_t d = batch_deg[graphs[g].v0 + (u - p.voff[j])];
    const float    x = (float)(1.0 / (double)graphs[g].n);
    deg[r] = d;
    rank[r] = x;
    contrib[r] = x / (float)d;
  }
}

// After a sweep's finishing kernel, the per-graph sums in two fixed-order
// steps: one warp per chunk of kUnionChunk vertices of a running graph sums
// their rows' FP64 changes (lane-strided in vertex order, then a fixed tree);
// then one warp per running graph sums its chunks in order.
__global__ void __launch_bounds__(256) union_chunk_kernel(UnionParts p, const uint32_t* __restrict__ perm,
                                                          const double* __restrict__ row_res, RaggedState rs,
                                                          const PrState* st) {
  if (*(const volatile unsigned int*)&st->done) return;
  const uint32_t lane = threadIdx.x & 31, nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < p.chunks; c += nwarps) {
    uint32_t lo = 0, hi = p.m - 1;  // the part holding chunk c: the last j with coff[j] <= c
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (p.coff[mid] <= c)
        lo = mid;
      else
        hi = mid - 1;
    }
    if (rs.done[p.ids[lo]]) continue;  // uniform across the warp
    const uint64_t u0 = p.voff[lo] + (uint64_t)(c - p.coff[lo]) * kUnionChunk;
    const uint64_t u1 = u0 + kUnionChunk < p.voff[lo + 1] ? u0 + kUnionChunk : p.voff[lo + 1];
    double         e = 0.0;
    for (uint64_t u = u0 + lane; u < u1; u += 32) e += __ldcg(row_res + perm[u]);
    e = warp_sum_lane0(e);
    if (lane == 0) p.chunk_part[c] = e;
  }
}

// One warp per running graph: its change (its chunks' sums in order), the
// sweep count, and the stop at the first change below the threshold or at
// max_iters. The last CTA to arrive ends the loop once no graph runs (or on
// abort), and otherwise keeps the CUDA-graph loop going within its chunk.
__global__ void __launch_bounds__(256) union_converge_kernel(UnionParts p, RaggedState rs, PrState* st,
                                                             double threshold, const volatile unsigned int* abort_word,
                                                             cudaGraphConditionalHandle cond, int use_cond) {
  __shared__ int s_last;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;  // sweeps done, this one included
  const uint32_t lane = threadIdx.x & 31, nwarps = gridDim.x * (blockDim.x >> 5);
  unsigned int   running = 0;
  for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < p.m; j += nwarps) {
    const uint32_t g = p.ids[j];
    if (rs.done[g]) continue;  // uniform across the warp
    double e = 0.0;
    for (uint32_t c = p.coff[j] + lane; c < p.coff[j + 1]; c += 32) e += __ldcg(p.chunk_part + c);
    e = warp_sum_lane0(e);
    if (lane == 0) {
      const bool conv = e < threshold;
      rs.err[g] = e;
      rs.iters[g] = (uint32_t)it;
      rs.conv[g] = conv ? 1u : 0u;
      if (conv || it >= st->max_iters)
        rs.done[g] = 1u;
      else
        ++running;
    }
  }
  if (running) atomicAdd(&st->pending, running);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1u);
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  const unsigned int left = *(volatile unsigned int*)&st->pending;
  const bool         abort = abort_word && *abort_word;
  const bool         done = left == 0u || it >= st->max_iters || abort;
  st->aborted = (abort && left) ? 1u : 0u;
  st->converged = left == 0u ? 1u : 0u;
  st->done = done ? 1u : 0u;
  st->pending = 0u;
  st->ticket = 0u;
  __threadfence();
  if (use_cond && !done && it < st->chunk_end) cudaGraphSetConditional(cond, 1u);
}

// The union's ranks (internal order) into the batch's rank array.
__global__ void union_output_kernel(const RaggedGraph* __restrict__ graphs, UnionParts p, const uint32_t* __restrict__ perm,
                                    const float* __restrict__ rank, float* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < p.n; u += stride) {
    const uint32_t j = part_of(p.voff, p.m, u);
    out[graphs[p.ids[j]].v0 + (u - p.voff[j])] = rank[perm[u]];
  }
}

__global__ void union_arm_kernel(PrState* st) { st->chunk_end = st->iter + kGraphChunk; }

cudaError_t launch_union_build(const RaggedGraph* graphs, const uint32_t* batch_row_ptr, const uint32_t* batch_col,
                               const UnionParts& p, uint32_t* rp, uint32_t* col, int sms, cudaStream_t s) {
  if (p.m == 0) return cudaSuccess;
  union_rows_kernel<<<sms * 8, 256, 0, s>>>(graphs, batch_row_ptr, p, rp);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || p.nnz == 0) return e;
  union_cols_kernel<<<sms * 8, 256, 0, s>>>(graphs, batch_col, p, col);
  return cudaGetLastError();
}

cudaError_t launch_union_row_graph(const uint32_t* inv, const UnionParts& p, uint32_t* row_graph, int sms,
                                   cudaStream_t s) {
  if (p.n == 0) return cudaSuccess;
  union_row_graph_kernel<<<sms * 8, 256, 0, s>>>(inv, p, row_graph);
  return cudaGetLastError();
}

cudaError_t launch_union_start(const RaggedGraph* graphs, const UnionParts& p, const uint32_t* inv,
                               const uint32_t* row_graph, const uint32_t* batch_deg, float damping, uint32_t stopped,
                               float* base, const RaggedState& rs, uint32_t* deg, float* rank, float* contrib, int sms,
                               cudaStream_t s) {
  if (p.m == 0) return cudaSuccess;
  union_start_kernel<<<sms * 8, 256, 0, s>>>(graphs, p, inv, row_graph, batch_deg, damping, stopped, base, rs, deg, rank,
                                             contrib);
  return cudaGetLastError();
}

static int warp_grid(uint64_t warps, int sms) {  // one warp per item, at most 8 CTAs of 256 per SM
  const uint64_t blocks = (warps + 7u) / 8u;
  const uint64_t cap = (uint64_t)sms * 8u;
  return (int)(blocks == 0 ? 1 : (blocks < cap ? blocks : cap));
}

cudaError_t launch_union_converge(const UnionParts& p, const uint32_t* perm, const double* row_res,
                                  const RaggedState& rs, PrState* st, double threshold,
                                  const volatile unsigned int* abort_word, int sms, cudaStream_t s) {
  union_chunk_kernel<<<warp_grid(p.chunks, sms), 256, 0, s>>>(p, perm, row_res, rs, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  union_converge_kernel<<<warp_grid(p.m, sms), 256, 0, s>>>(p, rs, st, threshold, abort_word,
                                                            cudaGraphConditionalHandle{}, 0);
  return cudaGetLastError();
}

cudaError_t launch_union_output(const RaggedGraph* graphs, const UnionParts& p, const uint32_t* perm, const float* rank,
                                float* out, int sms, cudaStream_t s) {
  if (p.n == 0) return cudaSuccess;
  union_output_kernel<<<sms * 8, 256, 0, s>>>(graphs, p, perm, rank, out);
  return cudaGetLastError();
}

cudaError_t build_union_graph(cudaGraph_t cg, const BinnedArgs& proto, int sweep_grid, int finish_grid,
                              const UnionParts& p, const uint32_t* perm, const double* row_res, const RaggedState& rs,
                              PrState* st, double threshold, const volatile unsigned int* abort_word, int sms,
                              cudaGraphExec_t* exec) {
  cudaGraphNode_t      arm;
  cudaKernelNodeParams kp = {};
  void*                aargs[] = {(void*)&st};
  kp.func = (void*)union_arm_kernel;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(1);
  kp.kernelParams = aargs;
  cudaError_t e = cudaGraphAddKernelNode(&arm, cg, nullptr, 0, &kp);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle cond;
  if ((e = cudaGraphConditionalHandleCreate(&cond, cg, 1u, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wnode;
  if ((e = cudaGraphAddNode(&wnode, cg, &arm, 1, &cp)) != cudaSuccess) return e;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  BinnedArgs  a = proto;
  a.sw.cond = cond;
  a.sw.use_cond = 1;
  cudaGraphNode_t last;  // the chunk sums and the convergence node go after the finishing kernel
  if ((e = add_binned_nodes(body, a, true, kModeRagged, sweep_grid, finish_grid, &last)) != cudaSuccess) return e;
  UnionParts                   pp = p;
  const uint32_t*              pm = perm;
  const double*                rr = row_res;
  RaggedState                  rss = rs;
  PrState*                     sp = st;
  const PrState*               csp = st;
  double                       thr = threshold;
  const volatile unsigned int* ab = abort_word;
  int                          one = 1;
  void*                        kargs[] = {(void*)&pp, (void*)&pm, (void*)&rr, (void*)&rss, (void*)&csp};
  cudaKernelNodeParams         kn = {};
  kn.func = (void*)union_chunk_kernel;
  kn.gridDim = dim3((unsigned)warp_grid(p.chunks, sms));
  kn.blockDim = dim3(256);
  kn.kernelParams = kargs;
  cudaGraphNode_t chunk;
  if ((e = cudaGraphAddKernelNode(&chunk, body, &last, 1, &kn)) != cudaSuccess) return e;
  void*                cargs[] = {(void*)&pp, (void*)&rss, (void*)&sp, (void*)&thr, (void*)&ab, (void*)&cond, (void*)&one};
  cudaKernelNodeParams cn = {};
  cn.func = (void*)union_converge_kernel;
  cn.gridDim = dim3((unsigned)warp_grid(p.m, sms));
  cn.blockDim = dim3(256);
  cn.kernelParams = cargs;
  cudaGraphNode_t conv;
  if ((e = cudaGraphAddKernelNode(&conv, body, &chunk, 1, &cn)) != cudaSuccess) return e;
  return cudaGraphInstantiate(exec, cg, 0);
}

}  // namespace nwgpu
