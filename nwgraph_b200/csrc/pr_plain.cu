// Plain PageRank sweep kernels for sm_100a.
//
// One sweep = the body of page_rank_v10's iteration
// (include/nwgraph/experimental/algorithms/page_rank.hpp:400-423):
//   z_i   = sum_{k in row i} contrib[col[k]]          (pull gather, :413-415)
//   r_i'  = base + d * z_i                            (:417)
//   err  += |r_i' - r_i|   (FP64)                     (:418)
// fused with the next sweep's contrib_i = r_i' / deg_i (:401-405), written to
// the other half of a ping-pong pair, so a sweep is one kernel.
//
// Work decomposition: merge-path tiles. The sweep is a merge of the n row-end
// items with the nnz entry items; tile t owns items [t*D, (t+1)*D), D = NT*IPT,
// so every tile does the same work whatever the degree skew. Per tile:
//   1. coalesced loads of the tile's col[] slice and row ends, and the random
//      gathers of contrib, staged in shared memory (IPT independent gathers per
//      thread in flight);
//   2. each thread walks IPT items of the merge path over shared memory;
//      rows that cross threads are combined by a block-wide segmented scan;
//   3. coalesced epilogue over the tile's complete rows (rank, degree, the
//      new contribution, the FP64 residual).
// A row that crosses tiles (power-law hubs) leaves one partial per tile; the
// last tile to arrive (atomic counter keyed by the row's first tile) sums the
// partials in tile order and runs that row's epilogue. No CTA ever waits on
// another, so the kernel cannot deadlock whatever the grid size.
// All sums have a fixed order: ranks are bit-reproducible run to run.
#include <cstdio>

#include "common.cuh"
#include "engine.h"

namespace nwgpu {

// ---------------------------------------------------------------------------
// Graph set-up kernels
// ---------------------------------------------------------------------------

// Merge-path coordinate of diagonal d: the row i such that the first d items
// are rows [0, i) and entries [0, d - i).
__device__ __forceinline__ uint32_t merge_path_row(const uint32_t* row_ptr, uint64_t n, uint64_t nnz, uint64_t d) {
  uint64_t lo = d > nnz ? d - nnz : 0;
  uint64_t hi = d < n ? d : n;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    // row mid ends (row_ptr[mid+1]) at or before entry (d - mid - 1): it is consumed.
    if ((uint64_t)row_ptr[mid + 1] + mid + 1 <= d)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (uint32_t)lo;
}

__global__ void tiling_kernel(const uint32_t* __restrict__ row_ptr, uint64_t n, uint64_t nnz, uint32_t D,
                              uint32_t num_tiles, uint32_t* __restrict__ tile_row, uint32_t* __restrict__ tile_nnz) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > num_tiles) return;
  uint64_t d = t * D;
  if (d > n + nnz) d = n + nnz;
  uint32_t i = merge_path_row(row_ptr, n, nnz, d);
  tile_row[t] = i;
  tile_nnz[t] = (uint32_t)(d - i);
}

cudaError_t build_tiling(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, int ipt, Tiling* t, cudaStream_t s) {
  const uint64_t D = (uint64_t)kSweepThreads * ipt;
  const uint64_t tiles = (n + nnz + D - 1) / D;
  if (tiles >= 0xFFFFFFFFull) return cudaErrorInvalidValue;
  t->items_per_thread = ipt;
  t->num_tiles = (uint32_t)tiles;
  cudaError_t e = cudaMalloc(&t->tile_row, (tiles + 1) * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  e = cudaMalloc(&t->tile_nnz, (tiles + 1) * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  const int bs = 256;
  const unsigned blocks = (unsigned)((tiles + 1 + bs - 1) / bs);
  tiling_kernel<<<blocks, bs, 0, s>>>(d_row_ptr, n, nnz, (uint32_t)D, (uint32_t)tiles, t->tile_row, t->tile_nnz);
  return cudaGetLastError();
}

// Bit 0: row_ptr[0] != 0 or row_ptr[n] != nnz; bit 1: row_ptr decreasing;
// bit 2: some col >= n.
__global__ void validate_kernel(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col, uint64_t n,
                                uint64_t nnz, unsigned int* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int bad = 0;
  if (tid == 0 && (row_ptr[0] != 0 || (uint64_t)row_ptr[n] != nnz)) bad |= 1u;
  for (uint64_t i = tid; i < n; i += stride)
    if (row_ptr[i + 1] < row_ptr[i]) bad |= 2u;
  for (uint64_t k = tid; k < nnz; k += stride)
    if ((uint64_t)__ldcs(col + k) >= n) bad |= 4u;
  bad = __reduce_or_sync(kFullMask, bad);
  if ((threadIdx.x & 31) == 0 && bad) atomicOr(err, bad);
}

cudaError_t validate_csr(const uint32_t* d_row_ptr, const uint32_t* d_col, uint64_t n, uint64_t nnz,
                         unsigned int* d_err, cudaStream_t s) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  validate_kernel<<<sms * 8, 256, 0, s>>>(d_row_ptr, d_col, n, nnz, d_err);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Solve kernels
// ---------------------------------------------------------------------------

// rank = init, contrib = init / deg (page_rank.hpp:100-104 and v10 :401-405
// of the first sweep).
__global__ void pr_init_kernel(float* __restrict__ rank, float* __restrict__ contrib, const uint32_t* __restrict__ deg,
                               uint64_t n, float init) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    rank[i] = init;
    contrib[i] = init / (float)deg[i];
  }
}

cudaError_t launch_pr_init(const SweepArgs& a, uint64_t n, float init, cudaStream_t s) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint64_t want = (n + 255) / 256;
  unsigned blocks = (unsigned)(want < (uint64_t)sms * 16 ? (want ? want : 1) : (uint64_t)sms * 16);
  pr_init_kernel<<<blocks, 256, 0, s>>>(a.rank, a.contrib0, a.deg, n, init);
  return cudaGetLastError();
}

// Sets the sweep bound of one graph launch (first node of the graph).
__global__ void pr_arm_kernel(PrState* st) {
  st->chunk_end = st->iter + kGraphChunk;
}

cudaError_t add_pr_arm_node(cudaGraph_t g, PrState* st, cudaGraphNode_t* node) {
  cudaKernelNodeParams kp = {};
  void*                args[] = {(void*)&st};
  kp.func = (void*)pr_arm_kernel;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(1);
  kp.kernelParams = args;
  return cudaGraphAddKernelNode(node, g, nullptr, 0, &kp);
}

// Epilogue of one row: the update of page_rank.hpp:132-135 in Jacobi form.
__device__ __forceinline__ double row_epilogue(const SweepArgs& a, float* cout, uint32_t r, float z, uint64_t pol) {
  const float nr = fmaf(a.damping, z, a.base);
  const float old = ld_stream(a.rank + r);
  st_stream(a.rank + r, nr);
  st_keep(cout + r, nr / (float)ld_stream(a.deg + r), pol);
  return (double)fabsf(nr - old);
}

// A tile's share of row S, which spans tiles [ta, tb]. The last of the
// (tb - ta + 1) contributors sums the shares in tile order and finishes S.
// Called by a whole warp; returns this row's |dr| in lane 0 (0 elsewhere).
template <int D>
__device__ __forceinline__ double span_arrive(const SweepArgs& a, float* cout, uint32_t S, float part, float* slot,
                                              uint64_t pol) {
  const int lane = threadIdx.x & 31;
  uint64_t  ta = 0, tb = 0;
  int       fin = 0;
  if (lane == 0) {
    ta = ((uint64_t)S + a.row_ptr[S]) / D;
    tb = ((uint64_t)S + a.row_ptr[S + 1]) / D;
    *slot = part;
    __threadfence();
    unsigned prev = atomicAdd(a.cnt + ta, 1u);
    fin = (prev == (unsigned)(tb - ta));
  }
  fin = __shfl_sync(kFullMask, fin, 0);
  if (!fin) return 0.0;
  ta = __shfl_sync(kFullMask, ta, 0);
  tb = __shfl_sync(kFullMask, tb, 0);
  __threadfence();
  float s = 0.f;
  for (uint64_t u = ta + lane; u < tb; u += 32) s += __ldcg(a.cpart + u);
  s = warp_sum_lane0(s);
  double dr = 0.0;
  if (lane == 0) {
    const float z = s + __ldcg(a.epart + tb);
    dr = row_epilogue(a, cout, S, z, pol);
    a.cnt[ta] = 0u;  // last arrival: nobody else touches this counter in this sweep
  }
  return dr;
}

template <int NT, int IPT>
__global__ void __launch_bounds__(NT) pr_sweep_kernel(const SweepArgs a) {
  constexpr int D = NT * IPT;
  constexpr int NW = NT / 32;
  __shared__ uint32_t s_buf[D + 1];  // row ends [0, R] (+ sentinel), then gathered values
  __shared__ float    s_z[D];        // row sums of the tile
  __shared__ uint32_t s_key[NT];     // segmented scan of per-thread carries
  __shared__ float    s_sum[NT];
  __shared__ uint32_t s_wkey[NW];
  __shared__ float    s_wsum[NW];
  __shared__ double   s_red[NW];
  __shared__ int      s_last;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  PrState*  st = a.st;

  // Fail-safe for the graph loop: block 0 clears the loop condition before it
  // arrives; only the last CTA of a sweep that must continue sets it again.
  if (a.use_cond && blockIdx.x == 0 && tid == 0) cudaGraphSetConditional(a.cond, 0u);
  if (*(volatile unsigned int*)&st->done) return;  // stable for the whole sweep

  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  const float* __restrict__ cin = (it & 1ull) ? a.contrib1 : a.contrib0;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const uint64_t pol = policy_evict_last();
  double         res = 0.0;

  for (uint32_t t = blockIdx.x; t < a.num_tiles; t += gridDim.x) {
    const uint32_t r0 = a.tile_row[t], r1 = a.tile_row[t + 1];
    const uint32_t k0 = a.tile_nnz[t], k1 = a.tile_nnz[t + 1];
    const int      R = (int)(r1 - r0), E = (int)(k1 - k0);
    uint32_t*      s_end = s_buf;
    float*         s_val = reinterpret_cast<float*>(s_buf + R + 1);

    // 1. loads: row ends (relative to k0) and gathered contributions.
    for (int j = tid; j < R; j += NT) s_end[j] = ld_stream(a.row_ptr + r0 + j + 1) - k0;
    if (tid == 0) s_end[R] = 0x7fffffffu;
    uint32_t c[IPT];
#pragma unroll
    for (int u = 0; u < IPT; ++u) {
      const int j = tid + u * NT;
      c[u] = (j < E) ? ld_stream(a.col + k0 + j) : 0u;
    }
    float v[IPT];
#pragma unroll
    for (int u = 0; u < IPT; ++u) {
      const int j = tid + u * NT;
      v[u] = (j < E) ? ld_gather(cin + c[u], pol) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < IPT; ++u) {
      const int j = tid + u * NT;
      if (j < E) s_val[j] = v[u];
    }
    __syncthreads();

    // 2. merge-path walk over shared memory.
    const int total = R + E;
    const int d0 = min(tid * IPT, total);
    const int d1 = min(d0 + IPT, total);
    int       lo = max(0, d0 - E), hi = min(d0, R);
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((int)s_end[mid] <= d0 - mid - 1)
        lo = mid + 1;
      else
        hi = mid;
    }
    int   i = lo, k = d0 - lo, first = -1;
    float acc = 0.f;
#pragma unroll
    for (int s = 0; s < IPT; ++s) {
      if (d0 + s < d1) {
        if (k < (int)s_end[i]) {
          acc += s_val[k];
          ++k;
        } else {
          s_z[i] = acc;
          if (first < 0) first = i;
          acc = 0.f;
          ++i;
        }
      }
    }
    // Segmented inclusive scan of the carries (key = row the thread ends in).
    uint32_t key = (uint32_t)i;
    float    sv = acc;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t k2 = __shfl_up_sync(kFullMask, key, off);
      const float    v2 = __shfl_up_sync(kFullMask, sv, off);
      if (lane >= off && k2 == key) sv = v2 + sv;
    }
    if (lane == 31) {
      s_wkey[warp] = key;
      s_wsum[warp] = sv;
    }
    __syncthreads();
    {
      int w0 = warp;
      while (w0 > 0 && s_wkey[w0 - 1] == key) --w0;
      if (w0 < warp) {
        float pre = s_wsum[w0];
        for (int w = w0 + 1; w < warp; ++w) pre += s_wsum[w];
        sv = pre + sv;
      }
    }
    s_key[tid] = key;
    s_sum[tid] = sv;
    __syncthreads();
    if (first >= 0 && tid > 0 && s_key[tid - 1] == (uint32_t)first) s_z[first] = s_sum[tid - 1] + s_z[first];
    __syncthreads();

    // 3. epilogue over the tile's complete rows.
    const bool is_cont = ld_stream(a.row_ptr + r0) < k0;   // row r0 began in an earlier tile
    const bool has_co = k1 > ld_stream(a.row_ptr + r1);     // row r1 continues into the next tile
    for (int j = (is_cont ? 1 : 0) + tid; j < R; j += NT) res += row_epilogue(a, cout, r0 + j, s_z[j], pol);
    if (warp == 0) {
      if (is_cont && R >= 1) res += span_arrive<D>(a, cout, r0, s_z[0], a.epart + t, pol);
      if (has_co) {
        const float part = (s_key[NT - 1] == (uint32_t)R) ? s_sum[NT - 1] : 0.f;
        res += span_arrive<D>(a, cout, r1, part, a.cpart + t, pol);
      }
    }
    __syncthreads();  // shared buffers are reused by the next tile
  }

  // FP64 residual: fixed-order block reduction, one partial per CTA.
  res = warp_sum_lane0(res);
  if (lane == 0) s_red[warp] = res;
  __syncthreads();
  if (tid == 0) {
    double b = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) b += s_red[w];
    a.res_part[blockIdx.x] = b;
    __threadfence();
    const unsigned prev = atomicAdd(&st->ticket, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last || warp != 0) return;

  // Last CTA: reduce the residual, record it, test convergence on the device.
  __threadfence();
  double e = 0.0;
  for (unsigned u = lane; u < gridDim.x; u += 32) e += __ldcg(a.res_part + u);
  e = warp_sum_lane0(e);
  if (lane == 0) {
    const unsigned long long done_iters = it + 1ull;
    st->iter = done_iters;
    st->last_error = e;
    if (a.err_hist) a.err_hist[it % a.err_cap] = e;
    const bool conv = e < st->threshold;
    const bool abort = a.abort_word && *a.abort_word;
    const bool done = conv || done_iters >= st->max_iters || abort;
    st->converged = conv ? 1u : 0u;
    st->aborted = (abort && !conv) ? 1u : 0u;
    st->done = done ? 1u : 0u;
    st->ticket = 0u;
    __threadfence();
    if (a.use_cond && !done && done_iters < st->chunk_end) cudaGraphSetConditional(a.cond, 1u);
  }
}

template <int IPT>
static cudaError_t launch_ipt(const SweepArgs& a, int grid, cudaStream_t s) {
  pr_sweep_kernel<kSweepThreads, IPT><<<grid, kSweepThreads, 0, s>>>(a);
  return cudaGetLastError();
}

template <int IPT>
static void* sweep_fn() {
  return (void*)pr_sweep_kernel<kSweepThreads, IPT>;
}

static void* sweep_fn_for(int ipt) {
  switch (ipt) {
    case 4: return sweep_fn<4>();
    case 6: return sweep_fn<6>();
    case 8: return sweep_fn<8>();
    case 12: return sweep_fn<12>();
    case 16: return sweep_fn<16>();
    default: return nullptr;
  }
}

bool ipt_supported(int ipt) { return sweep_fn_for(ipt) != nullptr; }

int sweep_blocks_per_sm(int ipt) {
  void* fn = sweep_fn_for(ipt);
  int   nb = 0;
  if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kSweepThreads, 0) != cudaSuccess) return 1;
  return nb > 0 ? nb : 1;
}

cudaError_t launch_pr_sweep(const SweepArgs& a, int ipt, int grid, cudaStream_t s) {
  switch (ipt) {
    case 4: return launch_ipt<4>(a, grid, s);
    case 6: return launch_ipt<6>(a, grid, s);
    case 8: return launch_ipt<8>(a, grid, s);
    case 12: return launch_ipt<12>(a, grid, s);
    case 16: return launch_ipt<16>(a, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t add_pr_sweep_node(cudaGraph_t body, const SweepArgs& a, int ipt, int grid) {
  void* fn = sweep_fn_for(ipt);
  if (!fn) return cudaErrorInvalidValue;
  cudaKernelNodeParams kp = {};
  void*                args[] = {(void*)&a};
  kp.func = fn;
  kp.gridDim = dim3((unsigned)grid);
  kp.blockDim = dim3(kSweepThreads);
  kp.kernelParams = args;
  cudaGraphNode_t node;
  return cudaGraphAddKernelNode(&node, body, nullptr, 0, &kp);
}

}  // namespace nwgpu
