// Batched personalized PageRank: K teleport vectors per sweep as one SpMM.
//
// Scores are an n x K row-major FP32 matrix (K columns interleaved per
// vertex), so one column-index load feeds K gathers and each gathered
// contribution row is K*4 contiguous bytes (fully used sectors). Column c is
// personalised PageRank with a one-hot teleport at seed_c:
//   r_c' = (1 - d) e_{seed_c} + d * A^T D^{-1} r_c,   r_c(0) = e_{seed_c},
// the per-vector form of the plain update (page_rank.hpp:133) with base_i
// replaced by (1 - d) [i == seed_c]. Each column stops at its own first sweep
// whose FP64 L1 change is below the threshold; its values are then frozen
// while the other columns continue.
//
// Work decomposition: merge-path tiles of W items per WARP (lanes own K/32
// columns each). A warp walks its tile's entries in order with U gathers in
// flight, finishing rows as their end items come up; rows that cross tiles
// leave a K-vector partial per tile, summed in tile order by the finishing
// kernel, which also reduces the per-column residuals and tests convergence.
#include "common.cuh"
#include "engine.h"
#include "ppr.h"

namespace nwgpu {

template <int K>
struct Cols {
  static constexpr int PER_LANE = K / 32;
  float v[PER_LANE];
};

template <int K>
__device__ __forceinline__ void load_row(Cols<K>& out, const float* __restrict__ base, uint32_t row, int lane,
                                         uint64_t pol) {
  const float* p = base + (uint64_t)row * K + lane * Cols<K>::PER_LANE;
  if constexpr (Cols<K>::PER_LANE == 1) {
    out.v[0] = ld_gather(p, pol);
  } else if constexpr (Cols<K>::PER_LANE == 2) {
    float2 t;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;" : "=f"(t.x), "=f"(t.y) : "l"(p), "l"(pol));
    out.v[0] = t.x;
    out.v[1] = t.y;
  } else {
    const float4 t = ld_gather4(reinterpret_cast<const float4*>(p), pol);
    out.v[0] = t.x;
    out.v[1] = t.y;
    out.v[2] = t.z;
    out.v[3] = t.w;
  }
}

// Row epilogue for the K columns of internal row r; returns nothing, adds the
// per-column |dr| into res.
template <int K>
__device__ __forceinline__ void ppr_row_epilogue(const PprArgs& a, float* __restrict__ cout, uint32_t r,
                                                 const Cols<K>& z, double (&res)[Cols<K>::PER_LANE], int lane,
                                                 uint32_t active_bits, const uint32_t (&seed)[Cols<K>::PER_LANE]) {
  constexpr int P = Cols<K>::PER_LANE;
  const float   dg = (float)__ldg(a.deg + r);
  float*        rk = a.rank + (uint64_t)r * K + lane * P;
  float*        co = cout + (uint64_t)r * K + lane * P;
#pragma unroll
  for (int q = 0; q < P; ++q) {
    if (!((active_bits >> q) & 1u)) continue;
    const float tele = (seed[q] == r) ? a.one_minus_d : 0.f;
    const float nr = fmaf(a.damping, z.v[q], tele);
    const float old = rk[q];
    rk[q] = nr;
    co[q] = nr / dg;
    res[q] += (double)fabsf(nr - old);
  }
}

template <int K, int W, int U>
__global__ void __launch_bounds__(256) ppr_sweep_kernel(const PprArgs a) {
  constexpr int P = Cols<K>::PER_LANE;
  constexpr int NWARP = 256 / 32;
  __shared__ uint32_t s_col[NWARP][W + 1];
  __shared__ uint32_t s_rp[NWARP][W + 2];
  __shared__ double   s_res[NWARP][K];
  const int           lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  PprState*           st = a.st;
  if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0u);
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  const float* __restrict__ cin = (it & 1ull) ? a.contrib1 : a.contrib0;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const uint64_t pol = policy_evict_last();

  // this lane's columns: active mask and internal seeds
  uint32_t active = 0, seed[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const int c = lane * P + q;
    seed[q] = a.seeds[c];
    if (!a.col_done[c]) active |= 1u << q;
  }
  double res[P];
#pragma unroll
  for (int q = 0; q < P; ++q) res[q] = 0.0;

  const uint32_t gwarp = blockIdx.x * NWARP + warp, nwarps = gridDim.x * NWARP;
  for (uint32_t t = gwarp; t < a.num_tiles; t += nwarps) {
    const uint32_t r0 = a.tile_row[t], r1 = a.tile_row[t + 1], k0 = a.tile_nnz[t], k1 = a.tile_nnz[t + 1];
    const int      R = (int)(r1 - r0), E = (int)(k1 - k0);
    for (int j = lane; j < E; j += 32) s_col[warp][j] = __ldcs(a.col + k0 + j);
    for (int j = lane; j <= R; j += 32) s_rp[warp][j] = __ldcs(a.row_ptr + r0 + j);
    __syncwarp();
    const bool is_cont = s_rp[warp][0] < k0;
    const bool has_co = k1 > s_rp[warp][R];
    Cols<K>    acc;
#pragma unroll
    for (int q = 0; q < P; ++q) acc.v[q] = 0.f;
    int i = 0;  // next row (relative) whose end item has not been consumed
    // finish rows whose end comes before entry index `upto` (relative)
    auto finish_rows = [&](int upto) {
      while (i < R && (int)(s_rp[warp][i + 1] - k0) <= upto) {
        if (i == 0 && is_cont) {
#pragma unroll
          for (int q = 0; q < P; ++q) a.epart[(uint64_t)t * K + lane * P + q] = acc.v[q];
        } else {
          ppr_row_epilogue<K>(a, cout, r0 + i, acc, res, lane, active, seed);
        }
#pragma unroll
        for (int q = 0; q < P; ++q) acc.v[q] = 0.f;
        ++i;
      }
    };
    for (int kk = 0; kk < E; kk += U) {
      Cols<K> v[U];
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (kk + u < E) load_row<K>(v[u], cin, s_col[warp][kk + u], lane, pol);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (kk + u < E) {
          finish_rows(kk + u);
#pragma unroll
          for (int q = 0; q < P; ++q) acc.v[q] += v[u].v[q];
        }
      }
    }
    finish_rows(0x7fffffff);
    if (has_co) {
#pragma unroll
      for (int q = 0; q < P; ++q) a.cpart[(uint64_t)t * K + lane * P + q] = acc.v[q];
    }
    __syncwarp();
  }
  // per-column residual: warps -> CTA partial (fixed order)
#pragma unroll
  for (int q = 0; q < P; ++q) s_res[warp][lane * P + q] = res[q];
  __syncthreads();
  for (int c = threadIdx.x; c < K; c += blockDim.x) {
    double b = 0.0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) b += s_res[w][c];
    a.res_part[(uint64_t)blockIdx.x * K + c] = b;
  }
}

// Rows crossing warp tiles, per-column residual reduction and convergence.
template <int K>
__global__ void __launch_bounds__(256) ppr_finish_kernel(const PprArgs a) {
  constexpr int P = Cols<K>::PER_LANE;
  constexpr int NWARP = 256 / 32;
  __shared__ double s_res[NWARP][K];
  __shared__ int    s_last;
  const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  PprState*         st = a.st;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const uint32_t D = a.tile_items, T = a.num_tiles;
  uint32_t       active = 0, seed[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const int c = lane * P + q;
    seed[q] = a.seeds[c];
    if (!a.col_done[c]) active |= 1u << q;
  }
  double res[P];
#pragma unroll
  for (int q = 0; q < P; ++q) res[q] = 0.0;
  // one warp per tile boundary: the row carried out of tile ta, if it starts there
  const uint32_t gwarp = blockIdx.x * NWARP + warp, nwarps = gridDim.x * NWARP;
  for (uint32_t ta = gwarp; ta + 1 < T; ta += nwarps) {
    const uint32_t S = a.tile_row[ta + 1];
    const uint32_t k1 = a.tile_nnz[ta + 1], rs = a.row_ptr[S];
    if (!(k1 > rs && ((uint64_t)S + rs) / D == ta)) continue;
    const uint32_t tb = (uint32_t)(((uint64_t)S + a.row_ptr[S + 1]) / D);
    Cols<K>        z;
#pragma unroll
    for (int q = 0; q < P; ++q) z.v[q] = 0.f;
    for (uint32_t u = ta; u < tb; ++u)
#pragma unroll
      for (int q = 0; q < P; ++q) z.v[q] += __ldcg(a.cpart + (uint64_t)u * K + lane * P + q);
#pragma unroll
    for (int q = 0; q < P; ++q) z.v[q] += __ldcg(a.epart + (uint64_t)tb * K + lane * P + q);
    ppr_row_epilogue<K>(a, cout, S, z, res, lane, active, seed);
  }
#pragma unroll
  for (int q = 0; q < P; ++q) s_res[warp][lane * P + q] = res[q];
  __syncthreads();
  for (int c = threadIdx.x; c < K; c += blockDim.x) {
    double b = 0.0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) b += s_res[w][c];
    a.res_part[(uint64_t)(a.sweep_grid + blockIdx.x) * K + c] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // last CTA: one warp per column sums the CTA partials (lane-strided, fixed tree)
  __shared__ int s_all_done;
  if (threadIdx.x == 0) s_all_done = 1;
  __syncthreads();
  const uint32_t parts = a.sweep_grid + gridDim.x;
  for (int c = warp; c < K; c += NWARP) {
    if (a.col_done[c]) continue;  // uniform across the warp
    double e = 0.0;
    for (uint32_t u = lane; u < parts; u += 32) e += __ldcg(a.res_part + (uint64_t)u * K + c);
    e = warp_sum_lane0(e);
    if (lane == 0) {
      a.col_err[c] = e;
      a.col_iters[c] = (uint32_t)(it + 1ull);
      if (e < st->threshold) {
        a.col_done[c] = 1u;
        a.col_conv[c] = 1u;
      } else {
        s_all_done = 0;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long done_iters = it + 1ull;
    st->iter = done_iters;
    const bool abort = a.abort_word && *a.abort_word;
    const bool done = s_all_done || done_iters >= st->max_iters || abort;
    st->aborted = (abort && !s_all_done) ? 1u : 0u;
    st->done = done ? 1u : 0u;
    st->ticket = 0u;
    __threadfence();
    if (a.use_cond && !done && done_iters < st->chunk_end) cudaGraphSetConditional(a.cond, 1u);
  }
}

// rank(i, c) = [i == seed_c], contrib = rank / deg.
template <int K>
__global__ void ppr_init_kernel(const PprArgs a, uint64_t n) {
  const uint64_t total = n * K;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += stride) {
    const uint32_t i = (uint32_t)(x / K);
    const int      c = (int)(x % K);
    const float    r = (a.seeds[c] == i) ? 1.0f : 0.0f;
    a.rank[x] = r;
    a.contrib0[x] = r / (float)a.deg[i];
  }
}

// out[i * k + c] = rank[perm[i] * K + c] for c < k (input order, unpadded).
template <int K>
__global__ void ppr_output_kernel(const float* __restrict__ rank, const uint32_t* __restrict__ perm, uint64_t n,
                                  uint32_t k, float* __restrict__ out) {
  const uint64_t total = n * k;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += stride) {
    const uint64_t i = x / k;
    const uint32_t c = (uint32_t)(x % k);
    const uint64_t src = perm ? perm[i] : i;
    out[x] = rank[src * K + c];
  }
}

// Column set-up: internal seed ids, padding columns inactive from the start.
__global__ void ppr_seed_kernel(const uint32_t* __restrict__ seeds_in, uint32_t k, int K,
                                const uint32_t* __restrict__ perm, PprArgs a) {
  const int c = threadIdx.x;
  if (c >= K) return;
  if ((uint32_t)c < k) {
    const uint32_t s = seeds_in[c];
    const_cast<uint32_t*>(a.seeds)[c] = perm ? perm[s] : s;
    a.col_done[c] = 0u;
  } else {
    const_cast<uint32_t*>(a.seeds)[c] = 0xffffffffu;
    a.col_done[c] = 1u;
  }
  a.col_conv[c] = 0u;
  a.col_iters[c] = 0u;
  a.col_err[c] = 0.0;
}

cudaError_t launch_ppr_seeds(const uint32_t* seeds_in, uint32_t k, int K, const uint32_t* perm, const PprArgs& a,
                             cudaStream_t s) {
  ppr_seed_kernel<<<1, 128, 0, s>>>(seeds_in, k, K, perm, a);
  return cudaGetLastError();
}

__global__ void ppr_arm_kernel(PprState* st) { st->chunk_end = st->iter + kGraphChunk; }

template <int K>
struct PprKernels {
  static void* sweep() { return (void*)ppr_sweep_kernel<K, kPprTileItems, kPprPrefetch>; }
  static void* finish() { return (void*)ppr_finish_kernel<K>; }
};

static void* ppr_sweep_fn(int K) {
  switch (K) {
    case 32: return PprKernels<32>::sweep();
    case 64: return PprKernels<64>::sweep();
    case 128: return PprKernels<128>::sweep();
    default: return nullptr;
  }
}
static void* ppr_finish_fn(int K) {
  switch (K) {
    case 32: return PprKernels<32>::finish();
    case 64: return PprKernels<64>::finish();
    case 128: return PprKernels<128>::finish();
    default: return nullptr;
  }
}

int ppr_padded_k(uint32_t k) { return k <= 32 ? 32 : (k <= 64 ? 64 : (k <= 128 ? 128 : 0)); }

int ppr_sweep_grid(int K, int sms) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppr_sweep_fn(K), 256, 0) != cudaSuccess || nb < 1) nb = 1;
  return sms * nb;
}

cudaError_t launch_ppr_init(const PprArgs& a, int K, uint64_t n, int sms, cudaStream_t s) {
  switch (K) {
    case 32: ppr_init_kernel<32><<<sms * 8, 256, 0, s>>>(a, n); break;
    case 64: ppr_init_kernel<64><<<sms * 8, 256, 0, s>>>(a, n); break;
    case 128: ppr_init_kernel<128><<<sms * 8, 256, 0, s>>>(a, n); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_ppr_output(const float* rank, const uint32_t* perm, uint64_t n, int K, uint32_t k, float* out,
                              int sms, cudaStream_t s) {
  switch (K) {
    case 32: ppr_output_kernel<32><<<sms * 8, 256, 0, s>>>(rank, perm, n, k, out); break;
    case 64: ppr_output_kernel<64><<<sms * 8, 256, 0, s>>>(rank, perm, n, k, out); break;
    case 128: ppr_output_kernel<128><<<sms * 8, 256, 0, s>>>(rank, perm, n, k, out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_ppr_sweep(const PprArgs& a, int K, int sweep_grid, int finish_grid, cudaStream_t s) {
  void* args[] = {(void*)&a};
  cudaError_t e = cudaLaunchKernel(ppr_sweep_fn(K), dim3(sweep_grid), dim3(256), args, 0, s);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernel(ppr_finish_fn(K), dim3(finish_grid), dim3(256), args, 0, s);
}

cudaError_t build_ppr_graph(cudaGraph_t g, const PprArgs& proto, int K, int sweep_grid, int finish_grid,
                            PprState* st, cudaGraphExec_t* exec) {
  cudaGraphNode_t      arm;
  cudaKernelNodeParams kp = {};
  void*                sargs[] = {(void*)&st};
  kp.func = (void*)ppr_arm_kernel;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(1);
  kp.kernelParams = sargs;
  cudaError_t e = cudaGraphAddKernelNode(&arm, g, nullptr, 0, &kp);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle cond;
  if ((e = cudaGraphConditionalHandleCreate(&cond, g, 1u, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wnode;
  if ((e = cudaGraphAddNode(&wnode, g, &arm, 1, &cp)) != cudaSuccess) return e;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  PprArgs     a = proto;
  a.cond = cond;
  a.use_cond = 1;
  void*                args[] = {(void*)&a};
  cudaKernelNodeParams sp = {};
  sp.func = ppr_sweep_fn(K);
  sp.gridDim = dim3(sweep_grid);
  sp.blockDim = dim3(256);
  sp.kernelParams = args;
  cudaGraphNode_t sn, fn;
  if ((e = cudaGraphAddKernelNode(&sn, body, nullptr, 0, &sp)) != cudaSuccess) return e;
  cudaKernelNodeParams fp = sp;
  fp.func = ppr_finish_fn(K);
  fp.gridDim = dim3(finish_grid);
  if ((e = cudaGraphAddKernelNode(&fn, body, &sn, 1, &fp)) != cudaSuccess) return e;
  return cudaGraphInstantiate(exec, g, 0);
}

}  // namespace nwgpu
