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
// One sweep is four kernels: the gather (merge-path tiles of W items per
// warp, lanes owning K/32 columns each, rows of the contribution matrix
// loaded U at a time with the next group in flight), the fix-up of rows that
// cross tiles, a streaming epilogue over the n x K matrix (update, FP64
// per-column residual, next contributions) and the per-column convergence
// test.
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

// ---------------------------------------------------------------------------
// Gather: merge-path tiles of W items per warp. A warp walks its tile's
// entries in order, U rows of the contribution matrix per group, and loads
// the next group while it sums the current one (2 * U * K * 4 bytes in flight
// per warp: 4 KB for every K). Column ids and row ends of the tile are staged
// in shared memory; the next row end sits in a register. A finished row only
// stores its K sums (z) into the output contribution matrix: the update, the
// residual and the next contributions are the epilogue kernel's, so nothing
// in this loop waits on a load other than the gathers. The first row of a
// tile that started in an earlier tile leaves its partial in epart[t], the
// last row that continues past the tile in cpart[t].
// ---------------------------------------------------------------------------
template <int K, int U>
__device__ __forceinline__ void load_group(Cols<K> (&v)[U], const float* __restrict__ cin, const uint32_t* s_col, int g,
                                           int E, int lane, uint64_t pol) {
  if ((g + 1) * U <= E) {  // a full group: no bounds checks
#pragma unroll
    for (int u = 0; u < U; ++u) load_row<K>(v[u], cin, s_col[g * U + u], lane, pol);
  } else {
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (g * U + u < E) load_row<K>(v[u], cin, s_col[g * U + u], lane, pol);
  }
}
// Weighted solves: the group's entry weights (the same address in every lane).
template <int U>
__device__ __forceinline__ void load_weights(float (&wv)[U], const float* __restrict__ w, uint32_t k0, int g, int E) {
#pragma unroll
  for (int u = 0; u < U; ++u) wv[u] = (g * U + u < E) ? __ldg(w + k0 + g * U + u) : 0.f;
}

template <int K, int W, int U, bool WEIGHTED>
__global__ void __launch_bounds__(256) ppr_gather_kernel(const PprArgs a) {
  constexpr int P = Cols<K>::PER_LANE;
  constexpr int NWARP = 256 / 32;
  __shared__ uint32_t s_col[NWARP][W + 1];
  __shared__ uint32_t s_rp[NWARP][W + 2];
  const int           lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  PprState*           st = a.st;
  if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0u);
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  const float* __restrict__ cin = (it & 1ull) ? a.contrib1 : a.contrib0;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const uint64_t pol = policy_evict_last();

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
    int i = 0;  // next row (relative) to finish
    int next_end = (R > 0) ? (int)(s_rp[warp][1] - k0) : 0x7fffffff;
    auto flush = [&]() {
      float* dst = (i == 0 && is_cont) ? a.epart + (uint64_t)t * K : cout + (uint64_t)(r0 + i) * K;
#pragma unroll
      for (int q = 0; q < P; ++q) {
        dst[lane * P + q] = acc.v[q];
        acc.v[q] = 0.f;
      }
      ++i;
      next_end = (i < R) ? (int)(s_rp[warp][i + 1] - k0) : 0x7fffffff;
    };
    // one term: the gathered contribution (times the entry's weight when weighted)
    auto add = [&](const Cols<K>& v, float wgt) {
#pragma unroll
      for (int q = 0; q < P; ++q) acc.v[q] = WEIGHTED ? fmaf(wgt, v.v[q], acc.v[q]) : acc.v[q] + v.v[q];
    };
    auto consume = [&](const Cols<K>(&v)[U], const float(&wv)[U], int g) {
      const int e0 = g * U;
      if (next_end >= e0 + U && e0 + U <= E) {  // a full group inside the current row
#pragma unroll
        for (int u = 0; u < U; ++u) add(v[u], wv[u]);
        return;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = e0 + u;
        if (e < E) {
          while (next_end <= e) flush();
          add(v[u], wv[u]);
        }
      }
    };
    Cols<K> va[U], vb[U];
    float   wa[U], wb[U];
#pragma unroll
    for (int u = 0; u < U; ++u) wa[u] = wb[u] = 1.f;
    load_group<K, U>(va, cin, s_col[warp], 0, E, lane, pol);
    if (WEIGHTED) load_weights<U>(wa, a.w, k0, 0, E);
    for (int g = 0; g * U < E; g += 2) {
      load_group<K, U>(vb, cin, s_col[warp], g + 1, E, lane, pol);
      if (WEIGHTED) load_weights<U>(wb, a.w, k0, g + 1, E);
      consume(va, wa, g);
      if ((g + 1) * U >= E) break;
      load_group<K, U>(va, cin, s_col[warp], g + 2, E, lane, pol);
      if (WEIGHTED) load_weights<U>(wa, a.w, k0, g + 2, E);
      consume(vb, wb, g + 1);
    }
    while (next_end <= E) flush();  // rows ending at the tile's last entry, and empty rows after it
    if (has_co) {
#pragma unroll
      for (int q = 0; q < P; ++q) a.cpart[(uint64_t)t * K + lane * P + q] = acc.v[q];
    }
    __syncwarp();
  }
}

// Rows that cross warp tiles are fixed by the tiling: listed once per graph
// as (row, first tile, last tile). One warp per listed row sums its tile
// partials in tile order into z.
__global__ void ppr_spans_kernel(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ tile_row,
                                 const uint32_t* __restrict__ tile_nnz, uint32_t T, uint32_t D, uint4* __restrict__ spans,
                                 unsigned int* __restrict__ count) {
  for (uint32_t ta = blockIdx.x * blockDim.x + threadIdx.x; ta + 1 < T; ta += gridDim.x * blockDim.x) {
    const uint32_t S = tile_row[ta + 1];
    const uint32_t k1 = tile_nnz[ta + 1], rs = row_ptr[S];
    if (!(k1 > rs && ((uint64_t)S + rs) / D == ta)) continue;  // the carried-out row does not start in ta
    const uint32_t tb = (uint32_t)(((uint64_t)S + row_ptr[S + 1]) / D);
    spans[atomicAdd(count, 1u)] = make_uint4(S, ta, tb, 0u);
  }
}

template <int K>
__global__ void __launch_bounds__(256) ppr_fixup_kernel(const PprArgs a) {
  constexpr int P = Cols<K>::PER_LANE;
  PprState*     st = a.st;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const int      lane = threadIdx.x & 31;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t sp = gwarp; sp < a.num_spans; sp += nwarps) {
    const uint4 span = a.spans[sp];
    // 8 interleaved partial sums (tile u goes to sum (u - first) % 8), combined in order
    float z[8][P];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int q = 0; q < P; ++q) z[j][q] = 0.f;
    uint32_t u = span.y;
    for (; u + 8 <= span.z; u += 8)
#pragma unroll
      for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int q = 0; q < P; ++q) z[j][q] += __ldcg(a.cpart + (uint64_t)(u + j) * K + lane * P + q);
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (u + j < span.z)
#pragma unroll
        for (int q = 0; q < P; ++q) z[j][q] += __ldcg(a.cpart + (uint64_t)(u + j) * K + lane * P + q);
#pragma unroll
    for (int q = 0; q < P; ++q) {
      float t = 0.f;
#pragma unroll
      for (int j = 0; j < 8; ++j) t += z[j][q];
      cout[(uint64_t)span.x * K + lane * P + q] = t + __ldcg(a.epart + (uint64_t)span.z * K + lane * P + q);
    }
  }
}

// Epilogue, streaming over the n x K matrix, four columns per thread (16-byte
// loads and stores): for each active column c, r' = (1 - d)[i == seed_c] + d z
// (or (1 - d) t_ic + d z with teleport vectors),
// FP64 |r' - r| into per-CTA column partials; converged columns keep their
// ranks. contrib = r' / deg_i for every column. The grid stride is a multiple
// of K / 4, so every thread stays on one group of four columns.
// EPI: kPprSeeds (one-hot teleports, out-degrees), kPprWeighted (base terms
// (1 - d) t, out-weight sums), kPprTeleports (base terms, out-degrees).
template <int K, int EPI>
__global__ void __launch_bounds__(256) ppr_epilogue_kernel(const PprArgs a, uint64_t n) {
  constexpr int     C4 = K / 4;
  __shared__ double s_res[256][4];
  PprState*         st = a.st;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const uint64_t total = n * C4, stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t x0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int      c0 = (int)(x0 % C4) * 4;
  bool           act[4];
  uint32_t       seed[4];
  bool           any = false;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    act[q] = a.col_done[c0 + q] == 0u;
    seed[q] = a.seeds[c0 + q];
    any = any || act[q];
  }
  const uint64_t pol = policy_evict_last();
  double         res[4] = {0.0, 0.0, 0.0, 0.0};
  if (any) {
    for (uint64_t x = x0; x < total; x += stride) {
      const uint32_t i = (uint32_t)(x / C4);
      const float4   z = __ldcs(reinterpret_cast<const float4*>(cout) + x);
      const float4   old = __ldcs(reinterpret_cast<const float4*>(a.rank) + x);
      // weighted: divide by the out-weight sum; the base terms are (1 - d) t
      const float    dg = EPI == kPprWeighted ? __ldg(a.vaux + i) : (float)__ldg(a.deg + i);
      float4         tb = make_float4(0.f, 0.f, 0.f, 0.f);
      if (EPI != kPprSeeds) tb = __ldg(reinterpret_cast<const float4*>(a.vbase) + x);
      const float    zv[4] = {z.x, z.y, z.z, z.w}, ov[4] = {old.x, old.y, old.z, old.w};
      const float    bv[4] = {tb.x, tb.y, tb.z, tb.w};
      float          nr[4], co[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float tele = EPI != kPprSeeds ? bv[q] : ((seed[q] == i) ? a.one_minus_d : 0.f);
        nr[q] = act[q] ? fmaf(a.damping, zv[q], tele) : ov[q];
        co[q] = nr[q] / dg;
        if (act[q]) res[q] += (double)fabsf(nr[q] - ov[q]);
      }
      __stcs(reinterpret_cast<float4*>(a.rank) + x, make_float4(nr[0], nr[1], nr[2], nr[3]));
      st_keep4(reinterpret_cast<float4*>(cout) + x, make_float4(co[0], co[1], co[2], co[3]), pol);
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) s_res[threadIdx.x][q] = res[q];
  __syncthreads();
  if (threadIdx.x < K) {
    const int g = threadIdx.x / 4, q = threadIdx.x % 4;
    double    b = 0.0;
    for (int j = g; j < (int)blockDim.x; j += C4) b += s_res[j][q];
    a.res_part[(uint64_t)blockIdx.x * K + threadIdx.x] = b;
  }
}

// Per-column residuals over the epilogue's CTAs and the per-column
// convergence test: one warp per column (K / 8 CTAs), lane-strided over the
// partials with a fixed tree; the last CTA to arrive updates the solve state.
template <int K>
__global__ void __launch_bounds__(256) ppr_finish_kernel(const PprArgs a) {
  __shared__ int s_last;
  PprState*      st = a.st;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  const int      lane = threadIdx.x & 31, c = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (c < K && !a.col_done[c]) {  // uniform across the warp
    double e = 0.0;
    for (uint32_t u = lane; u < a.epi_grid; u += 32) e += __ldcg(a.res_part + (uint64_t)u * K + c);
    e = warp_sum_lane0(e);
    if (lane == 0) {
      a.col_err[c] = e;
      a.col_iters[c] = (uint32_t)(it + 1ull);
      if (e < st->threshold) {
        a.col_done[c] = 1u;
        a.col_conv[c] = 1u;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1u);
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  unsigned int running = 0u;
  for (int q = 0; q < K; ++q) running += *(volatile uint32_t*)&a.col_done[q] == 0u ? 1u : 0u;
  const bool               all_done = running == 0u;
  const unsigned long long done_iters = it + 1ull;
  st->iter = done_iters;
  const bool abort = a.abort_word && *a.abort_word;
  const bool end = all_done || done_iters >= st->max_iters || abort;
  // few enough columns still run to continue in a narrower layout: stop here for the host to repack
  const bool narrow = !end && st->narrow_at != 0u && running <= st->narrow_at;
  const bool done = end || narrow;
  st->aborted = (abort && !all_done) ? 1u : 0u;
  st->narrowed = narrow ? 1u : 0u;
  st->done = done ? 1u : 0u;
  st->ticket = 0u;
  __threadfence();
  if (a.use_cond && !done && done_iters < st->chunk_end) cudaGraphSetConditional(a.cond, 1u);
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

// Start from teleport vectors: per column c < k, t = t_in[inv[i] * k + c];
// vbase = (1 - d) t, rank = t, contrib = t / s_i with s the out-weight sums
// (weighted graphs: the single weighted solve's start, per column) or the
// out-degrees (vaux null); padding columns are 0.
template <int K>
__global__ void ppr_winit_kernel(const PprArgs a, const float* __restrict__ t_in, uint32_t k,
                                 const uint32_t* __restrict__ inv, uint64_t n, float* __restrict__ vbase) {
  const uint64_t total = n * K;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += stride) {
    const uint64_t i = x / K;
    const uint32_t c = (uint32_t)(x % K);
    const uint64_t src = inv ? inv[i] : i;
    const float    t = (c < k) ? t_in[src * k + c] : 0.f;
    vbase[x] = a.one_minus_d * t;
    a.rank[x] = t;
    a.contrib0[x] = t / (a.vaux ? a.vaux[i] : (float)a.deg[i]);
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

// Narrowing. The gather sums every column in the same order whatever K is (the
// tiles, the rows within a tile and the crossing rows' partials do not depend
// on it), so moving the running columns into a narrower matrix changes no
// column's values.
__global__ void ppr_repack_kernel(const float* __restrict__ src, float* __restrict__ dst, uint64_t n, uint32_t K_from,
                                  uint32_t K_to, const uint32_t* __restrict__ map, uint32_t nact) {
  const uint64_t total = n * K_to;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += stride) {
    const uint64_t i = x / K_to;
    const uint32_t j = (uint32_t)(x % K_to);
    dst[x] = j < nact ? src[i * K_from + map[j]] : 0.f;
  }
}

// One CTA of 128 threads: every slot's state is read before any is written.
__global__ void ppr_repack_cols_kernel(PprArgs a, uint32_t K_to, const uint32_t* __restrict__ map, uint32_t nact) {
  __shared__ uint32_t s_seed[128], s_done[128], s_conv[128], s_iters[128];
  __shared__ double   s_err[128];
  const uint32_t      j = threadIdx.x;
  if (j < nact) {
    const uint32_t o = map[j];
    s_seed[j] = a.seeds[o];
    s_done[j] = a.col_done[o];
    s_conv[j] = a.col_conv[o];
    s_iters[j] = a.col_iters[o];
    s_err[j] = a.col_err[o];
  }
  __syncthreads();
  if (j >= K_to) return;
  const bool live = j < nact;
  const_cast<uint32_t*>(a.seeds)[j] = live ? s_seed[j] : 0xffffffffu;
  a.col_done[j] = live ? s_done[j] : 1u;
  a.col_conv[j] = live ? s_conv[j] : 0u;
  a.col_iters[j] = live ? s_iters[j] : 0u;
  a.col_err[j] = live ? s_err[j] : 0.0;
}

__global__ void ppr_output_slots_kernel(const float* __restrict__ rank, const uint32_t* __restrict__ perm, uint64_t n,
                                        uint32_t K, const uint32_t* __restrict__ slot_orig, uint32_t k,
                                        float* __restrict__ out) {
  const uint64_t total = n * K;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += stride) {
    const uint64_t i = x / K;
    const uint32_t j = (uint32_t)(x % K), c = slot_orig[j];
    if (c < k) out[i * k + c] = rank[(perm ? (uint64_t)perm[i] : i) * K + j];
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

cudaError_t launch_ppr_spans(const uint32_t* row_ptr, const uint32_t* tile_row, const uint32_t* tile_nnz, uint32_t T,
                             uint32_t D, uint4* spans, unsigned int* count, int sms, cudaStream_t s) {
  if (T < 2) return cudaSuccess;
  ppr_spans_kernel<<<sms * 4, 256, 0, s>>>(row_ptr, tile_row, tile_nnz, T, D, spans, count);
  return cudaGetLastError();
}

cudaError_t launch_ppr_seeds(const uint32_t* seeds_in, uint32_t k, int K, const uint32_t* perm, const PprArgs& a,
                             cudaStream_t s) {
  ppr_seed_kernel<<<1, 128, 0, s>>>(seeds_in, k, K, perm, a);
  return cudaGetLastError();
}

cudaError_t launch_ppr_repack(const float* src, float* dst, uint64_t n, int K_from, int K_to, const uint32_t* map,
                              uint32_t nact, int sms, cudaStream_t s) {
  if (K_to <= 0 || K_to > K_from || nact > (uint32_t)K_to) return cudaErrorInvalidValue;
  ppr_repack_kernel<<<sms * 8, 256, 0, s>>>(src, dst, n, (uint32_t)K_from, (uint32_t)K_to, map, nact);
  return cudaGetLastError();
}

cudaError_t launch_ppr_repack_cols(const PprArgs& a, int K_to, const uint32_t* map, uint32_t nact, cudaStream_t s) {
  if (K_to <= 0 || K_to > 128 || nact > (uint32_t)K_to) return cudaErrorInvalidValue;
  ppr_repack_cols_kernel<<<1, 128, 0, s>>>(a, (uint32_t)K_to, map, nact);
  return cudaGetLastError();
}

cudaError_t launch_ppr_output_slots(const float* rank, const uint32_t* perm, uint64_t n, int K, const uint32_t* slot_orig,
                                    uint32_t k, float* out, int sms, cudaStream_t s) {
  ppr_output_slots_kernel<<<sms * 8, 256, 0, s>>>(rank, perm, n, (uint32_t)K, slot_orig, k, out);
  return cudaGetLastError();
}

__global__ void ppr_arm_kernel(PprState* st) { st->chunk_end = st->iter + kGraphChunk; }

// Rows per group: U * K = 512 floats, 2 KB of rows per group (16 floats per lane).
template <int K, int EPI>
struct PprKernels {
  static constexpr int U = 512 / K;
  static void*         fn(int which) {
    return which == 0   ? (void*)ppr_gather_kernel<K, kPprTileItems, U, EPI == kPprWeighted>
           : which == 1 ? (void*)ppr_fixup_kernel<K>
           : which == 2 ? (void*)ppr_epilogue_kernel<K, EPI>
                        : (void*)ppr_finish_kernel<K>;
  }
};

template <int K>
static void* ppr_fn_k(int which, int mode) {
  return mode == kPprWeighted    ? PprKernels<K, kPprWeighted>::fn(which)
         : mode == kPprTeleports ? PprKernels<K, kPprTeleports>::fn(which)
                                 : PprKernels<K, kPprSeeds>::fn(which);
}

// kernel 0 gather, 1 fix-up, 2 epilogue, 3 finish, for the solve's mode
static void* ppr_fn(int K, int which, int mode = kPprSeeds) {
  switch (K) {
    case 32: return ppr_fn_k<32>(which, mode);
    case 64: return ppr_fn_k<64>(which, mode);
    case 128: return ppr_fn_k<128>(which, mode);
    default: return nullptr;
  }
}

int ppr_mode(const PprArgs& a) { return a.w ? kPprWeighted : (a.vbase ? kPprTeleports : kPprSeeds); }

// Grid of each kernel: gather persistent at its occupancy, fix-up one warp
// per row crossing tiles, epilogue epi_grid CTAs, finish one warp per column.
static int K_of(const PprArgs& a) { return (int)a.K; }
static dim3 ppr_grid(const PprArgs& a, int which, int sweep_grid) {
  if (which == 0) return dim3((unsigned)sweep_grid);
  if (which == 1) return dim3(a.num_spans ? (a.num_spans + 7u) / 8u : 1u);
  if (which == 2) return dim3(a.epi_grid);
  return dim3((unsigned)(K_of(a) / 8));
}

int ppr_padded_k(uint32_t k) { return k <= 32 ? 32 : (k <= 64 ? 64 : (k <= 128 ? 128 : 0)); }

int ppr_sweep_grid(int K, int sms) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppr_fn(K, 0), 256, 0) != cudaSuccess || nb < 1) nb = 1;
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

cudaError_t launch_ppr_winit(const PprArgs& a, int K, const float* t_in, uint32_t k, const uint32_t* inv, uint64_t n,
                             float* vbase, int sms, cudaStream_t s) {
  switch (K) {
    case 32: ppr_winit_kernel<32><<<sms * 8, 256, 0, s>>>(a, t_in, k, inv, n, vbase); break;
    case 64: ppr_winit_kernel<64><<<sms * 8, 256, 0, s>>>(a, t_in, k, inv, n, vbase); break;
    case 128: ppr_winit_kernel<128><<<sms * 8, 256, 0, s>>>(a, t_in, k, inv, n, vbase); break;
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

cudaError_t launch_ppr_sweep(const PprArgs& a, int K, int sweep_grid, cudaStream_t s) {
  void* args[] = {(void*)&a};
  for (int w = 0; w < 4; ++w) {
    uint64_t    n = a.n;
    void*       eargs[] = {(void*)&a, (void*)&n};
    cudaError_t e = cudaLaunchKernel(ppr_fn(K, w, ppr_mode(a)), ppr_grid(a, w, sweep_grid), dim3(256),
                                     w == 2 ? eargs : args, 0, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t build_ppr_graph(cudaGraph_t g, const PprArgs& proto, int K, int sweep_grid, PprState* st,
                            cudaGraphExec_t* exec) {
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
  uint64_t             n = a.n;
  void*                args[] = {(void*)&a};
  void*                eargs[] = {(void*)&a, (void*)&n};
  cudaGraphNode_t      prev = nullptr;
  for (int w = 0; w < 4; ++w) {
    cudaKernelNodeParams kp2 = {};
    kp2.func = ppr_fn(K, w, ppr_mode(a));
    kp2.gridDim = ppr_grid(a, w, sweep_grid);
    kp2.blockDim = dim3(256);
    kp2.kernelParams = w == 2 ? eargs : args;
    cudaGraphNode_t node;
    if ((e = cudaGraphAddKernelNode(&node, body, prev ? &prev : nullptr, prev ? 1 : 0, &kp2)) != cudaSuccess) return e;
    prev = node;
  }
  return cudaGraphInstantiate(exec, g, 0);
}

}  // namespace nwgpu
