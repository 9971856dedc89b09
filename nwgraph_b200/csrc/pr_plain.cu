// PageRank sweep kernels for sm_100a.
//
// One sweep = the body of page_rank_v10's iteration
// (include/nwgraph/experimental/algorithms/page_rank.hpp:400-423):
//   z_i  = sum_{k in row i} contrib[col[k]]           (pull gather, :413-415)
//   r_i' = base_i + d * z_i                           (:417)
//   err += |r_i' - r_i|   (FP64)                      (:418)
// fused with the next sweep's contrib_i = r_i' / deg_i (:401-405), written to
// the other half of a ping-pong pair.
//
// Work decomposition: merge-path tiles. A sweep is the merge of the n row-end
// items with the nnz entry items; tile t owns items [t*D, (t+1)*D), D = NT*IPT,
// so every tile costs the same whatever the degree skew.
//
// pr_sweep_kernel (persistent, one CTA per tile at a time) pipelines tiles:
//   * TMA bulk copies (cp.async.bulk + mbarrier) bring tile i+2's slices of
//     col, row_ptr, rank and degree into shared memory,
//   * the random gathers of contrib for tile i+1 are in flight in registers,
//   * while tile i is reduced from shared memory: each thread walks IPT merge
//     items, rows crossing threads are combined by a block-wide segmented scan,
//     and complete rows run the epilogue (rank, contrib, FP64 |dr|).
// A row that crosses a tile boundary leaves one FP32 partial per tile
// (cpart / epart); pr_finish_kernel, launched right after, sums each such
// row's partials in tile order, runs its epilogue, reduces the residual and
// tests convergence on the device. All sums have a fixed order, so ranks are
// bit-reproducible run to run. No CTA waits on another CTA.
#include <cstdio>

#include "common.cuh"
#include "engine.h"

namespace nwgpu {

// ---------------------------------------------------------------------------
// TMA bulk copy + mbarrier helpers (each copy lands in the issuing CTA's own shared memory)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `polls` suspended polls; the sweeps allow 2^20.
__device__ __forceinline__ bool mbar_wait_n(uint64_t* bar, uint32_t parity, uint32_t polls) {
#pragma unroll 1
  for (uint32_t it = 0; it < polls; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) { return mbar_wait_n(bar, parity, 1u << 20); }

// ---------------------------------------------------------------------------
// Shared-memory layout of the sweep kernel
// ---------------------------------------------------------------------------
struct TileMeta {
  uint32_t r0, r1, k0, k1;  // merge-path coordinates of the tile
  uint32_t col_at;          // stage word holding col[k0] (0..3)
  uint32_t rp_at;           // stage word holding row_ptr[r0] (row_ptr[r0..r1] follow)
  uint32_t rk_at;           // stage word holding rank[r0], or ~0u when rank/deg are not staged
  uint32_t dg_at;           // stage word holding deg[r0]
  float    base;            // ragged batches: the tile's graph's base term
  uint32_t tile;            // ragged batches: the tile (the sweep walks the running graphs' tile list)
  uint64_t v0;              // ragged batches: the tile's graph's first vertex
};

template <int NT, int IPT>
struct alignas(16) SweepSmem {
  static constexpr int D = NT * IPT;
  static constexpr int NW = NT / 32;
  // col[k0,k1) and row_ptr[r0..r1] rounded out to 16 bytes share D + 16 words
  // (E + R <= D); rank and deg of the tile's rows follow when R <= D / 4
  // (row-heavy tiles read them from global memory in the epilogue).
  static constexpr int RV = D / 4;
  static constexpr int STG = D + 16 + 2 * (RV + 8);
  uint32_t stage[2][STG];
  float    z[D];  // row sums of the tile
  uint32_t wkey[NW];
  float    wsum[NW];
  double   red[NW];
  uint64_t bar[3];  // two tile stages, the hot-id cache
  TileMeta meta[2];
};

template <int NT, int IPT>
constexpr size_t sweep_smem() {
  return sizeof(SweepSmem<NT, IPT>);
}

__device__ __forceinline__ float base_of(const SweepArgs& a, uint32_t r) {
  if (a.teleport == kTeleportSeed) return (r == a.seed) ? a.base : 0.f;
  return a.base;
}

// Thread 0, ragged batches: entry i of the running graphs' tile list, tile t
// of graph g, in local coordinates; the slices start at the graph's 64-bit
// bases and are rounded out to 16 bytes of the batch arrays.
template <int NT, int IPT>
__device__ __forceinline__ void issue_ragged_tile(const SweepArgs& a, uint32_t i, uint32_t* stg, TileMeta* m,
                                                  uint64_t* bar, uint64_t pol) {
  constexpr int  RV = SweepSmem<NT, IPT>::RV;
  const uint2    tg = __ldcg(a.act_list + i);
  const uint32_t t = tg.x, g = tg.y;
  const RaggedGraph* G = a.graphs + g;
  m->base = a.graph_base[g];
  m->v0 = G->v0;
  m->tile = t;
  const uint32_t e = t + g;
  const uint32_t r0 = a.tile_row[e], r1 = a.tile_row[e + 1], k0 = a.tile_nnz[e], k1 = a.tile_nnz[e + 1];
  const uint64_t K0 = G->e0 + k0, P0 = G->p0 + r0, V0 = G->v0 + r0;
  const uint64_t ca0 = K0 & ~3ull, ca1 = (G->e0 + k1 + 3ull) & ~3ull;  // col[k0, k1)
  const uint64_t pa0 = P0 & ~3ull, pa1 = (G->p0 + r1 + 4ull) & ~3ull;  // row_ptr[r0 .. r1]
  const uint64_t va0 = V0 & ~3ull, va1 = (G->v0 + r1 + 3ull) & ~3ull;  // rank / deg [r0, r1)
  const bool     stage_rows = (r1 > r0) && (r1 - r0 <= (uint32_t)RV);
  const uint32_t cw = (uint32_t)(ca1 - ca0), pw = (uint32_t)(pa1 - pa0), vw = stage_rows ? (uint32_t)(va1 - va0) : 0u;
  m->r0 = r0;
  m->r1 = r1;
  m->k0 = k0;
  m->k1 = k1;
  m->col_at = (uint32_t)(K0 - ca0);
  m->rp_at = cw + (uint32_t)(P0 - pa0);
  m->rk_at = stage_rows ? cw + pw + (uint32_t)(V0 - va0) : ~0u;
  m->dg_at = cw + pw + vw + (uint32_t)(V0 - va0);
  mbar_arrive_expect_tx(bar, 4u * (cw + pw + 2u * vw));
  if (cw) bulk_load(stg, a.col + ca0, 4u * cw, bar, pol);
  bulk_load(stg + cw, a.row_ptr + pa0, 4u * pw, bar, pol);
  if (vw) {
    bulk_load(stg + cw + pw, a.rank + va0, 4u * vw, bar, pol);
    bulk_load(stg + cw + pw + vw, a.deg + va0, 4u * vw, bar, pol);
  }
}

// Thread 0, arrays without spare elements: words [w0, w1) of src go to dst
// (w0 and w1 multiples of 4), but src holds only `len` words and nothing at
// or past len may be read. The words below min(w1, len & ~3) are left to the
// bulk copy, whose word count is returned; the at most 3 words of
// [len & ~3, len) inside the slice are loaded here with plain loads and
// stored to shared memory before the stage's mbarrier arrival, which
// releases them to the threads that wait on it. Stage words at or past len
// stay unwritten; the sweep never reads them as values.
__device__ __forceinline__ uint32_t stage_tail(uint32_t* dst, const uint32_t* src, uint32_t w0, uint32_t w1,
                                               uint32_t len) {
  if (w1 <= len) return w1 - w0;
  const uint32_t b1 = max(w0, len & ~3u);
  for (uint32_t w = b1; w < len; ++w) dst[w - w0] = __ldcg(src + w);
  return b1 - w0;
}

// Thread 0: bring tile t's slices into stage `stg` and record where they landed.
template <int NT, int IPT>
__device__ __forceinline__ void issue_tile(const SweepArgs& a, uint32_t t, uint32_t* stg, TileMeta* m, uint64_t* bar,
                                           uint64_t pol) {
  constexpr int  RV = SweepSmem<NT, IPT>::RV;
  const uint32_t r0 = a.tile_row[t], r1 = a.tile_row[t + 1], k0 = a.tile_nnz[t], k1 = a.tile_nnz[t + 1];
  const uint32_t ca0 = k0 & ~3u, ca1 = (k1 + 3u) & ~3u;  // col[k0, k1)
  const uint32_t pa0 = r0 & ~3u, pa1 = (r1 + 4u) & ~3u;  // row_ptr[r0 .. r1]
  const uint32_t va0 = r0 & ~3u, va1 = (r1 + 3u) & ~3u;  // rank / deg [r0, r1)
  const bool     stage_rows = (r1 > r0) && (r1 - r0 <= (uint32_t)RV);
  const uint32_t cw = ca1 - ca0, pw = pa1 - pa0, vw = stage_rows ? va1 - va0 : 0u;
  m->r0 = r0;
  m->r1 = r1;
  m->k0 = k0;
  m->k1 = k1;
  m->col_at = k0 - ca0;
  m->rp_at = cw + (r0 - pa0);
  m->rk_at = stage_rows ? cw + pw + (r0 - va0) : ~0u;
  m->dg_at = cw + pw + vw + (r0 - va0);
  // words of each slice that the bulk copies bring in: all of them, unless
  // the slice runs past the end of an array without spare elements
  uint32_t bc = cw, bp = pw, bv = vw;
  if (a.exact_ends) {
    if (cw) bc = stage_tail(stg, a.col, ca0, ca1, a.n_entries);
    bp = stage_tail(stg + cw, a.row_ptr, pa0, pa1, a.n_rows + 1u);
    if (vw) {
      bv = stage_tail(stg + cw + pw, reinterpret_cast<const uint32_t*>(a.rank), va0, va1, a.n_rows);
      stage_tail(stg + cw + pw + vw, a.deg, va0, va1, a.n_rows);
    }
  }
  mbar_arrive_expect_tx(bar, 4u * (bc + bp + 2u * bv));
  if (bc) bulk_load(stg, a.col + ca0, 4u * bc, bar, pol);
  if (bp) bulk_load(stg + cw, a.row_ptr + pa0, 4u * bp, bar, pol);
  if (bv) {
    bulk_load(stg + cw + pw, a.rank + va0, 4u * bv, bar, pol);
    bulk_load(stg + cw + pw + vw, a.deg + va0, 4u * bv, bar, pol);
  }
}

// Each thread gathers the contributions of its IPT consecutive entries
// [tid*IPT, tid*IPT + IPT) of the tile into registers. The column ids are read
// as 16-byte words from the aligned stage and shifted by col_at (uniform).
template <int NT, int IPT, bool HOT>
__device__ __forceinline__ void gather_tile(const uint32_t* stg, const TileMeta& m, const float* __restrict__ cin,
                                            float (&v)[IPT], uint64_t pol, uint32_t hot, const float* hot_smem) {
  static_assert(IPT % 4 == 0, "IPT must be a multiple of 4");
  const int  E = (int)(m.k1 - m.k0);
  const int  e0 = (int)threadIdx.x * IPT;
  uint32_t   w[IPT + 4];
  const uint4* src = reinterpret_cast<const uint4*>(stg + e0);
#pragma unroll
  for (int q = 0; q < IPT / 4 + 1; ++q) {
    const uint4 x = src[q];
    w[4 * q + 0] = x.x;
    w[4 * q + 1] = x.y;
    w[4 * q + 2] = x.z;
    w[4 * q + 3] = x.w;
  }
  uint32_t idx[IPT];
  switch (m.col_at) {
    case 0:
#pragma unroll
      for (int u = 0; u < IPT; ++u) idx[u] = w[u];
      break;
    case 1:
#pragma unroll
      for (int u = 0; u < IPT; ++u) idx[u] = w[u + 1];
      break;
    case 2:
#pragma unroll
      for (int u = 0; u < IPT; ++u) idx[u] = w[u + 2];
      break;
    default:
#pragma unroll
      for (int u = 0; u < IPT; ++u) idx[u] = w[u + 3];
      break;
  }
  // Vertices below `hot` (the highest out-degrees after relabelling) come from
  // the shared-memory copy (HOT) or through L1; the rest bypass L1 allocation
  // so they cannot evict the hot lines.
  const uint32_t H = hot;
#pragma unroll
  for (int u = 0; u < IPT; ++u) {
    float x = 0.f;
    if (e0 + u < E) {
      if constexpr (HOT)
        x = (idx[u] < H) ? hot_smem[idx[u]] : ld_gather_cold(cin + idx[u], pol);
      else
        x = (idx[u] < H) ? ld_gather(cin + idx[u], pol) : ld_gather_cold(cin + idx[u], pol);
    }
    v[u] = x;
  }
}

// Reduce the tile in stage s from the gathered values v; returns this thread's
// FP64 |dr| sum. Entry-parallel: thread tid owns entries [tid*IPT, tid*IPT+IPT),
// finds the row of its first entry by binary search, and touches shared memory
// only where a row ends. Rows crossing threads are combined by a block-wide
// segmented scan of (row, partial) carries.
template <int NT, int IPT, bool RAGGED>
__device__ __forceinline__ double reduce_tile(const SweepArgs& a, SweepSmem<NT, IPT>& S, int s, uint32_t t,
                                              const float (&v)[IPT], float* __restrict__ cout, uint64_t pol_keep) {
  const TileMeta  m = S.meta[s];
  // ragged batches: t is the tile list entry; the tile's rows are local ids of its graph
  if (RAGGED) t = m.tile;
  float* const    rank = RAGGED ? a.rank + m.v0 : a.rank;
  const uint32_t* degv = RAGGED ? a.deg + m.v0 : a.deg;
  if (RAGGED) cout += m.v0;
  const int       R = (int)(m.r1 - m.r0), E = (int)(m.k1 - m.k0);
  const uint32_t* rp = S.stage[s] + m.rp_at;  // rp[j] = row_ptr[r0 + j], j = 0..R
  const int       tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int       e0 = tid * IPT;

  uint32_t key = 0xffffffffu;  // row this thread's range ends in (none without entries)
  float    acc = 0.f;
  int      first = -1;         // first row this thread finishes
  if (e0 < E) {
    const int e_end = min(e0 + IPT, E);
    int       lo = 0, hi = R;  // largest i in [0, R] whose start (rp[i] - k0) <= e0
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if ((int)(rp[mid] - m.k0) <= e0)
        lo = mid;
      else
        hi = mid - 1;
    }
    int i = lo;
    int nxt = (i < R) ? (int)(rp[i + 1] - m.k0) : 0x7fffffff;
#pragma unroll
    for (int u = 0; u < IPT; ++u) {
      const int e = e0 + u;
      if (e < e_end) {
        while (e >= nxt) {
          S.z[i] = acc;
          if (first < 0) first = i;
          acc = 0.f;
          ++i;
          nxt = (i < R) ? (int)(rp[i + 1] - m.k0) : 0x7fffffff;
        }
        acc += v[u];
      }
    }
    while (e_end >= nxt) {  // rows ending exactly at the end of this range
      S.z[i] = acc;
      if (first < 0) first = i;
      acc = 0.f;
      ++i;
      nxt = (i < R) ? (int)(rp[i + 1] - m.k0) : 0x7fffffff;
    }
    key = (uint32_t)i;
  }
  // segmented inclusive scan of the carries
  float sv = acc;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t k2 = __shfl_up_sync(kFullMask, key, off);
    const float    v2 = __shfl_up_sync(kFullMask, sv, off);
    if (lane >= off && k2 == key) sv = v2 + sv;
  }
  if (lane == 31) {
    S.wkey[warp] = key;
    S.wsum[warp] = sv;
  }
  __syncthreads();
  // Every warp scans the NW warp totals itself (segmented, shuffles only):
  // wk/wi at lane w = key and block-inclusive carry of warp w's last thread.
  constexpr int NW = SweepSmem<NT, IPT>::NW;
  uint32_t      wk = (lane < NW) ? S.wkey[lane] : 0xfffffffdu;
  float         wi = (lane < NW) ? S.wsum[lane] : 0.f;
#pragma unroll
  for (int off = 1; off < NW; off <<= 1) {
    const uint32_t k2 = __shfl_up_sync(kFullMask, wk, off);
    const float    v2 = __shfl_up_sync(kFullMask, wi, off);
    if (lane >= off && lane < NW && k2 == wk) wi = v2 + wi;
  }
  // carry into this warp from earlier warps, for threads whose key continues it
  const uint32_t prev_wk = __shfl_sync(kFullMask, wk, warp > 0 ? warp - 1 : 0);
  const float    prev_wi = __shfl_sync(kFullMask, wi, warp > 0 ? warp - 1 : 0);
  const float    inc = (warp > 0 && prev_wk == key) ? prev_wi + sv : sv;  // inclusive over the block
  uint32_t       pkey = __shfl_up_sync(kFullMask, key, 1);
  float          pinc = __shfl_up_sync(kFullMask, inc, 1);
  if (lane == 0) {
    pkey = (warp > 0) ? prev_wk : 0xfffffffeu;
    pinc = (warp > 0) ? prev_wi : 0.f;
  }
  if (first >= 0 && pkey == (uint32_t)first) S.z[first] = pinc + S.z[first];
  __syncthreads();

  // epilogue of the rows that start and end in this tile; rows without
  // entries in the tile were never written and sum to zero
  const bool is_cont = rp[0] < m.k0;  // row r0 began in an earlier tile
  const bool has_co = m.k1 > rp[R];   // row r1 continues into the next tile
  double     res = 0.0;
  if (m.rk_at != ~0u) {
    const float*    rk = reinterpret_cast<const float*>(S.stage[s] + m.rk_at);
    const uint32_t* dg = S.stage[s] + m.dg_at;
    for (int j = (is_cont ? 1 : 0) + tid; j < R; j += NT) {
      const uint32_t r = m.r0 + j;
      const float    z = (rp[j + 1] > rp[j]) ? S.z[j] : 0.f;
      const float    nr = fmaf(a.damping, z, RAGGED ? m.base : base_of(a, r));
      st_stream(rank + r, nr);
      st_keep(cout + r, nr / (float)dg[j], pol_keep);
      res += (double)fabsf(nr - rk[j]);
    }
  } else {
    for (int j = (is_cont ? 1 : 0) + tid; j < R; j += NT) {
      const uint32_t r = m.r0 + j;
      const float    z = (rp[j + 1] > rp[j]) ? S.z[j] : 0.f;
      const float    nr = fmaf(a.damping, z, RAGGED ? m.base : base_of(a, r));
      const float    old = ld_stream(rank + r);
      const uint32_t dg = ld_stream(degv + r);
      st_stream(rank + r, nr);
      st_keep(cout + r, nr / (float)dg, pol_keep);
      res += (double)fabsf(nr - old);
    }
  }
  if (tid == 0 && is_cont && R >= 1) a.epart[t] = (rp[1] > m.k0) ? S.z[0] : 0.f;
  if (has_co && E > 0 && tid == (E - 1) / IPT) a.cpart[t] = (key == (uint32_t)R) ? inc : 0.f;
  return res;
}

template <int NT, int IPT, bool RAGGED>
__device__ __forceinline__ void issue_any(const SweepArgs& a, uint32_t t, uint32_t* stg, TileMeta* m, uint64_t* bar,
                                          uint64_t pol) {
  if constexpr (RAGGED)
    issue_ragged_tile<NT, IPT>(a, t, stg, m, bar, pol);
  else
    issue_tile<NT, IPT>(a, t, stg, m, bar, pol);
}

// Ragged batches: the FP64 L1 change of the rows tile t completes goes to
// res_tile[t] (warp sums in shared memory, added in warp order by thread 0
// after the barrier that follows). Every tile belongs to one graph, so the
// per-graph sums need no atomics.
template <int NT, int IPT, bool RAGGED>
__device__ __forceinline__ double tile_residual(SweepSmem<NT, IPT>& S, double r) {
  if constexpr (RAGGED) {
    r = warp_sum_lane0(r);
    if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5] = r;
    return 0.0;
  } else {
    return r;
  }
}
template <int NT, int IPT>
__device__ __forceinline__ void store_tile_residual(const SweepArgs& a, const SweepSmem<NT, IPT>& S, uint32_t t) {
  double b = 0.0;
#pragma unroll
  for (int w = 0; w < SweepSmem<NT, IPT>::NW; ++w) b += S.red[w];
  a.res_tile[t] = b;
}

template <int NT, int IPT, bool HOT, bool RAGGED = false>
__global__ void __launch_bounds__(NT, HOT ? 1 : 4) pr_sweep_kernel(const SweepArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  auto&          S = *reinterpret_cast<SweepSmem<NT, IPT>*>(smem_raw);
  float*         hot_smem = reinterpret_cast<float*>(smem_raw + sizeof(SweepSmem<NT, IPT>));
  const int      tid = threadIdx.x;
  PrState*       st = a.st;

  // Graph loop fail-safe: block 0 clears the loop condition before anything
  // else; only the finishing kernel's last CTA sets it again.
  if (a.use_cond && blockIdx.x == 0 && tid == 0) cudaGraphSetConditional(a.cond, 0u);
  if (*(volatile unsigned int*)&st->done) return;  // stable for the whole sweep

  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  const float* __restrict__ cin = (it & 1ull) ? a.contrib1 : a.contrib0;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const uint64_t pol_keep = policy_evict_last();
  const uint64_t pol_stream = policy_evict_first();
  // ragged batches walk the running graphs' tile list
  const uint32_t G = gridDim.x, T = RAGGED ? *(const volatile uint32_t*)(a.act_off + a.num_graphs) : a.num_tiles;
  double         res = 0.0;
  int            ok = 1;

  if (tid == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
    mbar_init(&S.bar[2], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t t = blockIdx.x;
  if (HOT && t < T && a.hot_ids) {
    // this sweep's contributions of ids [0, hot_ids) into shared memory
    if (tid == 0) {
      const uint32_t bytes = a.hot_ids * 4u;  // hot_ids is a multiple of 4 and <= 256K ids
      mbar_arrive_expect_tx(&S.bar[2], bytes);
      for (uint32_t off = 0; off < bytes; off += 65536u) {
        const uint32_t chunk = (bytes - off) < 65536u ? (bytes - off) : 65536u;
        bulk_load(reinterpret_cast<unsigned char*>(hot_smem) + off, reinterpret_cast<const unsigned char*>(cin) + off,
                  chunk, &S.bar[2], pol_keep);
      }
    }
    ok = mbar_wait(&S.bar[2], 0u);
  }
  if (t < T) {
    if (tid == 0) {
      issue_any<NT, IPT, RAGGED>(a, t, S.stage[0], &S.meta[0], &S.bar[0], pol_stream);
      if (t + G < T) issue_any<NT, IPT, RAGGED>(a, t + G, S.stage[1], &S.meta[1], &S.bar[1], pol_stream);
    }
    float v0[IPT], v1[IPT];
    ok = mbar_wait(&S.bar[0], 0u);
    if (ok)
      gather_tile<NT, IPT, HOT>(S.stage[0], S.meta[0], RAGGED ? cin + S.meta[0].v0 : cin, v0, pol_keep, a.hot_ids,
                                hot_smem);
    ok = __syncthreads_and(ok);
    // two tiles per trip so the register sets alternate without copies
    for (int i = 0; ok && t < T; i += 2) {
      // even tile t in stage 0 (values v0); prefetch tile t+G into v1
      uint32_t tn = t + G;
      if (tn < T) {
        ok = mbar_wait(&S.bar[1], (uint32_t)(i >> 1) & 1u);
        if (ok)
          gather_tile<NT, IPT, HOT>(S.stage[1], S.meta[1], RAGGED ? cin + S.meta[1].v0 : cin, v1, pol_keep, a.hot_ids,
                                    hot_smem);
      }
      res += tile_residual<NT, IPT, RAGGED>(S, reduce_tile<NT, IPT, RAGGED>(a, S, 0, t, v0, cout, pol_keep));
      ok = __syncthreads_and(ok);
      if (RAGGED && tid == 0) store_tile_residual<NT, IPT>(a, S, S.meta[0].tile);
      if (ok && tid == 0 && t + 2 * G < T)
        issue_any<NT, IPT, RAGGED>(a, t + 2 * G, S.stage[0], &S.meta[0], &S.bar[0], pol_stream);
      t = tn;
      if (!ok || t >= T) break;
      // odd tile t in stage 1 (values v1); prefetch tile t+G into v0
      tn = t + G;
      if (tn < T) {
        ok = mbar_wait(&S.bar[0], (uint32_t)((i >> 1) + 1) & 1u);
        if (ok)
          gather_tile<NT, IPT, HOT>(S.stage[0], S.meta[0], RAGGED ? cin + S.meta[0].v0 : cin, v0, pol_keep, a.hot_ids,
                                    hot_smem);
      }
      res += tile_residual<NT, IPT, RAGGED>(S, reduce_tile<NT, IPT, RAGGED>(a, S, 1, t, v1, cout, pol_keep));
      ok = __syncthreads_and(ok);
      if (RAGGED && tid == 0) store_tile_residual<NT, IPT>(a, S, S.meta[1].tile);
      if (ok && tid == 0 && t + 2 * G < T)
        issue_any<NT, IPT, RAGGED>(a, t + 2 * G, S.stage[1], &S.meta[1], &S.bar[1], pol_stream);
      t = tn;
    }
  }

  if constexpr (RAGGED) {  // residuals went to res_tile; thread 0 may still be reading S.red
    if (tid == 0 && !ok) atomicOr(&st->fault, 1u);
    return;
  }
  // FP64 residual: fixed-order block reduction, one partial per CTA.
  res = warp_sum_lane0(res);
  if ((tid & 31) == 0) S.red[tid >> 5] = res;
  __syncthreads();
  if (tid == 0) {
    double b = 0.0;
#pragma unroll
    for (int w = 0; w < SweepSmem<NT, IPT>::NW; ++w) b += S.red[w];
    a.res_part[blockIdx.x] = b;
    if (!ok) atomicOr(&st->fault, 1u);
  }
}

// Epilogue of one row read straight from global memory.
__device__ __forceinline__ double row_epilogue(const SweepArgs& a, float* cout, uint32_t r, float z, uint64_t pol) {
  const float nr = fmaf(a.damping, z, base_of(a, r));
  const float old = a.rank[r];
  a.rank[r] = nr;
  st_keep(cout + r, nr / (float)a.deg[r], pol);
  return (double)fabsf(nr - old);
}

// Rows that cross tile boundaries, the residual and the convergence test.
// Thread ta handles the row carried out of tile ta when that row starts there.
__global__ void __launch_bounds__(256) pr_finish_kernel(const SweepArgs a) {
  __shared__ double s_red[8];
  __shared__ int    s_last;
  PrState*          st = a.st;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const uint64_t pol = policy_evict_last();
  const uint32_t D = a.tile_items, T = a.num_tiles;
  const int      tid = threadIdx.x, lane = tid & 31;
  double         res = 0.0;

  const uint32_t ta = blockIdx.x * blockDim.x + tid;
  uint32_t       S = 0, tb = 0;
  bool           mine = false;
  if (ta + 1 < T) {
    S = a.tile_row[ta + 1];
    const uint32_t k1 = a.tile_nnz[ta + 1], rs = a.row_ptr[S];
    if (k1 > rs && ((uint64_t)S + rs) / D == ta) {
      mine = true;
      tb = (uint32_t)(((uint64_t)S + a.row_ptr[S + 1]) / D);
    }
  }
  const bool longspan = mine && (tb - ta > 8u);
  if (mine && !longspan) {
    float z = 0.f;
    for (uint32_t u = ta; u < tb; ++u) z += __ldcg(a.cpart + u);
    z += __ldcg(a.epart + tb);
    res += row_epilogue(a, cout, S, z, pol);
  }
  unsigned mask = __ballot_sync(kFullMask, longspan);
  while (mask) {
    const int src = __ffs(mask) - 1;
    mask &= mask - 1;
    const uint32_t sS = __shfl_sync(kFullMask, S, src);
    const uint32_t sa = __shfl_sync(kFullMask, ta, src);
    const uint32_t sb = __shfl_sync(kFullMask, tb, src);
    float          p = 0.f;
    for (uint32_t u = sa + lane; u < sb; u += 32) p += __ldcg(a.cpart + u);
    p = warp_sum_lane0(p);
    if (lane == 0) res += row_epilogue(a, cout, sS, p + __ldcg(a.epart + sb), pol);
  }

  res = warp_sum_lane0(res);
  if (lane == 0) s_red[tid >> 5] = res;
  __syncthreads();
  if (tid == 0) {
    double b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += s_red[w];
    a.res_part[a.sweep_grid + blockIdx.x] = b;
    __threadfence();
    const unsigned prev = atomicAdd(&st->ticket, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last || tid >= 32) return;

  // Last CTA: reduce all partials in a fixed order and test convergence.
  __threadfence();
  const uint32_t parts = a.sweep_grid + gridDim.x;
  double         e = 0.0;
  for (uint32_t u = lane; u < parts; u += 32) e += __ldcg(a.res_part + u);
  e = warp_sum_lane0(e);
  if (lane == 0) {
    const unsigned long long done_iters = it + 1ull;
    st->iter = done_iters;
    st->last_error = e;
    if (a.err_hist && it < a.err_cap) a.err_hist[it] = e;  // the first err_cap sweeps
    const bool conv = e < st->threshold;
    const bool abort = a.abort_word && *a.abort_word;
    const bool fault = *(volatile unsigned int*)&st->fault != 0u;
    const bool done = conv || done_iters >= st->max_iters || abort || fault;
    st->converged = conv ? 1u : 0u;
    st->aborted = (abort && !conv) ? 1u : 0u;
    st->done = done ? 1u : 0u;
    st->ticket = 0u;
    __threadfence();
    if (a.use_cond && !done && done_iters < st->chunk_end) cudaGraphSetConditional(a.cond, 1u);
  }
}

// ---------------------------------------------------------------------------
// Ragged batches: rows crossing tiles, per-graph convergence, set-up
// ---------------------------------------------------------------------------
// Thread i takes entry i of the running graphs' tile list, tile ta, and
// completes the row carried out of ta when that row starts there (local
// merge-path coordinates of the tile's graph; rows never cross graphs),
// adding its L1 change to res_tile[ta]. Spans of more than 8 tiles are summed
// by the whole warp.
__global__ void __launch_bounds__(256) pr_ragged_finish_kernel(const SweepArgs a) {
  if (*(volatile unsigned int*)&a.st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&a.st->iter;
  float* __restrict__ cout = (it & 1ull) ? a.contrib0 : a.contrib1;
  const uint64_t pol = policy_evict_last();
  const uint32_t D = a.tile_items;
  const int      lane = threadIdx.x & 31;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // entry of the running graphs' tile list
  const uint32_t L = *(const volatile uint32_t*)(a.act_off + a.num_graphs);
  uint32_t       S = 0, ta = 0, tb = 0, g = 0;
  bool           mine = false;
  if (i < L) {
    const uint2 tg = __ldcg(a.act_list + i);
    ta = tg.x;
    g = tg.y;
    const RaggedGraph& G = a.graphs[g];
    const uint32_t*    rp = a.row_ptr + G.p0;
    S = a.tile_row[ta + g + 1];  // the tile's end; S = n at the graph's last tile
    const uint32_t k1 = a.tile_nnz[ta + g + 1], rs = rp[S];
    if (k1 > rs && ((uint64_t)S + rs) / D == ta - G.tile0) {
      mine = true;
      tb = G.tile0 + (uint32_t)(((uint64_t)S + rp[S + 1]) / D);
    }
  }
  const bool longspan = mine && (tb - ta > 8u);
  float      z = 0.f;
  if (mine && !longspan) {
    for (uint32_t u = ta; u < tb; ++u) z += __ldcg(a.cpart + u);
    z += __ldcg(a.epart + tb);
  }
  unsigned mask = __ballot_sync(kFullMask, longspan);
  while (mask) {
    const int src = __ffs(mask) - 1;
    mask &= mask - 1;
    const uint32_t sa = __shfl_sync(kFullMask, ta, src);
    const uint32_t sb = __shfl_sync(kFullMask, tb, src);
    float          p = 0.f;
    for (uint32_t u = sa + lane; u < sb; u += 32) p += __ldcg(a.cpart + u);
    p = __shfl_sync(kFullMask, warp_sum_lane0(p), 0);
    if (lane == src) z = p + __ldcg(a.epart + sb);
  }
  if (mine) {
    const uint64_t v = a.graphs[g].v0 + S;
    const float    nr = fmaf(a.damping, z, a.graph_base[g]);
    const float    old = a.rank[v];
    a.rank[v] = nr;
    st_keep(cout + v, nr / (float)a.deg[v], pol);
    a.res_tile[ta] += (double)fabsf(nr - old);
  }
}

// One warp per running graph: its sweep error is the sum of its tiles'
// residuals in tile order (lane-strided FP64 partials, then a fixed shuffle
// tree); the graph stops on err < threshold, at max_iters, or when the solve
// is aborted or failed. The last CTA rebuilds the running graphs' tile list
// offsets for the next sweep, advances the sweep count, records the summed
// error of the sweep and ends the loop once no graph is running.
__global__ void __launch_bounds__(256) pr_ragged_converge_kernel(const SweepArgs a, uint32_t num_graphs,
                                                                 RaggedState rs) {
  __shared__ double   s_err[8];
  __shared__ uint32_t s_run[8];
  __shared__ int      s_last;
  PrState*            st = a.st;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  const int                tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool               abort = a.abort_word && *a.abort_word;
  const bool               fault = *(volatile unsigned int*)&st->fault != 0u;
  const bool               last_sweep = it + 1ull >= st->max_iters;
  const double             thr = st->threshold;
  double                   esum = 0.0;
  uint32_t                 running = 0;
  const uint32_t           nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t g = blockIdx.x * (blockDim.x >> 5) + warp; g < num_graphs; g += nwarps) {
    if (rs.done[g]) continue;
    const uint32_t t0 = a.graphs[g].tile0, nt = a.graphs[g].tiles;
    double         e = 0.0;
    for (uint32_t u = lane; u < nt; u += 32) e += __ldcg(a.res_tile + t0 + u);
    e = warp_sum_lane0(e);
    if (lane == 0) {
      const bool conv = e < thr;
      const bool more = !conv && !last_sweep;  // the graph would take another sweep
      rs.iters[g] = (uint32_t)(it + 1ull);
      rs.err[g] = e;
      rs.conv[g] = conv ? 1u : 0u;
      rs.done[g] = (more && !abort && !fault) ? 0u : 1u;
      esum += e;
      running += more ? 1u : 0u;
    }
  }
  if (lane == 0) {
    s_err[warp] = esum;
    s_run[warp] = running;
  }
  __syncthreads();
  if (tid == 0) {
    double   b = 0.0;
    uint32_t r = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      b += s_err[w];
      r += s_run[w];
    }
    a.res_part[blockIdx.x] = b;
    if (r) atomicAdd(&st->pending, r);
    __threadfence();
    const unsigned prev = atomicAdd(&st->ticket, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  {
    // act_off = exclusive scan over the graphs of (running ? tiles : 0):
    // thread tid owns graphs [tid * per, tid * per + per)
    __shared__ uint32_t s_wsum[8];
    const uint32_t      per = (num_graphs + blockDim.x - 1) / blockDim.x;
    const uint32_t      g0 = tid * per, g1 = min(num_graphs, g0 + per);
    uint32_t            mine = 0;
    for (uint32_t g = g0; g < g1; ++g) mine += *(volatile uint32_t*)(rs.done + g) ? 0u : a.graphs[g].tiles;
    uint32_t incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += s_wsum[w];
    uint32_t off = before + incl - mine;
    for (uint32_t g = g0; g < g1; ++g) {
      rs.act_off[g] = off;
      off += *(volatile uint32_t*)(rs.done + g) ? 0u : a.graphs[g].tiles;
    }
    if (tid == blockDim.x - 1) rs.act_off[num_graphs] = before + incl;
  }
  if (tid >= 32) return;
  double e = 0.0;
  for (uint32_t u = lane; u < gridDim.x; u += 32) e += __ldcg(a.res_part + u);
  e = warp_sum_lane0(e);
  if (lane == 0) {
    const unsigned long long done_iters = it + 1ull;
    const unsigned int       pending = *(volatile unsigned int*)&st->pending;
    st->iter = done_iters;
    st->last_error = e;
    if (a.err_hist && it < a.err_cap) a.err_hist[it] = e;  // the first err_cap sweeps
    const bool done = pending == 0u || done_iters >= st->max_iters || abort || fault;
    st->converged = 0u;
    st->aborted = (abort && pending) ? 1u : 0u;  // graphs were still running
    st->done = done ? 1u : 0u;
    st->pending = 0u;
    st->ticket = 0u;
    __threadfence();
    if (a.use_cond && !done && done_iters < st->chunk_end) cudaGraphSetConditional(a.cond, 1u);
  }
}

// One warp per running graph writes its entries of the tile list.
__global__ void ragged_list_kernel(const RaggedGraph* __restrict__ graphs, uint32_t num_graphs,
                                   const uint32_t* __restrict__ done, const uint32_t* __restrict__ act_off,
                                   uint2* __restrict__ list) {
  const uint32_t lane = threadIdx.x & 31, nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < num_graphs; g += nwarps) {
    if (done[g]) continue;
    const uint32_t t0 = graphs[g].tile0, nt = graphs[g].tiles, o = act_off[g];
    for (uint32_t j = lane; j < nt; j += 32) list[o + j] = make_uint2(t0 + j, g);
  }
}

// rank_v = 1/n_g (page_rank.hpp:100-104 per graph), contrib_v = rank_v / deg_v;
// thread v finds its graph by binary search over the graphs' first vertices.
// One warp per graph (grid-strided) sets the base term (1 - d)/n_g and resets
// the graph's state: stopped = `stopped` (max_iters == 0), no sweeps yet.
__global__ void ragged_init_kernel(const SweepArgs a, RaggedState rs, uint32_t num_graphs, uint64_t nv, float damping,
                                   uint32_t stopped, float* __restrict__ base) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t g = tid; g < num_graphs; g += stride) {
    const uint32_t n = a.graphs[g].n;
    // page_rank.hpp:93-94: constants in double, stored as float
    base[g] = n ? (float)((1.0 - (double)damping) / (double)n) : 0.f;
    rs.done[g] = stopped;
    rs.iters[g] = 0u;
    rs.err[g] = 0.0;
    rs.conv[g] = 0u;
  }
  for (uint64_t v = tid; v < nv; v += stride) {
    uint32_t lo = 0, hi = num_graphs - 1;  // last graph whose first vertex is <= v
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (a.graphs[mid].v0 <= v)
        lo = mid;
      else
        hi = mid - 1;
    }
    const float r = (float)(1.0 / (double)a.graphs[lo].n);
    a.rank[v] = r;
    a.contrib0[v] = r / (float)a.deg[v];
  }
}

// ---------------------------------------------------------------------------
// Solve set-up kernels
// ---------------------------------------------------------------------------
__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx,
                                  uint32_t* __restrict__ dst, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[idx[i]];
}
__global__ void gather_f32_kernel(const float* __restrict__ src, const uint32_t* __restrict__ idx,
                                  float* __restrict__ dst, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[idx[i]];
}

cudaError_t launch_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint64_t n, int sms,
                              cudaStream_t s) {
  if (!n) return cudaSuccess;
  gather_u32_kernel<<<sms * 8, 256, 0, s>>>(src, idx, dst, n);
  return cudaGetLastError();
}
cudaError_t launch_gather_f32(const float* src, const uint32_t* idx, float* dst, uint64_t n, int sms, cudaStream_t s) {
  if (!n) return cudaSuccess;
  gather_f32_kernel<<<sms * 8, 256, 0, s>>>(src, idx, dst, n);
  return cudaGetLastError();
}

// rank = r0 (1/n, or the one-hot seed), contrib = rank / deg
// (page_rank.hpp:100-104 and page_rank_v10's first :401-405).
__global__ void pr_init_kernel(float* __restrict__ rank, float* __restrict__ contrib, const uint32_t* __restrict__ deg,
                               uint64_t n, float init, int teleport, uint32_t seed) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float r = (teleport == kTeleportSeed) ? ((i == seed) ? 1.0f : 0.0f) : init;
    rank[i] = r;
    contrib[i] = r / (float)deg[i];
  }
}

cudaError_t launch_pr_init(const SweepArgs& a, uint64_t n, float init, int sms, cudaStream_t s) {
  if (!n) return cudaSuccess;
  pr_init_kernel<<<sms * 8, 256, 0, s>>>(a.rank, a.contrib0, a.deg, n, init, a.teleport, a.seed);
  return cudaGetLastError();
}

__global__ void residual_init_kernel(float* __restrict__ rank, float* __restrict__ delta, const uint32_t* __restrict__ deg,
                                     uint64_t n, float r0, float damping, int push, unsigned int* pushed) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned int   cnt = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t dg = deg[i];
    const bool     moved = push && dg > 0u;
    rank[i] = push ? r0 : 0.f;
    delta[i] = moved ? r0 * damping / (float)dg : 0.f;
    cnt += moved ? 1u : 0u;
  }
  cnt = __reduce_add_sync(kFullMask, cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(pushed, cnt);
}

cudaError_t launch_residual_init(float* rank, float* delta, const uint32_t* deg, uint64_t n, float r0, float damping,
                                 bool push, unsigned int* pushed, int sms, cudaStream_t s) {
  residual_init_kernel<<<sms * 8, 256, 0, s>>>(rank, delta, deg, n, r0, damping, push ? 1 : 0, pushed);
  return cudaGetLastError();
}

// Sets the sweep bound of one graph launch (first node of the graph).
__global__ void pr_arm_kernel(PrState* st) { st->chunk_end = st->iter + kGraphChunk; }

cudaError_t add_pr_arm_node(cudaGraph_t g, PrState* st, cudaGraphNode_t* node) {
  cudaKernelNodeParams kp = {};
  void*                args[] = {(void*)&st};
  kp.func = (void*)pr_arm_kernel;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(1);
  kp.kernelParams = args;
  return cudaGraphAddKernelNode(node, g, nullptr, 0, &kp);
}

// ---------------------------------------------------------------------------
// Dispatch over the items-per-thread variants
// ---------------------------------------------------------------------------
// Variants: (threads, IPT, hot-in-shared-memory).
struct VariantEntry {
  int    threads, ipt;
  bool   hot;
  void*  fn;
  size_t fixed_smem;
};

template <int NT, int IPT, bool HOT>
static VariantEntry entry() {
  return {NT, IPT, HOT, (void*)pr_sweep_kernel<NT, IPT, HOT>, sizeof(SweepSmem<NT, IPT>)};
}

static const VariantEntry* find_variant(const SweepVariant& v) {
  static const VariantEntry table[] = {entry<256, 4, false>(),  entry<256, 8, false>(),  entry<256, 12, false>(),
                                       entry<256, 16, false>(), entry<1024, 4, true>(),  entry<512, 8, true>(),
                                       entry<1024, 8, true>()};
  for (const auto& e : table)
    if (e.threads == v.threads && e.ipt == v.ipt && e.hot == v.hot_smem) return &e;
  return nullptr;
}

static int max_dyn_smem() {
  int dev = 0, bytes = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) bytes = 232448;
  return bytes;
}

bool sweep_variant_supported(const SweepVariant& v) { return find_variant(v) != nullptr; }

uint32_t sweep_hot_capacity(const SweepVariant& v) {
  const VariantEntry* e = find_variant(v);
  if (!e || !e->hot) return 0;
  const long spare = (long)max_dyn_smem() - (long)e->fixed_smem - 1024;
  if (spare <= 0) return 0;
  uint32_t ids = (uint32_t)(spare / 4);
  ids &= ~31u;
  return ids > 262144u ? 262144u : ids;
}

size_t sweep_smem_bytes(const SweepVariant& v, uint32_t hot_ids) {
  const VariantEntry* e = find_variant(v);
  if (!e) return 0;
  return e->fixed_smem + (e->hot ? (size_t)hot_ids * 4u : 0u);
}

cudaError_t configure_sweep_kernels() {
  static const SweepVariant all[] = {{256, 4, false}, {256, 8, false}, {256, 12, false}, {256, 16, false},
                                     {1024, 4, true}, {512, 8, true},  {1024, 8, true}};
  const int maxb = max_dyn_smem();
  for (const auto& v : all) {
    const VariantEntry* e = find_variant(v);
    cudaError_t         err = cudaFuncSetAttribute(e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   e->hot ? maxb : (int)e->fixed_smem);
    if (err != cudaSuccess) return err;
  }
  return cudaFuncSetAttribute((void*)pr_sweep_kernel<256, 8, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sizeof(SweepSmem<256, 8>));
}

cudaError_t set_sweep_carveout(const SweepVariant& v, int percent) {
  const VariantEntry* e = find_variant(v);
  if (!e) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(e->fn, cudaFuncAttributePreferredSharedMemoryCarveout, percent);
}

int sweep_blocks_per_sm(const SweepVariant& v, uint32_t hot_ids) {
  const VariantEntry* e = find_variant(v);
  int                 nb = 0;
  if (!e ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e->fn, e->threads, sweep_smem_bytes(v, hot_ids)) != cudaSuccess)
    return 1;
  return nb > 0 ? nb : 1;
}

int finish_grid_for(uint32_t num_tiles) { return num_tiles ? (int)((num_tiles + 255u) / 256u) : 1; }

cudaError_t launch_pr_sweep(const SweepArgs& a, const SweepVariant& v, int grid, cudaStream_t s) {
  const VariantEntry* e = find_variant(v);
  if (!e) return cudaErrorInvalidValue;
  void* args[] = {(void*)&a};
  return cudaLaunchKernel(e->fn, dim3((unsigned)grid), dim3(e->threads), args, sweep_smem_bytes(v, a.hot_ids), s);
}

cudaError_t launch_pr_finish(const SweepArgs& a, int grid, cudaStream_t s) {
  pr_finish_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t add_pr_sweep_nodes(cudaGraph_t body, const SweepArgs& a, const SweepVariant& v, int sweep_grid,
                               int finish_grid) {
  const VariantEntry* ve = find_variant(v);
  if (!ve) return cudaErrorInvalidValue;
  void*                args[] = {(void*)&a};
  cudaKernelNodeParams kp = {};
  kp.func = ve->fn;
  kp.gridDim = dim3((unsigned)sweep_grid);
  kp.blockDim = dim3(ve->threads);
  kp.sharedMemBytes = (unsigned)sweep_smem_bytes(v, a.hot_ids);
  kp.kernelParams = args;
  cudaGraphNode_t sweep_node, finish_node;
  cudaError_t     e = cudaGraphAddKernelNode(&sweep_node, body, nullptr, 0, &kp);
  if (e != cudaSuccess) return e;
  cudaKernelNodeParams fp = {};
  fp.func = (void*)pr_finish_kernel;
  fp.gridDim = dim3((unsigned)finish_grid);
  fp.blockDim = dim3(256);
  fp.kernelParams = args;
  return cudaGraphAddKernelNode(&finish_node, body, &sweep_node, 1, &fp);
}

// ---------------------------------------------------------------------------
// Ragged batches: launches
// ---------------------------------------------------------------------------
static void* ragged_sweep_fn() { return (void*)pr_sweep_kernel<256, 8, false, true>; }
static size_t ragged_sweep_smem() { return sizeof(SweepSmem<256, 8>); }

static int ragged_list_grid(uint32_t num_graphs) { return (int)((num_graphs + 7) / 8 < 4096 ? (num_graphs + 7) / 8 : 4096); }

cudaError_t launch_ragged_list(const SweepArgs& a, const RaggedState& rs, int sms, cudaStream_t s) {
  (void)sms;
  ragged_list_kernel<<<ragged_list_grid(a.num_graphs), 256, 0, s>>>(a.graphs, a.num_graphs, rs.done, rs.act_off,
                                                                     rs.act_list);
  return cudaGetLastError();
}

cudaError_t launch_ragged_sweep(const SweepArgs& a, int sweep_grid, int finish_grid, uint32_t num_graphs,
                                const RaggedState& rs, int conv_grid, cudaStream_t s) {
  void*       args[] = {(void*)&a};
  cudaError_t e = cudaLaunchKernel(ragged_sweep_fn(), dim3((unsigned)sweep_grid), dim3(256), args, ragged_sweep_smem(), s);
  if (e != cudaSuccess) return e;
  pr_ragged_finish_kernel<<<finish_grid, 256, 0, s>>>(a);
  pr_ragged_converge_kernel<<<conv_grid, 256, 0, s>>>(a, num_graphs, rs);
  ragged_list_kernel<<<ragged_list_grid(num_graphs), 256, 0, s>>>(a.graphs, num_graphs, rs.done, rs.act_off,
                                                                   rs.act_list);
  return cudaGetLastError();
}

cudaError_t add_ragged_nodes(cudaGraph_t body, const SweepArgs& a, int sweep_grid, int finish_grid, uint32_t num_graphs,
                             const RaggedState& rs, int conv_grid) {
  void*                sargs[] = {(void*)&a};
  cudaKernelNodeParams kp = {};
  kp.func = ragged_sweep_fn();
  kp.gridDim = dim3((unsigned)sweep_grid);
  kp.blockDim = dim3(256);
  kp.sharedMemBytes = (unsigned)ragged_sweep_smem();
  kp.kernelParams = sargs;
  cudaGraphNode_t sweep_node, finish_node, conv_node;
  cudaError_t     e = cudaGraphAddKernelNode(&sweep_node, body, nullptr, 0, &kp);
  if (e != cudaSuccess) return e;
  cudaKernelNodeParams fp = {};
  fp.func = (void*)pr_ragged_finish_kernel;
  fp.gridDim = dim3((unsigned)finish_grid);
  fp.blockDim = dim3(256);
  fp.kernelParams = sargs;
  e = cudaGraphAddKernelNode(&finish_node, body, &sweep_node, 1, &fp);
  if (e != cudaSuccess) return e;
  RaggedState          r = rs;
  uint32_t             ng = num_graphs;
  void*                cargs[] = {(void*)&a, (void*)&ng, (void*)&r};
  cudaKernelNodeParams cp = {};
  cp.func = (void*)pr_ragged_converge_kernel;
  cp.gridDim = dim3((unsigned)conv_grid);
  cp.blockDim = dim3(256);
  cp.kernelParams = cargs;
  e = cudaGraphAddKernelNode(&conv_node, body, &finish_node, 1, &cp);
  if (e != cudaSuccess) return e;
  const RaggedGraph*   gr = a.graphs;
  const uint32_t*      dn = rs.done;
  const uint32_t*      ao = rs.act_off;
  uint2*               al = rs.act_list;
  void*                largs[] = {(void*)&gr, (void*)&ng, (void*)&dn, (void*)&ao, (void*)&al};
  cudaKernelNodeParams lp = {};
  lp.func = (void*)ragged_list_kernel;
  lp.gridDim = dim3((unsigned)ragged_list_grid(num_graphs));
  lp.blockDim = dim3(256);
  lp.kernelParams = largs;
  cudaGraphNode_t list_node;
  return cudaGraphAddKernelNode(&list_node, body, &conv_node, 1, &lp);
}

cudaError_t launch_ragged_init(const SweepArgs& a, const RaggedState& rs, uint32_t num_graphs, uint64_t num_vertices,
                               float damping, uint32_t stopped, int sms, cudaStream_t s) {
  if (!num_graphs) return cudaSuccess;
  ragged_init_kernel<<<sms * 8, 256, 0, s>>>(a, rs, num_graphs, num_vertices, damping, stopped,
                                              const_cast<float*>(a.graph_base));
  return cudaGetLastError();
}

}  // namespace nwgpu

// ---------------------------------------------------------------------------
// Self-test of the bounded wait: one thread waits on an mbarrier that nothing
// ever completes, with the sweeps' wait loop, and reports that it gave up.
// ---------------------------------------------------------------------------
namespace {
__device__ unsigned int g_wait_selftest;

__global__ void bounded_wait_selftest_kernel(uint32_t polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    nwgpu::mbar_init(&bar, 1);
    nwgpu::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) g_wait_selftest = nwgpu::mbar_wait_n(&bar, 0u, polls) ? 0u : 1u;
}
}  // namespace

namespace nwgpu {
cudaError_t run_wait_selftest(uint32_t polls, unsigned int* gave_up, float* ms) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const unsigned int unset = 7u;  // neither answer, so a kernel that did not run shows
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_wait_selftest, &unset, sizeof(unset));
  if (e == cudaSuccess) e = cudaEventRecord(e0);
  if (e == cudaSuccess) {
    bounded_wait_selftest_kernel<<<1, 32>>>(polls);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaMemcpyFromSymbol(gave_up, g_wait_selftest, sizeof(unsigned int));
  if (e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return e;
}
}  // namespace nwgpu
