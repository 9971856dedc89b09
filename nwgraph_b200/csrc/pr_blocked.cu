// Destination-blocked PageRank sweep, sm_100a.
//
// The pull gather of page_rank (include/nwgraph/algorithms/page_rank.hpp:
// 129-131) reads contrib[col[k]] for the entries of each row in turn: random
// 4-byte loads, each a separate 128-byte line lookup in the SM's L1TEX stage,
// which caps a row-order sweep at about one lookup per SM per clock. This
// sweep reorders the entries instead. The rows are cut into blocks of
// kBlockRows consecutive rows; a block's entries are stored sorted by their
// source (column id), as (source, row within the block) pairs. A CTA takes a
// block, zeroes its row sums in shared memory, and walks the block's entries
// in source order: consecutive lanes read contributions of nearby sources
// (mostly the same 128-byte line) and add them into the row sums of their
// rows with shared-memory atomics. The contribution vector is read about once
// per block in address order instead of once per entry at random.
//
// Row sums are 64-bit fixed point, contrib * 2^62 rounded to an integer, so
// their sums are exact and independent of the order in which the CTA's
// threads add them: the ranks are bit-reproducible whatever the scheduling,
// and each row sum is rounded once to FP32 (the reference rounds after every
// addition of its serial sum). A contribution is at most 1 (ranks sum to at
// most 1 with the reference's leak semantics, page_rank.hpp:94,133) and so is
// a row sum, so the integers stay below 2^62; a term loses at most 2^-63 to
// rounding.
//
// Blocks with more entries than the piece size are cut into several work
// items (pieces) of consecutive entries; each piece adds its shared-memory
// sums into a global fixed-point accumulator, and the last piece to finish (a
// per-block ticket) runs the block's epilogue from it and clears it. Items
// are handed out largest first from an atomic counter. Each block's FP64 L1
// change goes to res_blk[block]; the finishing kernel sums them in block
// order and runs the convergence test on the device (page_rank.hpp:125-144).
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "blocked.h"
#include "common.cuh"

namespace nwgpu {

namespace {

constexpr float kFix = 0x1p62f;     // contribution -> fixed point
constexpr float kUnfix = 0x1p-62f;  // fixed point -> row sum

__device__ __forceinline__ float blocked_base(const SweepArgs& a, uint32_t r) {
  if (a.teleport == kTeleportSeed) return (r == a.seed) ? a.base : 0.f;
  return a.base;
}

__device__ __forceinline__ uint32_t ld_stream_u16(const uint16_t* p) { return (uint32_t)__ldcs(p); }

// Block-wide FP64 sum in a fixed order (thread-strided partials, then a fixed
// tree over the warps); valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* s_red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum_lane0(v);
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = (lane < (int)(blockDim.x >> 5)) ? s_red[lane] : 0.0;
    t = warp_sum_lane0(t);
  }
  __syncthreads();
  return t;
}

// The epilogue of one row from its fixed-point sum: page_rank_v10's update
// (experimental/algorithms/page_rank.hpp:417-418) fused with the next sweep's
// contribution (:401-405).
__device__ __forceinline__ double row_update(const BlockedArgs& a, float* __restrict__ cout, uint32_t r,
                                             unsigned long long acc, uint64_t pol) {
  const float z = __ll2float_rn((long long)acc) * kUnfix;
  const float nr = fmaf(a.sw.damping, z, blocked_base(a.sw, r));
  const float old = ld_stream(a.sw.rank + r);
  const uint32_t dg = ld_stream(a.sw.deg + r);
  st_stream(a.sw.rank + r, nr);
  st_keep(cout + r, nr / (float)dg, pol);
  return (double)fabsf(nr - old);
}

}  // namespace

// Adds the contributions of entries [e0, e1) of block b into the row sums,
// LOADS entries in flight per thread. Unpacked: thread t takes entries
// e0 + t + 1024 u. Packed: warp w takes the block's 32-entry groups
// g0 + w + 32 u, one entry per lane; the group's base word is one broadcast
// load per warp.
template <int LOADS, bool PACKED>
__device__ __forceinline__ void accumulate(const BlockedArgs& a, const float* __restrict__ cin, uint32_t b,
                                           uint32_t e0, uint32_t e1, unsigned long long* s_acc) {
  const int tid = threadIdx.x;
  if constexpr (!PACKED) {
#pragma unroll 1
    for (uint32_t base = e0 + (uint32_t)tid; base < e1; base += kBlockedThreads * LOADS) {
      uint32_t s[LOADS], d[LOADS];
#pragma unroll
      for (int u = 0; u < LOADS; ++u) {
        const uint32_t e = base + (uint32_t)u * kBlockedThreads;
        s[u] = (e < e1) ? ld_stream(a.src + e) : 0u;
        d[u] = (e < e1) ? ld_stream_u16(a.dst + e) : 0u;
      }
      float v[LOADS];
#pragma unroll
      for (int u = 0; u < LOADS; ++u) {
        const uint32_t e = base + (uint32_t)u * kBlockedThreads;
        v[u] = (e < e1) ? __ldg(cin + s[u]) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < LOADS; ++u) {
        const uint32_t e = base + (uint32_t)u * kBlockedThreads;
        if (e < e1) atomicAdd(s_acc + d[u], (unsigned long long)__float2ll_rn(v[u] * kFix));
      }
    }
  } else {
    const int      lane = tid & 31, warp = tid >> 5;
    const uint32_t be0 = a.blk_e0[b], bg0 = a.blk_g0[b];
    const uint32_t g_lo = (e0 - be0) >> 5, g_hi = (e1 - be0 + 31u) >> 5;  // the item's groups (block-relative)
#pragma unroll 1
    for (uint32_t g = g_lo + (uint32_t)warp; g < g_hi; g += 32u * LOADS) {
      uint32_t word[LOADS], gb[LOADS];
#pragma unroll
      for (int u = 0; u < LOADS; ++u) {
        const uint32_t gg = g + (uint32_t)u * 32u;
        const uint32_t e = be0 + gg * 32u + (uint32_t)lane;
        word[u] = (gg < g_hi && e < e1) ? ld_stream(a.src + e) : 0u;
        gb[u] = (gg < g_hi) ? __ldg(a.gbase + bg0 + gg) : 0u;
      }
      float v[LOADS];
      uint32_t d[LOADS];
#pragma unroll
      for (int u = 0; u < LOADS; ++u) {
        const uint32_t gg = g + (uint32_t)u * 32u;
        const uint32_t e = be0 + gg * 32u + (uint32_t)lane;
        const bool     ok = gg < g_hi && e < e1;
        uint32_t       src;
        if (gb[u] & kWideGroup)  // warp-uniform
          src = ok ? __ldg(a.wide + (size_t)(gb[u] & ~kWideGroup) * 32u + (uint32_t)lane) : 0u;
        else
          src = gb[u] + (word[u] >> kPackRowBits);
        d[u] = word[u] & ((1u << kPackRowBits) - 1u);
        v[u] = ok ? __ldg(cin + src) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < LOADS; ++u) {
        const uint32_t gg = g + (uint32_t)u * 32u;
        const uint32_t e = be0 + gg * 32u + (uint32_t)lane;
        if (gg < g_hi && e < e1) atomicAdd(s_acc + d[u], (unsigned long long)__float2ll_rn(v[u] * kFix));
      }
    }
  }
}

// LOADS: entries in flight per thread; PACKED: the 4-byte entry format.
template <int LOADS, bool PACKED>
__global__ void __launch_bounds__(kBlockedThreads, 1) pr_blocked_sweep_kernel(const BlockedArgs a) {
  extern __shared__ unsigned long long s_acc[];  // kBlockRows row sums
  __shared__ double   s_red[32];
  __shared__ uint32_t s_item;
  __shared__ int      s_last;
  const int           tid = threadIdx.x;
  PrState*            st = a.sw.st;
  if (a.sw.use_cond && blockIdx.x == 0 && tid == 0) cudaGraphSetConditional(a.sw.cond, 0u);
  if (*(volatile unsigned int*)&st->done) return;
  if (*(volatile unsigned int*)&st->fault) return;  // degrees below the entry counts: the finishing kernel stops
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  const float* __restrict__ cin = (it & 1ull) ? a.sw.contrib1 : a.sw.contrib0;
  float* __restrict__ cout = (it & 1ull) ? a.sw.contrib0 : a.sw.contrib1;
  const uint64_t pol = policy_evict_last();

#pragma unroll 1
  for (;;) {
    if (tid == 0) s_item = atomicAdd(a.next_item, 1u);
    __syncthreads();
    const uint32_t i = s_item;
    if (i >= a.num_items) break;  // uniform
    const BlockItem w = a.items[i];
    const uint32_t  r0 = w.block * kBlockRows;
    const uint32_t  rows = min(kBlockRows, a.n - r0);
    for (uint32_t j = tid; j < rows; j += kBlockedThreads) s_acc[j] = 0ull;
    __syncthreads();

    accumulate<LOADS, PACKED>(a, cin, w.block, w.e0, w.e1, s_acc);
    __syncthreads();

    if (w.pieces == 1) {
      double res = 0.0;
      for (uint32_t j = tid; j < rows; j += kBlockedThreads) res += row_update(a, cout, r0 + j, s_acc[j], pol);
      res = block_sum(res, s_red);
      if (tid == 0) a.res_blk[w.block] = res;
    } else {
      unsigned long long* z = a.zacc + a.zoff[w.block];
      for (uint32_t j = tid; j < rows; j += kBlockedThreads) {
        const unsigned long long v = s_acc[j];
        if (v) atomicAdd(z + j, v);
      }
      __threadfence();
      __syncthreads();
      if (tid == 0) s_last = (atomicAdd(a.ticket + w.block, 1u) == w.pieces - 1u);
      __syncthreads();
      if (s_last) {
        __threadfence();
        double res = 0.0;
        for (uint32_t j = tid; j < rows; j += kBlockedThreads) {
          const unsigned long long v = __ldcg(z + j);
          z[j] = 0ull;  // clear for the next sweep
          res += row_update(a, cout, r0 + j, v, pol);
        }
        res = block_sum(res, s_red);
        if (tid == 0) {
          a.res_blk[w.block] = res;
          a.ticket[w.block] = 0u;
        }
      }
    }
    __syncthreads();  // s_item, s_acc and s_last are reused by the next item
  }
}

// After the sweep: the FP64 L1 change summed over the blocks in block order,
// the convergence test and the loop condition (page_rank.hpp:125-144).
__global__ void __launch_bounds__(1024) pr_blocked_finish_kernel(const BlockedArgs a) {
  __shared__ double s_red[32];
  PrState*          st = a.sw.st;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  double                   e = 0.0;
  for (uint32_t b = threadIdx.x; b < a.num_blocks; b += blockDim.x) e += __ldcg(a.res_blk + b);
  e = block_sum(e, s_red);
  if (threadIdx.x == 0) {
    const unsigned long long done_iters = it + 1ull;
    st->iter = done_iters;
    st->last_error = e;
    if (a.sw.err_hist && it < a.sw.err_cap) a.sw.err_hist[it] = e;  // the first err_cap sweeps
    const bool fault = *(volatile unsigned int*)&st->fault != 0u;
    const bool conv = !fault && e < st->threshold;
    const bool abort = a.sw.abort_word && *a.sw.abort_word;
    const bool done = conv || done_iters >= st->max_iters || abort || fault;
    st->converged = conv ? 1u : 0u;
    st->aborted = (abort && !conv) ? 1u : 0u;
    st->done = done ? 1u : 0u;
    *a.next_item = 0u;
    __threadfence();
    if (a.sw.use_cond && !done && done_iters < st->chunk_end) cudaGraphSetConditional(a.sw.cond, 1u);
  }
}

// ---------------------------------------------------------------------------
// Set-up: the blocked entry order and the work list
// ---------------------------------------------------------------------------
namespace {

constexpr uint32_t kKeyEntries = 4096;  // entries per CTA of the key kernel

// key = block << id_bits | source, value = row within the block, for every entry.
// A CTA takes kKeyEntries consecutive entries; thread 0 finds the rows they
// span, and each thread finds its entry's row by binary search inside that span.
__global__ void __launch_bounds__(256) block_keys_kernel(const uint32_t* __restrict__ row_ptr,
                                                         const uint32_t* __restrict__ col, uint64_t n, uint64_t nnz,
                                                         int id_bits, unsigned long long* __restrict__ keys,
                                                         uint16_t* __restrict__ vals) {
  __shared__ uint64_t s_lo, s_hi;
  const uint64_t k0 = (uint64_t)blockIdx.x * kKeyEntries;
  if (k0 >= nnz) return;
  const uint64_t k1 = min(nnz, k0 + kKeyEntries);
  if (threadIdx.x == 0) {
    // last row whose start is <= x, for x = k0 and x = k1 - 1
    auto row_of = [&](uint64_t x) {
      uint64_t lo = 0, hi = n - 1;
      while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) >> 1;
        if ((uint64_t)row_ptr[mid] <= x) lo = mid; else hi = mid - 1;
      }
      return lo;
    };
    s_lo = row_of(k0);
    s_hi = row_of(k1 - 1);
  }
  __syncthreads();
  const uint64_t rlo = s_lo, rhi = s_hi;
  for (uint64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    uint64_t lo = rlo, hi = rhi;
    while (lo < hi) {
      const uint64_t mid = (lo + hi + 1) >> 1;
      if ((uint64_t)row_ptr[mid] <= k) lo = mid; else hi = mid - 1;
    }
    keys[k] = ((unsigned long long)(lo / kBlockRows) << id_bits) | (unsigned long long)col[k];
    vals[k] = (uint16_t)(lo % kBlockRows);
  }
}

__global__ void low_words_kernel(const unsigned long long* __restrict__ keys, uint64_t nnz, int id_bits,
                                 uint32_t* __restrict__ out) {
  const uint64_t           stride = (uint64_t)gridDim.x * blockDim.x;
  const unsigned long long mask = (1ull << id_bits) - 1ull;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride)
    out[k] = (uint32_t)(keys[k] & mask);
}

__global__ void block_ptr_kernel(const uint32_t* __restrict__ row_ptr, uint64_t n, uint32_t nb, uint32_t* __restrict__ out) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= nb; b += gridDim.x * blockDim.x) {
    const uint64_t r = min((uint64_t)b * kBlockRows, n);
    out[b] = row_ptr[r];
  }
}

// Packed words: one warp per 32-entry group of a block (grid-stride over the
// groups). With wide == nullptr it only counts the wide groups into *count.
__global__ void __launch_bounds__(256) pack_groups_kernel(const unsigned long long* __restrict__ keys,
                                                          const uint16_t* __restrict__ rows, int id_bits,
                                                          const uint32_t* __restrict__ blk_e0,
                                                          const uint32_t* __restrict__ blk_g0, uint32_t nb,
                                                          uint32_t* __restrict__ words, uint32_t* __restrict__ gbase,
                                                          uint32_t* __restrict__ wide, uint32_t* __restrict__ count) {
  const unsigned long long mask = (1ull << id_bits) - 1ull;
  const uint32_t           lane = threadIdx.x & 31u;
  const uint64_t           warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint32_t           groups = blk_g0[nb];
  for (uint64_t g = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < groups; g += warps) {
    uint32_t lo = 0, hi = nb - 1;  // the block holding group g: last b with blk_g0[b] <= g
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (blk_g0[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const uint64_t e_first = (uint64_t)blk_e0[lo] + ((uint64_t)g - blk_g0[lo]) * 32u;
    const uint64_t e_end = blk_e0[lo + 1];
    const uint64_t e = e_first + lane;
    const bool     ok = e < e_end;
    const uint32_t src = ok ? (uint32_t)(keys[e] & mask) : 0u;
    const uint64_t span_left = e_end - 1 - e_first;
    const uint32_t last_lane = span_left < 31u ? (uint32_t)span_left : 31u;
    const uint32_t first = __shfl_sync(kFullMask, src, 0);
    const uint32_t last = __shfl_sync(kFullMask, src, last_lane);
    const bool     is_wide = (last - first >= kPackSpan) || (first & kWideGroup);
    if (!wide) {
      if (lane == 0 && is_wide) atomicAdd(count, 1u);
      continue;
    }
    uint32_t w = 0;
    if (is_wide) {
      if (lane == 0) w = atomicAdd(count, 1u);
      w = __shfl_sync(kFullMask, w, 0);
      wide[(uint64_t)w * 32u + lane] = src;
    }
    if (ok) words[e] = (is_wide ? 0u : ((src - first) << kPackRowBits)) | (uint32_t)rows[e];
    if (lane == 0) gbase[g] = is_wide ? (kWideGroup | w) : first;
  }
}

// outcount[source] += entries, one atomic per run of equal sources in a warp's
// 32 consecutive sorted entries.
__global__ void count_sources_kernel(const unsigned long long* __restrict__ keys, uint64_t nnz, int id_bits,
                                     uint32_t* __restrict__ outcount) {
  const unsigned long long mask = (1ull << id_bits) - 1ull;
  const uint64_t           stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < nnz; base += stride) {
    const uint64_t k = base + threadIdx.x;
    const bool     ok = k < nnz;
    const uint32_t src = ok ? (uint32_t)(keys[k] & mask) : 0xffffffffu;
    const unsigned same = __match_any_sync(kFullMask, src);
    if (ok && (threadIdx.x & 31u) == (unsigned)(__ffs(same) - 1)) atomicAdd(outcount + src, (uint32_t)__popc(same));
  }
}

__global__ void check_degrees_kernel(const uint32_t* __restrict__ deg, const uint32_t* __restrict__ outcount,
                                     uint64_t n, PrState* st) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  bool           bad = false;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) bad |= deg[j] < outcount[j];
  if (__any_sync(kFullMask, bad) && (threadIdx.x & 31u) == 0u) atomicOr(&st->fault, kFaultDegrees);
}

template <class T>
void free_ptr(T*& p, cudaStream_t s) {
  pool_free(p, s);
  p = nullptr;
}

}  // namespace

void BlockPlan::release(cudaStream_t s) {
  free_ptr(src, s);
  free_ptr(dst, s);
  free_ptr(gbase, s);
  free_ptr(wide, s);
  free_ptr(blk_e0, s);
  free_ptr(blk_g0, s);
  free_ptr(outcount, s);
  packed = false;
  wide_groups = 0;
  free_ptr(items, s);
  free_ptr(zoff, s);
  free_ptr(zacc, s);
  free_ptr(ticket, s);
  free_ptr(res_blk, s);
  free_ptr(next_item, s);
  ok = false;
}

#define BK(call)                                  \
  do {                                            \
    cudaError_t _e = (call);                      \
    if (_e != cudaSuccess) {                      \
      pool_free(keys0, s);                        \
      pool_free(keys1, s);                        \
      pool_free(vals1, s);                        \
      pool_free(tmp, s);                          \
      pool_free(bptr, s);                         \
      p->release(s);                              \
      return _e;                                  \
    }                                             \
  } while (0)

cudaError_t build_block_plan(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, uint64_t nnz, uint64_t id_bound,
                             int sms, uint64_t piece_entries, bool packed, BlockPlan* p, cudaStream_t s) {
  p->release(s);
  unsigned long long *keys0 = nullptr, *keys1 = nullptr;
  uint16_t*           vals1 = nullptr;
  void*               tmp = nullptr;
  uint32_t*           bptr = nullptr;
  if (n == 0) return cudaSuccess;
  const uint32_t nb = (uint32_t)((n + kBlockRows - 1) / kBlockRows);
  int            bits = 1;  // block id bits
  while (bits < 32 && (1ull << bits) < nb) ++bits;
  int id_bits = 1;  // column id bits
  while (id_bits < 32 && (1ull << id_bits) < id_bound) ++id_bits;
  p->num_blocks = nb;
  // blocks' entry ranges: rows [b S, (b+1) S) are consecutive in the CSR
  BK(pool_alloc_n(&bptr, (uint64_t)nb + 1, s));
  block_ptr_kernel<<<(nb + 256) / 256, 256, 0, s>>>(row_ptr, n, nb, bptr);
  BK(cudaGetLastError());
  std::vector<uint32_t> h_ptr((size_t)nb + 1);
  BK(cudaMemcpyAsync(h_ptr.data(), bptr, ((size_t)nb + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (nnz) {
    BK(pool_alloc_n(&keys0, nnz, s));
    BK(pool_alloc_n(&keys1, nnz, s));
    BK(pool_alloc_n(&p->dst, nnz + kPad, s));
    BK(pool_alloc_n(&vals1, nnz, s));
    const uint64_t ctas = (nnz + kKeyEntries - 1) / kKeyEntries;
    block_keys_kernel<<<(unsigned)ctas, 256, 0, s>>>(row_ptr, col, n, nnz, id_bits, keys0, p->dst);
    BK(cudaGetLastError());
    cub::DoubleBuffer<unsigned long long> kb(keys0, keys1);
    cub::DoubleBuffer<uint16_t>           vb(p->dst, vals1);
    size_t                                tmp_bytes = 0;
    BK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, (int64_t)nnz, 0, id_bits + bits, s));
    BK(pool_alloc((void**)&tmp, tmp_bytes, s));
    BK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kb, vb, (int64_t)nnz, 0, id_bits + bits, s));
    if (vb.Current() != p->dst) {  // keep the sorted values as dst
      uint16_t* t = p->dst;
      p->dst = vb.Current();
      vals1 = t;
    }
    BK(pool_alloc_n(&p->outcount, id_bound + kPad, s));
    BK(cudaMemsetAsync(p->outcount, 0, (id_bound + kPad) * sizeof(uint32_t), s));
    count_sources_kernel<<<sms * 8, 256, 0, s>>>(kb.Current(), nnz, id_bits, p->outcount);
    BK(cudaGetLastError());
    BK(pool_alloc_n(&p->src, nnz + kPad, s));
    if (packed && id_bound <= (uint64_t)kWideGroup) {
      // block and group offsets, then one word per entry and one base per group
      BK(cudaStreamSynchronize(s));  // h_ptr
      std::vector<uint32_t> h_g0((size_t)nb + 1, 0u);
      for (uint32_t b = 0; b < nb; ++b) h_g0[b + 1] = h_g0[b] + (h_ptr[b + 1] - h_ptr[b] + 31u) / 32u;
      BK(pool_alloc_n(&p->blk_e0, (uint64_t)nb + 1, s));
      BK(pool_alloc_n(&p->blk_g0, (uint64_t)nb + 1, s));
      BK(cudaMemcpyAsync(p->blk_e0, h_ptr.data(), ((size_t)nb + 1) * 4, cudaMemcpyHostToDevice, s));
      BK(cudaMemcpyAsync(p->blk_g0, h_g0.data(), ((size_t)nb + 1) * 4, cudaMemcpyHostToDevice, s));
      const uint32_t groups = h_g0[nb];
      BK(pool_alloc_n(&p->gbase, (uint64_t)groups + 1, s));
      uint32_t* d_count = nullptr;
      BK(pool_alloc_n(&d_count, 1, s));
      uint32_t h_count = 0;
      const unsigned pg = (unsigned)std::min<uint64_t>(((uint64_t)groups + 7) / 8, (uint64_t)sms * 64);
      BK(cudaMemsetAsync(d_count, 0, 4, s));
      pack_groups_kernel<<<pg ? pg : 1, 256, 0, s>>>(kb.Current(), vb.Current(), id_bits, p->blk_e0, p->blk_g0, nb,
                                                    p->src, p->gbase, nullptr, d_count);
      BK(cudaGetLastError());
      BK(cudaMemcpyAsync(&h_count, d_count, 4, cudaMemcpyDeviceToHost, s));
      BK(cudaStreamSynchronize(s));
      BK(pool_alloc_n(&p->wide, (uint64_t)h_count * 32u + 1u, s));
      BK(cudaMemsetAsync(d_count, 0, 4, s));
      pack_groups_kernel<<<pg ? pg : 1, 256, 0, s>>>(kb.Current(), vb.Current(), id_bits, p->blk_e0, p->blk_g0, nb,
                                                    p->src, p->gbase, p->wide, d_count);
      BK(cudaGetLastError());
      BK(cudaStreamSynchronize(s));
      pool_free(d_count, s);
      free_ptr(p->dst, s);  // the rows live in the words
      p->packed = true;
      p->wide_groups = h_count;
    } else {
      low_words_kernel<<<sms * 8, 256, 0, s>>>(kb.Current(), nnz, id_bits, p->src);
      BK(cudaGetLastError());
    }
  }
  BK(cudaStreamSynchronize(s));
  pool_free(keys0, s);
  pool_free(keys1, s);
  pool_free(vals1, s);
  pool_free(tmp, s);
  pool_free(bptr, s);
  keys0 = keys1 = nullptr;
  vals1 = nullptr;
  tmp = nullptr;
  bptr = nullptr;

  p->block_ptr = std::move(h_ptr);
  p->n = n;
  p->nnz = nnz;
  BK(pool_alloc_n(&p->ticket, nb, s));
  BK(cudaMemsetAsync(p->ticket, 0, nb * sizeof(uint32_t), s));
  BK(pool_alloc_n(&p->res_blk, nb, s));
  BK(cudaMemsetAsync(p->res_blk, 0, nb * sizeof(double), s));
  BK(pool_alloc_n(&p->next_item, 1, s));
  BK(cudaMemsetAsync(p->next_item, 0, sizeof(uint32_t), s));
  p->sweep_grid = sms;
  BK(set_block_items(p, sms, piece_entries, s));
  p->ok = true;
  return cudaSuccess;
}
#undef BK

// The work list: blocks of more than piece_entries entries are cut into equal
// pieces; the others are one item each. Items are sorted largest first.
cudaError_t set_block_items(BlockPlan* p, int sms, uint64_t piece_entries, cudaStream_t s) {
  const uint32_t nb = p->num_blocks;
  const uint64_t n = p->n, nnz = p->nnz;
  if (!piece_entries) piece_entries = std::max<uint64_t>(1ull << 16, nnz / ((uint64_t)(sms > 0 ? sms : 1) * 2ull));
  std::vector<BlockItem> items;
  std::vector<uint32_t>  zoff(nb, ~0u);
  uint64_t               zrows = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    const uint64_t cnt = (uint64_t)p->block_ptr[b + 1] - p->block_ptr[b];
    const uint32_t pieces = (uint32_t)std::max<uint64_t>(1, (cnt + piece_entries - 1) / piece_entries);
    if (pieces > 1) {
      zoff[b] = (uint32_t)zrows;
      zrows += std::min<uint64_t>(kBlockRows, n - (uint64_t)b * kBlockRows);
    }
    // pieces start at 32-entry group boundaries of the block (the packed format's groups)
    const uint64_t e0 = p->block_ptr[b], e1 = p->block_ptr[b + 1], groups = (cnt + 31) / 32;
    for (uint32_t q = 0; q < pieces; ++q) {
      const uint64_t a0 = e0 + 32ull * (groups * q / pieces), a1 = std::min<uint64_t>(e1, e0 + 32ull * (groups * (q + 1) / pieces));
      items.push_back(BlockItem{b, (uint32_t)a0, (uint32_t)a1, pieces});
    }
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const BlockItem& x, const BlockItem& y) { return x.e1 - x.e0 > y.e1 - y.e0; });
  free_ptr(p->items, s);
  free_ptr(p->zoff, s);
  free_ptr(p->zacc, s);
  cudaError_t e;
  if ((e = pool_alloc_n(&p->items, items.size(), s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(p->items, items.data(), items.size() * sizeof(BlockItem), cudaMemcpyHostToDevice, s)) !=
      cudaSuccess)
    return e;
  if ((e = pool_alloc_n(&p->zoff, nb, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(p->zoff, zoff.data(), nb * sizeof(uint32_t), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return e;
  if ((e = pool_alloc_n(&p->zacc, zrows ? zrows : 1, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(p->zacc, 0, (zrows ? zrows : 1) * sizeof(unsigned long long), s)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;  // the host vectors go out of scope
  p->num_items = (uint32_t)items.size();
  p->piece_entries = piece_entries;
  p->bytes = (nnz + kPad) * (p->packed ? 4 : 6) + (p->packed ? (nnz / 32 + nb) * 4 + p->wide_groups * 128 : 0) +
             items.size() * sizeof(BlockItem) + (uint64_t)nb * 16 + zrows * 8;
  return cudaSuccess;
}

cudaError_t launch_check_degrees(const BlockPlan& p, const uint32_t* deg, PrState* st, int sms, cudaStream_t s) {
  if (!p.outcount || !p.n) return cudaSuccess;
  check_degrees_kernel<<<sms * 4, 256, 0, s>>>(deg, p.outcount, p.n, st);
  return cudaGetLastError();
}

BlockedArgs make_blocked_args(const BlockPlan& p, const SweepArgs& sw, uint64_t n) {
  BlockedArgs a = {};
  a.sw = sw;
  a.src = p.src;
  a.dst = p.dst;
  a.gbase = p.packed ? p.gbase : nullptr;
  a.wide = p.wide;
  a.blk_e0 = p.blk_e0;
  a.blk_g0 = p.blk_g0;
  a.items = p.items;
  a.num_items = p.num_items;
  a.num_blocks = p.num_blocks;
  a.n = (uint32_t)n;
  a.zoff = p.zoff;
  a.zacc = p.zacc;
  a.ticket = p.ticket;
  a.res_blk = p.res_blk;
  a.next_item = p.next_item;
  return a;
}

static void* blocked_fn(int loads, bool packed) {
  if (packed) {
    if (loads <= 4) return (void*)pr_blocked_sweep_kernel<4, true>;
    if (loads >= 16) return (void*)pr_blocked_sweep_kernel<16, true>;
    return (void*)pr_blocked_sweep_kernel<8, true>;
  }
  if (loads <= 4) return (void*)pr_blocked_sweep_kernel<4, false>;
  if (loads >= 16) return (void*)pr_blocked_sweep_kernel<16, false>;
  return (void*)pr_blocked_sweep_kernel<8, false>;
}

cudaError_t configure_blocked_kernels() {
  for (bool packed : {false, true})
    for (int loads : {4, 8, 16}) {
      cudaError_t e = cudaFuncSetAttribute(blocked_fn(loads, packed), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(kBlockRows * sizeof(unsigned long long)));
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

cudaError_t launch_blocked_sweep(const BlockedArgs& a, int sweep_grid, int loads, cudaStream_t s) {
  void*       args[] = {(void*)&a};
  cudaError_t e = cudaLaunchKernel(blocked_fn(loads, a.gbase != nullptr), dim3((unsigned)sweep_grid),
                                   dim3(kBlockedThreads), args,
                                   kBlockRows * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  pr_blocked_finish_kernel<<<1, 1024, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t add_blocked_nodes(cudaGraph_t body, const BlockedArgs& a, int sweep_grid, int loads) {
  void*                args[] = {(void*)&a};
  cudaKernelNodeParams kp = {};
  kp.func = blocked_fn(loads, a.gbase != nullptr);
  kp.gridDim = dim3((unsigned)sweep_grid);
  kp.blockDim = dim3(kBlockedThreads);
  kp.sharedMemBytes = (unsigned)(kBlockRows * sizeof(unsigned long long));
  kp.kernelParams = args;
  cudaGraphNode_t sn, fn;
  cudaError_t     e = cudaGraphAddKernelNode(&sn, body, nullptr, 0, &kp);
  if (e != cudaSuccess) return e;
  cudaKernelNodeParams fp = {};
  fp.func = (void*)pr_blocked_finish_kernel;
  fp.gridDim = dim3(1);
  fp.blockDim = dim3(1024);
  fp.kernelParams = args;
  return cudaGraphAddKernelNode(&fn, body, &sn, 1, &fp);
}

}  // namespace nwgpu
