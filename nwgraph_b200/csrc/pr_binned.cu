// Degree-binned PageRank sweep for relabelled graphs (rows in descending
// length order), sm_100a.
//
// After relabelling, rows of similar length are contiguous, so the sweep is
// split into bins without any per-row indirection:
//   long   len > long_row     : chunks of `chunk` entries, one warp per chunk;
//                               pr_binned_finish_kernel sums each row's chunk
//                               partials in chunk order
//   bin 0  128 < len <= long_row: half a warp per row (two rows per warp),
//                               16 lanes walk the row; or, as the plan
//                               sets (bin0_rows), a warp per row
// (long_row and chunk are the plan's, 2048 and 1024 unless tuned or set)
//   G = 32, 16, 8, 4, 2, 1      : rows of (G*2, G*4] entries (G = 1: 1..4),
//                               G lanes per row, two rows per lane group,
//                               <= 4 entries of each per lane
//   empty  len = 0             : epilogue only
// Every lane's entries are summed in a fixed order and combined by a fixed
// xor-shuffle tree, so ranks are bit-reproducible. Column ids stream through
// (coalesced, evict-first; 128-bit loads in the long-row chunks and bin 0);
// contributions are gathered with 8 loads in flight per lane. Each warp walks
// its units software-pipelined: while the gathers of one step are in flight,
// the column ids of the next step and the row bounds of the unit after it are
// already loading.
//
// pr_binned_finish_kernel, launched right after, finishes the long rows; its
// last CTA to finish (a ticket) reduces all FP64 residual partials in a fixed
// order and runs the convergence test on the device. Completing a long row
// inside the sweep (the warp of its last chunk) needs a memory fence per
// chunk, and a fence drains the warp's loads in flight: measured slower than
// the second, short kernel.
//
// Where the gathered values come from (ids are in descending-degree order, so
// small ids are the hubs):
//   HOT = false: 256-thread CTAs, four per SM; ids < l1_ids through L1 with
//                an evict-last policy, the rest with L1::no_allocate;
//   HOT = true:  one 1024-thread CTA per SM copies contrib[0, smem_ids) into
//                shared memory at the start of the sweep and gathers those ids
//                from there; [smem_ids, l1_ids) through L1, the rest
//                L1::no_allocate.
// A warp load whose lanes mix L1 hits and misses costs the L1 as much as one
// that misses in every lane, while shared-memory loads use a separate, much
// wider path; staging the hubs in shared memory leaves the L1->L2 request
// path to the misses alone. Both variants sum the same values in the same
// order, so their ranks are bitwise equal. The per-row update is page_rank_v10's
// (include/nwgraph/experimental/algorithms/page_rank.hpp:413-418) fused with
// the next sweep's contribution (:401-405).
#include "binned.h"
#include "common.cuh"
#include "engine.h"

namespace nwgpu {

__device__ __forceinline__ float binned_base(const BinnedArgs& a, uint32_t r) {
  if (a.sw.teleport == kTeleportSeed) return (r == a.sw.seed) ? a.sw.base : 0.f;
  return a.sw.base;
}

// Gather source of one contribution: shared memory (hot variant), L1, or L2.
struct Src {
  const float* __restrict__ cin;
  const float* s_hot;   // staged contrib[0, smem_ids); null in the plain variant
  uint32_t     smem_ids;
  uint32_t     l1_ids;
  uint64_t     pol;
};

template <bool HOT>
__device__ __forceinline__ float gather_one(const Src& s, uint32_t id) {
  if (HOT && id < s.smem_ids) return s.s_hot[id];
  return (id < s.l1_ids) ? ld_gather(s.cin + id, s.pol) : ld_gather_cold(s.cin + id, s.pol);
}

// What a row's epilogue reads besides its sum: the old value and, by mode,
// the out-degree (plain) or the per-row factor and base term (weighted,
// adjoint). Loaded early, while the row's gathers are in flight.
struct RowIn {
  float    old;
  uint32_t dg;    // kModePlain: out-degree
  float    aux;   // kModeWeighted: out-weight sum; kModeAdjoint: d / out-weight sum
  float    base;  // kModeWeighted: (1-d) t; kModeAdjoint: c
};

// kModeRagged: whether row r's graph has stopped (its rows are neither
// gathered nor updated).
__device__ __forceinline__ bool ragged_frozen(const BinnedArgs& a, uint32_t r) {
  return __ldg(a.sw.graph_done + __ldg(a.sw.row_graph + r)) != 0u;
}

template <int MODE>
__device__ __forceinline__ RowIn load_row_in(const BinnedArgs& a, uint32_t r) {
  RowIn x;
  x.old = ld_stream(a.sw.rank + r);
  if constexpr (MODE == kModePlain || MODE == kModeResidual || MODE == kModeRagged) {
    x.dg = ld_stream(a.sw.deg + r);
    x.aux = 1.f;
    x.base = 0.f;
  } else {
    x.dg = 1u;
    x.aux = ld_stream(a.sw.vaux + r);
    x.base = ld_stream(a.sw.vbase + r);
  }
  return x;
}
__device__ __forceinline__ RowIn no_row_in() { return RowIn{0.f, 1u, 1.f, 0.f}; }

// Epilogue of one row: new value, the next sweep's contribution, |dr| in FP64.
template <int MODE>
__device__ __forceinline__ double binned_update(const BinnedArgs& a, float* __restrict__ cout, uint32_t r, float z,
                                                const RowIn& in, uint64_t pol) {
  if constexpr (MODE == kModeRagged) {
    // the row's graph: stopped (its rank and contribution stay), else its base term (1 - d) / n_g; read here
    // rather than with the row's other inputs, which keeps them out of the registers held across a step
    const uint32_t g = __ldg(a.sw.row_graph + r);
    if (__ldg(a.sw.graph_done + g) != 0u) return 0.0;
    const float  nr = fmaf(a.sw.damping, z, __ldg(a.sw.graph_base + g));
    const double e = (double)fabsf(nr - in.old);
    st_stream(a.sw.rank + r, nr);
    st_keep(cout + r, nr / (float)in.dg, pol);
    a.sw.row_res[r] = e;
    return e;
  }
  float nr, c;
  if constexpr (MODE == kModePlain) {
    nr = fmaf(a.sw.damping, z, binned_base(a, r));
    c = nr / (float)in.dg;
  } else if constexpr (MODE == kModeWeighted) {
    nr = fmaf(a.sw.damping, z, in.base);
    c = nr / in.aux;
  } else if constexpr (MODE == kModeResidual) {
    // z is this row's new residual (page_rank_v13's second phase: the sum of
    // the positive deltas, all deltas being >= 0); then its first phase for
    // the next iteration: push a residual above the threshold into the rank
    // and, with out-degree > 0, spread residual * d / deg (FP32, :576-589).
    const float res = z > 0.f ? z : 0.f;
    const bool  push = res > a.sw.push_threshold;
    const bool  moved = push && in.dg > 0u;
    nr = push ? in.old + res : in.old;
    c = moved ? res * a.sw.damping / (float)in.dg : 0.f;
    st_stream(a.sw.rank + r, nr);
    st_keep(cout + r, c, pol);
    return moved ? 1.0 : 0.0;
  } else {
    nr = fmaf(in.aux, z, in.base);
    c = nr;
  }
  st_stream(a.sw.rank + r, nr);
  st_keep(cout + r, c, pol);
  return (double)fabsf(nr - in.old);
}
template <int MODE>
__device__ __forceinline__ double binned_epilogue(const BinnedArgs& a, float* __restrict__ cout, uint32_t r, float z,
                                                  uint64_t pol) {
  return binned_update<MODE>(a, cout, r, z, load_row_in<MODE>(a, r), pol);
}

// One term of a row sum: the gathered contribution, times the entry's weight
// in the weighted and adjoint modes.
template <bool HOT, int MODE>
__device__ __forceinline__ float term(const BinnedArgs& a, const Src& src, uint32_t id, uint32_t k) {
  const float c = gather_one<HOT>(src, id);
  if constexpr (MODE == kModePlain || MODE == kModeResidual || MODE == kModeRagged) return c;
  else return ld_stream(a.sw.w + k) * c;
}

// Rows without entries: four rows per lane.
template <int MODE>
__device__ __forceinline__ double empty_rows(const BinnedArgs& a, float* __restrict__ cout, uint32_t row0,
                                             uint32_t row_end, int lane, uint64_t pol) {
  double res = 0.0;
  RowIn  in[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t r = row0 + q * 32 + lane;
    in[q] = (r < row_end) ? load_row_in<MODE>(a, r) : no_row_in();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t r = row0 + q * 32 + lane;
    if (r < row_end) res += binned_update<MODE>(a, cout, r, 0.f, in[q], pol);
  }
  return res;
}

// ---------------------------------------------------------------------------
// Bin walkers. Units are numbered in one flat space (long-row chunks, then
// bins 0..7) and unit u goes to warp u mod nwarps; a warp takes the units of
// one bin at a time. While the gathers of one step are in flight, the column
// ids of the next step and the row bounds of the unit after it are already
// loading: a warp keeps loads of two or three stages outstanding instead of
// waiting through row_ptr -> col -> contrib in turn.
// ---------------------------------------------------------------------------
// First unit (bin-local index) of warp gwarp in a bin that starts at flat unit `begin`.
__device__ __forceinline__ uint32_t first_unit(uint32_t gwarp, uint32_t nwarps, uint32_t begin) {
  const uint32_t r = begin % nwarps;
  return gwarp >= r ? gwarp - r : gwarp + nwarps - r;
}

// Column ids in 128-bit loads. A step of a unit covers a window of L
// consecutive entries starting at `start` (the unit's first entry plus a
// multiple of L), walked by L/8 lanes (a warp for L = 256, a half-warp for
// L = 128): each lane takes 4 consecutive entries of each half of it, so slot
// q of lane i holds the entry
//   start + (L/2) * (q / 4) + 4 * i + q % 4.
// The mapping is relative to the row (or chunk) start, so a row is summed in
// the same order wherever it lies in the CSR: in a graph alone, in a union
// of graphs, in any shard. The ids arrive in 16-byte-aligned uint4 words:
// with p = start % 4, lane i's 4 entries of a half lie in the aligned word at
// start - p + (L/2) * half + 4 i and, for p > 0, partly in the next word,
// which the lane loads too; the words are then shifted by p. A word is loaded
// only when one of the lane's entries in it lies before `end`, so the loads
// reach at most 3 entries past the array's last one (inside the padding every
// column array of a handle carries) and never a word before the array's start.
template <uint32_t L>
__device__ __forceinline__ uint32_t window_entry(uint32_t start, uint32_t lanei, int q) {
  return start + (L / 2u) * (uint32_t)(q >> 2) + 4u * lanei + (uint32_t)(q & 3);
}
template <uint32_t L>
__device__ __forceinline__ void load_window(const uint32_t* __restrict__ col, uint32_t start, uint32_t end,
                                            uint32_t lanei, uint32_t (&dst)[8]) {
  const uint32_t p = start & 3u;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const uint32_t w0 = (start & ~3u) + (L / 2u) * (uint32_t)j + 4u * lanei;  // aligned word of the first entry
    uint4          x = make_uint4(0u, 0u, 0u, 0u), y = x;
    if (w0 + p < end) x = ld_stream4(reinterpret_cast<const uint4*>(col + w0));
    if (p != 0u && w0 + 4u < end) y = ld_stream4(reinterpret_cast<const uint4*>(col + w0 + 4u));
    dst[4 * j] = p == 0u ? x.x : p == 1u ? x.y : p == 2u ? x.z : x.w;
    dst[4 * j + 1] = p == 0u ? x.y : p == 1u ? x.z : p == 2u ? x.w : y.x;
    dst[4 * j + 2] = p == 0u ? x.z : p == 1u ? x.w : p == 2u ? y.x : y.y;
    dst[4 * j + 3] = p == 0u ? x.w : p == 1u ? y.x : p == 2u ? y.y : y.z;
  }
}

// Units that are entry ranges, one warp each, walked in 256-entry windows
// (load_window). CHUNK: unit c = chunk c of a long row, partial sum to
// chunk_part[c] (the long rows). Otherwise: unit w = row rb + w, epilogue
// (bin 0 when the plan gives it a warp per row).
template <bool HOT, bool CHUNK, int MODE>
__device__ __forceinline__ double range_bin(const BinnedArgs& a, const Src& src, float* __restrict__ cout, uint32_t rb,
                                            uint32_t nunits, uint32_t w, uint32_t nwarps, int lane) {
  constexpr int      U = 8;
  constexpr uint32_t STEP = U * 32;
  if (w >= nunits) return 0.0;
  auto bounds = [&](uint32_t unit, uint32_t& k0, uint32_t& k1, uint32_t& row) {
    if (CHUNK) {
      row = a.chunk_row[unit];
      const uint32_t rs = a.sw.row_ptr[row], re = a.sw.row_ptr[row + 1];
      k0 = rs + (unit - a.row_first_chunk[row]) * a.chunk;
      k1 = k0 + min(re - k0, a.chunk);  // no 32-bit wrap near the entry limit
      if (MODE == kModeRagged && ragged_frozen(a, row)) k1 = k0;  // a stopped graph's row: nothing to gather
    } else {
      row = rb + unit;
      k0 = ld_stream(a.sw.row_ptr + rb + unit);
      k1 = ld_stream(a.sw.row_ptr + rb + unit + 1);
      if (MODE == kModeRagged && ragged_frozen(a, row)) k1 = k0;  // a stopped graph's row: nothing to gather
    }
  };
  uint32_t k0, k1, row, nk0 = 0, nk1 = 0, nrow = 0;
  bounds(w, k0, k1, row);
  if (w + nwarps < nunits) bounds(w + nwarps, nk0, nk1, nrow);
  uint32_t id[U];
  uint32_t base = k0;  // the window's first entry
  load_window<STEP>(a.sw.col, base, k1, (uint32_t)lane, id);
  RowIn in = no_row_in();
  if (!CHUNK && lane == 0) in = load_row_in<MODE>(a, row);
  float  acc = 0.f;
  double res = 0.0;
  // A finished unit's reduction and epilogue wait one step, until the next
  // step's gathers are in flight, so the shuffle tree and the update run
  // under those loads instead of between them (warp-uniform).
  bool     pending = false;
  float    acc_done = 0.f;
  uint32_t unit_done = 0u;
  RowIn    in_done = no_row_in();
  auto     finish = [&]() {
    const float z = warp_sum_lane0(acc_done);
    if (CHUNK) {
      if (lane == 0) a.chunk_part[unit_done] = z;
    } else if (lane == 0) {
      res += binned_update<MODE>(a, cout, rb + unit_done, z, in_done, src.pol);
    }
  };
#pragma unroll 1
  for (;;) {
    float v[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
      const uint32_t k = window_entry<STEP>(base, (uint32_t)lane, q);
      v[q] = (k < k1) ? term<HOT, MODE>(a, src, id[q], k) : 0.f;
    }
    if (pending) {
      finish();
      pending = false;
    }
    // the next step: the rest of this unit, or the first step of the next one
    const bool     more = base + STEP < k1;  // warp-uniform
    const bool     has_next = w + nwarps < nunits;
    const uint32_t nbase = more ? base + STEP : nk0;
    const uint32_t nend = more ? k1 : (has_next ? nk1 : 0u);
    load_window<STEP>(a.sw.col, nbase, nend, (uint32_t)lane, id);
#pragma unroll
    for (int q = 0; q < U; ++q) acc += v[q];
    if (!more) {
      pending = true;
      acc_done = acc;
      unit_done = w;
      in_done = in;
      acc = 0.f;
      w += nwarps;
      if (w >= nunits) break;
      k1 = nk1;
      row = nrow;
      if (w + nwarps < nunits) bounds(w + nwarps, nk0, nk1, nrow);
      if (!CHUNK && lane == 0) in = load_row_in<MODE>(a, row);
    }
    base = nbase;
  }
  if (pending) finish();
  return res;
}

// Bin 0 (rows of 129 entries to the long-row cut-off): a unit is two
// consecutive rows, one per half-warp, 16 lanes walking each row in 128-entry
// windows (load_window). Half-warps waste fewer lanes on a row's last, partial
// step than a whole warp's 256-entry steps (adjacent rows have about the same
// length: the rows are in length order). The walk is range_bin's: the next
// step's column ids and the next unit's row bounds load while the gathers are
// in flight, and a unit's reduction (a 16-lane xor tree per half) and
// epilogue wait until the next unit's gathers are issued.
template <bool HOT, int MODE>
__device__ __forceinline__ double pair_bin(const BinnedArgs& a, const Src& src, float* __restrict__ cout, uint32_t rb,
                                           uint32_t re_bin, uint32_t nunits, uint32_t w, uint32_t nwarps, int lane) {
  constexpr int      U = 8;
  constexpr uint32_t STEP = U * 16;
  if (w >= nunits) return 0.0;
  const uint32_t h = (uint32_t)lane >> 4, sub = (uint32_t)lane & 15u;
  auto bounds = [&](uint32_t unit, uint32_t& k0, uint32_t& k1, uint32_t& row) {
    row = rb + 2u * unit + h;
    if (row < re_bin) {
      k0 = ld_stream(a.sw.row_ptr + row);
      k1 = ld_stream(a.sw.row_ptr + row + 1);
      if (MODE == kModeRagged && ragged_frozen(a, row)) k1 = k0;  // a stopped graph's row: nothing to gather
    } else {  // the bin's odd last row: this half has nothing
      k0 = k1 = 0u;
    }
  };
  uint32_t k0, k1, row, nk0 = 0, nk1 = 0, nrow = 0;
  bounds(w, k0, k1, row);
  if (w + nwarps < nunits) bounds(w + nwarps, nk0, nk1, nrow);
  uint32_t id[U];
  uint32_t base = k0;  // this half's window's first entry
  load_window<STEP>(a.sw.col, base, k1, sub, id);
  RowIn in = no_row_in();
  if (sub == 0 && row < re_bin) in = load_row_in<MODE>(a, row);
  float    acc = 0.f;
  double   res = 0.0;
  bool     pending = false;
  float    acc_done = 0.f;
  uint32_t row_done = 0u;
  RowIn    in_done = no_row_in();
  auto     finish = [&]() {
    float z = acc_done;
#pragma unroll
    for (int off = 8; off > 0; off >>= 1) z += __shfl_xor_sync(kFullMask, z, off);
    if (sub == 0 && row_done < re_bin) res += binned_update<MODE>(a, cout, row_done, z, in_done, src.pol);
  };
#pragma unroll 1
  for (;;) {
    float v[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
      const uint32_t k = window_entry<STEP>(base, sub, q);
      v[q] = (k < k1) ? term<HOT, MODE>(a, src, id[q], k) : 0.f;
    }
    if (pending) {
      finish();
      pending = false;
    }
    // the next step: the rest of this unit (either half still has entries), or the next unit's first
    const bool     mine = base + STEP < k1;
    const bool     more = __any_sync(kFullMask, mine);  // warp-uniform
    const bool     has_next = w + nwarps < nunits;
    const uint32_t nbase = more ? base + STEP : nk0;
    const uint32_t nend = more ? k1 : (has_next ? nk1 : 0u);
    load_window<STEP>(a.sw.col, nbase, nend, sub, id);
#pragma unroll
    for (int q = 0; q < U; ++q) acc += v[q];
    if (!more) {
      pending = true;
      acc_done = acc;
      row_done = row;
      in_done = in;
      acc = 0.f;
      w += nwarps;
      if (w >= nunits) break;
      k1 = nk1;
      row = nrow;
      if (w + nwarps < nunits) bounds(w + nwarps, nk0, nk1, nrow);
      if (sub == 0 && row < re_bin) in = load_row_in<MODE>(a, row);
    }
    base = nbase;
  }
  if (pending) finish();
  return res;
}

// Row bounds of the two rows a lane owns in unit w of a G-bin (len 0: no row).
template <int G, int MODE>
__device__ __forceinline__ void group_bounds(const BinnedArgs& a, uint32_t rb, uint32_t re_bin, uint32_t w,
                                             uint32_t nunits, int lane, uint32_t (&rs)[2], uint32_t (&len)[2]) {
  constexpr uint32_t PER = 32 / G;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    rs[h] = 0u;
    len[h] = 0u;
    if (w < nunits) {
      const uint32_t row = rb + w * (2u * PER) + (uint32_t)h * PER + (uint32_t)lane / G;
      if (row < re_bin) {
        const uint32_t s0 = ld_stream(a.sw.row_ptr + row);
        rs[h] = s0;
        len[h] = ld_stream(a.sw.row_ptr + row + 1) - s0;
        if (MODE == kModeRagged && ragged_frozen(a, row)) len[h] = 0u;  // a stopped graph's row
      }
    }
  }
}

template <int G>
__device__ __forceinline__ void group_ids(const BinnedArgs& a, const uint32_t (&rs)[2], const uint32_t (&len)[2], int sub,
                                          uint32_t (&id)[2][4]) {
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t o = (uint32_t)sub + (uint32_t)q * G;
      id[h][q] = (o < len[h]) ? ld_stream(a.sw.col + rs[h] + o) : 0u;
    }
}

// G-bins: a unit is 2 * 32/G consecutive rows, G lanes per row, each lane two
// rows and at most 4 entries of each.
template <bool HOT, int G, int MODE>
__device__ __forceinline__ double group_bin(const BinnedArgs& a, const Src& src, float* __restrict__ cout, uint32_t rb,
                                            uint32_t re_bin, uint32_t nunits, uint32_t w, uint32_t nwarps, int lane) {
  constexpr uint32_t PER = 32 / G;
  if (w >= nunits) return 0.0;
  const int sub = lane & (G - 1);
  uint32_t  rs[2], len[2], nrs[2], nlen[2], id[2][4];
  group_bounds<G, MODE>(a, rb, re_bin, w, nunits, lane, rs, len);
  group_ids<G>(a, rs, len, sub, id);
  group_bounds<G, MODE>(a, rb, re_bin, w + nwarps, nunits, lane, nrs, nlen);
  double res = 0.0;
  // As in range_bin, a unit's shuffle tree and epilogue wait until the next
  // unit's gathers are in flight; not in the weighted mode, whose wider
  // per-row inputs would not fit the register budget.
  constexpr bool kDefer = MODE != kModeWeighted;
  bool     pending = false;
  uint32_t unit_done = 0u;
  float    acc_done[2] = {0.f, 0.f};
  RowIn    in_done[2] = {no_row_in(), no_row_in()};
  auto     finish = [&]() {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float acc = acc_done[h];
#pragma unroll
      for (int off = G / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(kFullMask, acc, off);
      const uint32_t r = rb + unit_done * (2u * PER) + (uint32_t)h * PER + (uint32_t)lane / G;
      if (r < re_bin && sub == 0) res += binned_update<MODE>(a, cout, r, acc, in_done[h], src.pol);
    }
  };
#pragma unroll 1
  for (; w < nunits; w += nwarps) {
    RowIn in[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t r = rb + w * (2u * PER) + (uint32_t)h * PER + (uint32_t)lane / G;
      in[h] = (r < re_bin && sub == 0) ? load_row_in<MODE>(a, r) : no_row_in();
    }
    float v[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int q = 0; q < 4; ++q)
        v[h][q] = ((uint32_t)sub + (uint32_t)q * G < len[h])
                      ? term<HOT, MODE>(a, src, id[h][q], rs[h] + (uint32_t)sub + (uint32_t)q * G)
                      : 0.f;
    if (kDefer && pending) finish();
    // the next unit's column ids, the bounds of the unit after it
    group_ids<G>(a, nrs, nlen, sub, id);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      rs[h] = nrs[h];
      len[h] = nlen[h];
    }
    group_bounds<G, MODE>(a, rb, re_bin, w + 2u * nwarps, nunits, lane, nrs, nlen);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float acc = 0.f;
#pragma unroll
      for (int q = 0; q < 4; ++q) acc += v[h][q];
      acc_done[h] = acc;
      in_done[h] = in[h];
    }
    unit_done = w;
    pending = true;
    if (!kDefer) {
      finish();
      pending = false;
    }
  }
  if (pending) finish();
  return res;
}

template <int NT, bool HOT, int MODE>
__global__ void __launch_bounds__(NT, 1024 / NT) pr_binned_sweep_kernel(const BinnedArgs a) {
  constexpr int     NW = NT / 32;
  __shared__ double s_red[NW];
  extern __shared__ float4 s_hot4[];  // HOT: contrib[0, smem_ids)
  const int         tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  PrState*          st = a.sw.st;
  if (a.sw.use_cond && blockIdx.x == 0 && tid == 0) cudaGraphSetConditional(a.sw.cond, 0u);
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  const float* __restrict__ cin = (it & 1ull) ? a.sw.contrib1 : a.sw.contrib0;
  float* __restrict__ cout = (it & 1ull) ? a.sw.contrib0 : a.sw.contrib1;
  Src src{cin, nullptr, 0u, a.l1_ids, policy_evict_last()};
  if constexpr (HOT) {
    // smem_ids is a multiple of 4 and contrib is 16-byte aligned
    const float4* g4 = reinterpret_cast<const float4*>(cin);
    for (uint32_t i = tid; i < a.smem_ids / 4u; i += NT) s_hot4[i] = __ldcg(g4 + i);
    __syncthreads();
    src.s_hot = reinterpret_cast<const float*>(s_hot4);
    src.smem_ids = a.smem_ids;
  }
  double         res = 0.0;
  const uint32_t nwarps = gridDim.x * NW, gwarp = blockIdx.x * NW + warp;
  res += range_bin<HOT, true, MODE>(a, src, cout, 0u, a.num_chunks, gwarp, nwarps, lane);
  uint32_t begin = a.num_chunks;  // flat index of the bin's first unit
#pragma unroll 1
  for (int b = 0; b < kNumBins; ++b) {
    const uint32_t nu = a.bin_warp_end[b] - (b ? a.bin_warp_end[b - 1] : 0u);
    const uint32_t w0 = first_unit(gwarp, nwarps, begin);
    const uint32_t rb = a.bin_row_begin[b], re = a.bin_row_end[b];
    switch (b) {
      case 0:
        res += a.bin0_rows == 1u ? range_bin<HOT, false, MODE>(a, src, cout, rb, nu, w0, nwarps, lane)
                                 : pair_bin<HOT, MODE>(a, src, cout, rb, re, nu, w0, nwarps, lane);
        break;
      case 1: res += group_bin<HOT, 32, MODE>(a, src, cout, rb, re, nu, w0, nwarps, lane); break;
      case 2: res += group_bin<HOT, 16, MODE>(a, src, cout, rb, re, nu, w0, nwarps, lane); break;
      case 3: res += group_bin<HOT, 8, MODE>(a, src, cout, rb, re, nu, w0, nwarps, lane); break;
      case 4: res += group_bin<HOT, 4, MODE>(a, src, cout, rb, re, nu, w0, nwarps, lane); break;
      case 5: res += group_bin<HOT, 2, MODE>(a, src, cout, rb, re, nu, w0, nwarps, lane); break;
      case 6: res += group_bin<HOT, 1, MODE>(a, src, cout, rb, re, nu, w0, nwarps, lane); break;
      default:
        for (uint32_t w = w0; w < nu; w += nwarps) res += empty_rows<MODE>(a, cout, rb + w * 128u, re, lane, src.pol);
        break;
    }
    begin += nu;
  }

  res = warp_sum_lane0(res);
  if (lane == 0) s_red[warp] = res;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s += s_red[w];
    a.sw.res_part[blockIdx.x] = s;
  }
}

// Long rows, after the sweep: rows [0, num_big_rows) have more than 32 chunks
// and get a warp each (lane-strided partial sums, fixed tree); the other long
// rows get a thread each (partials in chunk order). Then the residual
// reduction over the sweep's and this kernel's CTA partials in a fixed order,
// and the device-side convergence test (page_rank.hpp:125-134).
template <int MODE>
__global__ void __launch_bounds__(256) pr_binned_finish_kernel(const BinnedArgs a) {
  __shared__ double s_red[8];
  __shared__ int    s_last;
  PrState*          st = a.sw.st;
  if (*(volatile unsigned int*)&st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&st->iter;
  float* __restrict__ cout = (it & 1ull) ? a.sw.contrib0 : a.sw.contrib1;
  const uint64_t pol = policy_evict_last();
  const int      tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t gt = blockIdx.x * 256u + (uint32_t)tid, gw = gt / 32u;
  double         res = 0.0;
  if (gw < a.num_big_rows) {
    const uint32_t c0 = a.row_first_chunk[gw], c1 = a.row_first_chunk[gw + 1];
    float          p = 0.f;
    for (uint32_t c = c0 + (uint32_t)lane; c < c1; c += 32u) p += __ldcg(a.chunk_part + c);
    p = warp_sum_lane0(p);
    if (lane == 0) res = binned_epilogue<MODE>(a, cout, gw, p, pol);
  } else {
    const uint32_t r = a.num_big_rows + (gt - a.num_big_rows * 32u);
    if (r < a.num_long_rows) {
      const uint32_t c0 = a.row_first_chunk[r], c1 = a.row_first_chunk[r + 1];
      float          p = 0.f;
#pragma unroll 4
      for (uint32_t c = c0; c < c1; ++c) p += __ldcg(a.chunk_part + c);
      res = binned_epilogue<MODE>(a, cout, r, p, pol);
    }
  }
  res = warp_sum_lane0(res);
  if (lane == 0) s_red[warp] = res;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) s += s_red[w];
    a.sw.res_part[a.sw.sweep_grid + blockIdx.x] = s;
    __threadfence();
    s_last = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1u);
  }
  __syncthreads();
  if (!s_last || tid >= 32) return;
  __threadfence();
  const uint32_t parts = a.sw.sweep_grid + gridDim.x;
  double         e = 0.0;
  for (uint32_t u = lane; u < parts; u += 32u) e += __ldcg(a.sw.res_part + u);
  e = warp_sum_lane0(e);
  if (lane == 0) {
    const unsigned long long done_iters = it + 1ull;
    st->iter = done_iters;
    st->last_error = e;
    if constexpr (MODE == kModeRagged) {
      // each graph's stopping test and the loop's continuation are the per-graph convergence kernel's
      st->ticket = 0u;
      __threadfence();
      return;
    }
    if (a.sw.err_hist && it < a.sw.err_cap) a.sw.err_hist[it] = e;  // the first err_cap sweeps
    const bool conv = e < st->threshold;
    const bool abort = a.sw.abort_word && *a.sw.abort_word;
    const bool done = conv || done_iters >= st->max_iters || abort;
    st->converged = conv ? 1u : 0u;
    st->aborted = (abort && !conv) ? 1u : 0u;
    st->done = done ? 1u : 0u;
    st->ticket = 0u;
    __threadfence();
    if (a.sw.use_cond && !done && done_iters < st->chunk_end) cudaGraphSetConditional(a.sw.cond, 1u);
  }
}

// ---------------------------------------------------------------------------
// Set-up: bin boundaries (rows are in non-increasing length order) and the
// chunk table of the long rows.
// ---------------------------------------------------------------------------
// first row whose length is <= len (lengths non-increasing)
__device__ uint32_t first_row_at_most(const uint32_t* row_ptr, uint32_t n, uint32_t len) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (row_ptr[mid + 1] - row_ptr[mid] <= len)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

// out[0] = end of long rows, out[1..kNumBins] = ends of bins 0..kNumBins-1,
// out[kNumBins + 1] = end of the rows of more than 32 chunks; flag = 1 if the
// lengths are not non-increasing (then the binned sweep cannot be used).
__global__ void bin_bounds_kernel(const uint32_t* __restrict__ row_ptr, uint32_t n, uint32_t long_row, uint32_t chunk,
                                  uint32_t* out, unsigned int* unsorted) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t limits[kNumBins] = {long_row, 128, 64, 32, 16, 8, 4, 0};
    for (int b = 0; b < kNumBins; ++b) out[b] = first_row_at_most(row_ptr, n, limits[b]);
    out[kNumBins] = n;
    out[kNumBins + 1] = first_row_at_most(row_ptr, n, 32u * chunk);  // rows of more than 32 chunks
  }
  unsigned int bad = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n; i += gridDim.x * blockDim.x)
    if (row_ptr[i + 2] - row_ptr[i + 1] > row_ptr[i + 1] - row_ptr[i]) bad = 1;
  if (bad) atomicOr(unsorted, 1u);
}

__global__ void chunk_count_kernel(const uint32_t* __restrict__ row_ptr, uint32_t nlong, uint32_t chunk,
                                   uint32_t* __restrict__ cnt) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nlong; r += gridDim.x * blockDim.x) {
    const uint32_t len = row_ptr[r + 1] - row_ptr[r];
    cnt[r] = len / chunk + (len % chunk != 0u ? 1u : 0u);
  }
}

__global__ void chunk_fill_kernel(const uint32_t* __restrict__ first, uint32_t nlong, uint32_t* __restrict__ chunk_row) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nlong; r += gridDim.x * blockDim.x)
    for (uint32_t c = first[r]; c < first[r + 1]; ++c) chunk_row[c] = r;
}

cudaError_t launch_bin_bounds(const uint32_t* row_ptr, uint32_t n, uint32_t long_row, uint32_t chunk, uint32_t* d_out,
                              unsigned int* d_unsorted, int sms, cudaStream_t s) {
  bin_bounds_kernel<<<sms * 4, 256, 0, s>>>(row_ptr, n, long_row, chunk, d_out, d_unsorted);
  return cudaGetLastError();
}
cudaError_t launch_chunk_count(const uint32_t* row_ptr, uint32_t nlong, uint32_t chunk, uint32_t* cnt, int sms,
                               cudaStream_t s) {
  if (!nlong) return cudaSuccess;
  chunk_count_kernel<<<sms, 256, 0, s>>>(row_ptr, nlong, chunk, cnt);
  return cudaGetLastError();
}
cudaError_t launch_chunk_fill(const uint32_t* first, uint32_t nlong, uint32_t* chunk_row, int sms, cudaStream_t s) {
  if (!nlong) return cudaSuccess;
  chunk_fill_kernel<<<sms, 256, 0, s>>>(first, nlong, chunk_row);
  return cudaGetLastError();
}

// Dynamic shared memory of the hot variant: the largest opt-in size less the
// kernel's static shared memory and a margin.
static int binned_hot_smem_bytes() {
  int dev = 0, bytes = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) bytes = 232448;
  bytes -= 1024;
  return bytes > 0 ? bytes & ~15 : 0;
}

uint32_t binned_hot_capacity() { return (uint32_t)(binned_hot_smem_bytes() / 4) & ~3u; }

cudaError_t configure_binned_kernels() {
  void* const hot[] = {(void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModePlain>,
                       (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModeWeighted>,
                       (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModeAdjoint>,
                       (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModeResidual>,
                       (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModeRagged>};
  for (void* fn : hot) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, binned_hot_smem_bytes());
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int binned_sweep_grid(int sms, bool hot) {
  if (hot) return sms;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pr_binned_sweep_kernel<kBinnedThreads, false, kModePlain>,
                                                    kBinnedThreads, 0) !=
          cudaSuccess ||
      nb < 1)
    nb = 1;
  return sms * nb;
}

// Plain sweeps come in both launch shapes; the weighted and adjoint sweeps in
// the hot shape only.
static void* binned_fn(bool hot, int mode) {
  if (mode == kModeWeighted) return (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModeWeighted>;
  if (mode == kModeAdjoint) return (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModeAdjoint>;
  if (mode == kModeResidual) return (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModeResidual>;
  if (mode == kModeRagged) return (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModeRagged>;
  return hot ? (void*)pr_binned_sweep_kernel<kBinnedHotThreads, true, kModePlain>
             : (void*)pr_binned_sweep_kernel<kBinnedThreads, false, kModePlain>;
}
static void* binned_finish_fn(int mode) {
  if (mode == kModeWeighted) return (void*)pr_binned_finish_kernel<kModeWeighted>;
  if (mode == kModeAdjoint) return (void*)pr_binned_finish_kernel<kModeAdjoint>;
  if (mode == kModeResidual) return (void*)pr_binned_finish_kernel<kModeResidual>;
  if (mode == kModeRagged) return (void*)pr_binned_finish_kernel<kModeRagged>;
  return (void*)pr_binned_finish_kernel<kModePlain>;
}
static bool binned_shape_hot(bool hot, int mode) { return hot || mode != kModePlain; }

int binned_finish_grid(const BinnedArgs& a) {
  const uint64_t threads = (uint64_t)a.num_big_rows * 32u + (a.num_long_rows - a.num_big_rows);
  const uint64_t blocks = (threads + 255u) / 256u;
  return blocks ? (int)blocks : 1;
}

cudaError_t launch_binned_sweep(const BinnedArgs& a, bool hot, int mode, int sweep_grid, int finish_grid, cudaStream_t s) {
  void*       args[] = {(void*)&a};
  const bool  h = binned_shape_hot(hot, mode);
  cudaError_t e = cudaLaunchKernel(binned_fn(hot, mode), dim3((unsigned)sweep_grid),
                                   dim3(h ? kBinnedHotThreads : kBinnedThreads), args, h ? (size_t)a.smem_ids * 4u : 0u, s);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernel(binned_finish_fn(mode), dim3((unsigned)finish_grid), dim3(256), args, 0, s);
}

cudaError_t add_binned_nodes(cudaGraph_t body, const BinnedArgs& a, bool hot, int mode, int sweep_grid, int finish_grid,
                             cudaGraphNode_t* finish_node) {
  void*                args[] = {(void*)&a};
  const bool           h = binned_shape_hot(hot, mode);
  cudaKernelNodeParams kp = {};
  kp.func = binned_fn(hot, mode);
  kp.gridDim = dim3((unsigned)sweep_grid);
  kp.blockDim = dim3(h ? kBinnedHotThreads : kBinnedThreads);
  kp.sharedMemBytes = h ? (unsigned)a.smem_ids * 4u : 0u;
  kp.kernelParams = args;
  cudaGraphNode_t sn, fn;
  cudaError_t     e = cudaGraphAddKernelNode(&sn, body, nullptr, 0, &kp);
  if (e != cudaSuccess) return e;
  cudaKernelNodeParams fp = {};
  fp.func = binned_finish_fn(mode);
  fp.gridDim = dim3((unsigned)finish_grid);
  fp.blockDim = dim3(256);
  fp.kernelParams = args;
  e = cudaGraphAddKernelNode(&fn, body, &sn, 1, &fp);
  if (e == cudaSuccess && finish_node) *finish_node = fn;
  return e;
}

}  // namespace nwgpu
