// Graph set-up on the device: validation, degree-ordered relabelling and
// merge-path tiling of the uploaded CSR.
//
// Relabelling: vertices are renumbered by descending row length, stably. Rows
// of similar length become contiguous (the binned sweep's bins need no index
// lists) and, on symmetric graphs, the hub vertices that most gathers hit get
// the smallest ids. Row i of the relabelled CSR is
// row inv[i] of the input with its entries in their original order and each
// column id mapped through perm, so every row is summed over the same terms in
// the same order as the input row (page_rank.hpp:129-131). Ranks go back to
// input order when a solve finishes.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "engine.h"

namespace nwgpu {

// ---------------------------------------------------------------------------
// Validation: bit 0 row_ptr[0] != 0 or row_ptr[n] != nnz; bit 1 row_ptr
// decreases; bit 2 some col >= n. Reads only in-bounds entries whatever the
// contents, so it is safe on arbitrary input.
// ---------------------------------------------------------------------------
__global__ void validate_kernel(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col, uint64_t n,
                                uint64_t nnz, unsigned int* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int   bad = 0;
  if (tid == 0 && (row_ptr[0] != 0 || (uint64_t)row_ptr[n] != nnz)) bad |= 1u;
  for (uint64_t i = tid; i < n; i += stride)
    if (row_ptr[i + 1] < row_ptr[i]) bad |= 2u;
  if (col)
    for (uint64_t k = tid; k < nnz; k += stride)
      if ((uint64_t)__ldcs(col + k) >= n) bad |= 4u;
  bad = __reduce_or_sync(kFullMask, bad);
  if ((threadIdx.x & 31) == 0 && bad) atomicOr(err, bad);
}

cudaError_t validate_csr(const uint32_t* d_row_ptr, const uint32_t* d_col, uint64_t n, uint64_t nnz,
                         unsigned int* d_err, int sms, cudaStream_t s) {
  validate_kernel<<<sms * 8, 256, 0, s>>>(d_row_ptr, d_col, n, nnz, d_err);
  return cudaGetLastError();
}

// The row pointers alone (bits 0 and 1): the streamed build checks them before
// any kernel indexes with them, while the column ids are still arriving.
cudaError_t validate_row_ptr(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, unsigned int* d_err, int sms,
                             cudaStream_t s) {
  validate_kernel<<<sms * 8, 256, 0, s>>>(d_row_ptr, nullptr, n, nnz, d_err);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Merge-path tiling
// ---------------------------------------------------------------------------
// Row i such that the first d merge items are rows [0, i) and entries [0, d - i).
__device__ __forceinline__ uint32_t merge_path_row(const uint32_t* row_ptr, uint64_t n, uint64_t nnz, uint64_t d) {
  uint64_t lo = d > nnz ? d - nnz : 0;
  uint64_t hi = d < n ? d : n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if ((uint64_t)row_ptr[mid + 1] + mid + 1 <= d)  // row mid's end item lies before d
      lo = mid + 1;
    else
      hi = mid;
  }
  return (uint32_t)lo;
}

__global__ void tiling_kernel(const uint32_t* __restrict__ row_ptr, uint64_t n, uint64_t nnz, uint32_t D,
                              uint32_t num_tiles, uint32_t* __restrict__ tile_row, uint32_t* __restrict__ tile_nnz) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > num_tiles) return;
  uint64_t d = t * D;
  if (d > n + nnz) d = n + nnz;
  const uint32_t i = merge_path_row(row_ptr, n, nnz, d);
  tile_row[t] = i;
  tile_nnz[t] = (uint32_t)(d - i);
}

cudaError_t build_tiling(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, uint32_t D, Tiling* t, cudaStream_t s) {
  const uint64_t tiles = (n + nnz + D - 1) / D;
  if (tiles >= 0xFFFFFFF0ull || D == 0) return cudaErrorInvalidValue;
  t->tile_items = D;
  t->num_tiles = (uint32_t)tiles;
  cudaError_t e = pool_alloc_n(&t->tile_row, tiles + 2, s);
  if (e != cudaSuccess) return e;
  e = pool_alloc_n(&t->tile_nnz, tiles + 2, s);
  if (e != cudaSuccess) return e;
  const unsigned blocks = (unsigned)((tiles + 1 + 255) / 256);
  tiling_kernel<<<blocks, 256, 0, s>>>(d_row_ptr, n, nnz, (uint32_t)D, (uint32_t)tiles, t->tile_row, t->tile_nnz);
  return cudaGetLastError();
}

cudaError_t fill_tiling(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, uint32_t D, uint32_t num_tiles,
                        uint32_t* tile_row, uint32_t* tile_nnz, cudaStream_t s) {
  if (D == 0 || (uint64_t)num_tiles * D < n + nnz) return cudaErrorInvalidValue;
  const unsigned blocks = (unsigned)(((uint64_t)num_tiles + 1 + 255) / 256);
  tiling_kernel<<<blocks, 256, 0, s>>>(d_row_ptr, n, nnz, D, num_tiles, tile_row, tile_nnz);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Ragged batches: per-graph tiling and validation
// ---------------------------------------------------------------------------
// Last graph g whose key(g) <= x, for a key non-decreasing in g.
template <class Key>
__device__ __forceinline__ uint32_t last_graph_at_or_below(uint32_t num_graphs, uint64_t x, Key key) {
  uint32_t lo = 0, hi = num_graphs - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (key(mid) <= x)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Entry e of the tile tables belongs to the graph g with tile0 + g <= e <
// tile0 + g + tiles + 1 (each graph has its tiles plus one end entry).
__global__ void ragged_tiling_kernel(const RaggedGraph* __restrict__ graphs, uint32_t num_graphs,
                                     const uint32_t* __restrict__ row_ptr, uint32_t D, uint64_t entries,
                                     uint32_t* __restrict__ tile_row, uint32_t* __restrict__ tile_nnz) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < entries; e += stride) {
    const uint32_t g = last_graph_at_or_below(num_graphs, e, [&](uint32_t x) { return (uint64_t)graphs[x].tile0 + x; });
    const RaggedGraph R = graphs[g];
    const uint64_t    j = e - ((uint64_t)R.tile0 + g);
    const uint64_t    items = (uint64_t)R.n + R.nnz;
    const uint64_t    d = j * D < items ? j * D : items;
    const uint32_t    i = merge_path_row(row_ptr + R.p0, R.n, R.nnz, d);
    tile_row[e] = i;
    tile_nnz[e] = (uint32_t)(d - i);
  }
}

cudaError_t fill_ragged_tiling(const RaggedGraph* graphs, uint32_t num_graphs, const uint32_t* row_ptr,
                               uint32_t num_tiles, uint32_t* tile_row, uint32_t* tile_nnz, int sms, cudaStream_t s) {
  if (!num_graphs) return cudaSuccess;
  ragged_tiling_kernel<<<sms * 8, 256, 0, s>>>(graphs, num_graphs, row_ptr, kRaggedTileItems,
                                                (uint64_t)num_tiles + num_graphs, tile_row, tile_nnz);
  return cudaGetLastError();
}

// Bits as validate_kernel: 1 a graph's row pointers do not start at 0 or end
// at its nnz, 2 they decrease, 4 a column id >= the graph's n.
__global__ void validate_ragged_kernel(const RaggedGraph* __restrict__ graphs, uint32_t num_graphs,
                                       const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col,
                                       uint64_t num_row_ptrs, uint64_t num_entries, unsigned int* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int   bad = 0;
  for (uint64_t q = tid; q < num_row_ptrs; q += stride) {
    const uint32_t g = last_graph_at_or_below(num_graphs, q, [&](uint32_t x) { return graphs[x].p0; });
    const uint64_t i = q - graphs[g].p0;
    const uint32_t v = row_ptr[q];
    if (i == 0 && v != 0u) bad |= 1u;
    if (i == graphs[g].n && v != graphs[g].nnz) bad |= 1u;
    if (i < graphs[g].n && row_ptr[q + 1] < v) bad |= 2u;
  }
  for (uint64_t k = tid; k < num_entries; k += stride) {
    const uint32_t g = last_graph_at_or_below(num_graphs, k, [&](uint32_t x) { return graphs[x].e0; });
    if (__ldcs(col + k) >= graphs[g].n) bad |= 4u;
  }
  bad = __reduce_or_sync(kFullMask, bad);
  if ((threadIdx.x & 31) == 0 && bad) atomicOr(err, bad);
}

cudaError_t validate_ragged(const RaggedGraph* graphs, uint32_t num_graphs, const uint32_t* row_ptr, const uint32_t* col,
                            uint64_t num_row_ptrs, uint64_t num_entries, unsigned int* err, int sms, cudaStream_t s) {
  if (!num_graphs) return cudaSuccess;
  validate_ragged_kernel<<<sms * 8, 256, 0, s>>>(graphs, num_graphs, row_ptr, col, num_row_ptrs, num_entries, err);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Relabelling
// ---------------------------------------------------------------------------
// Sort key: row length (in-degree). For the symmetric graphs of the benchmark
// this equals the out-degree, i.e. how often a vertex's contribution is gathered.
__global__ void row_length_kernel(const uint32_t* __restrict__ row_ptr, uint64_t n, uint32_t* __restrict__ len) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) len[i] = row_ptr[i + 1] - row_ptr[i];
}

__global__ void iota_kernel(uint32_t* __restrict__ v, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) v[i] = (uint32_t)i;
}

// perm[inv[i]] = i; new row lengths.
__global__ void invert_kernel(const uint32_t* __restrict__ inv, const uint32_t* __restrict__ row_ptr, uint64_t n,
                              uint32_t* __restrict__ perm, uint32_t* __restrict__ new_len) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t o = inv[i];
    perm[o] = (uint32_t)i;
    new_len[i] = row_ptr[o + 1] - row_ptr[o];
  }
}

// Fill the relabelled CSR one merge-path tile of the NEW row_ptr at a time:
// for new entry p in row i (new id), the source entry is
// old_row_ptr[inv[i]] + (p - new_row_ptr[i]).
template <int NT>
__global__ void __launch_bounds__(NT) permute_entries_kernel(const uint32_t* __restrict__ new_row_ptr,
                                                              const uint32_t* __restrict__ tile_row,
                                                              const uint32_t* __restrict__ tile_nnz, uint32_t num_tiles,
                                                              const uint32_t* __restrict__ inv,
                                                              const uint32_t* __restrict__ perm,
                                                              const uint32_t* __restrict__ old_row_ptr,
                                                              const uint32_t* __restrict__ old_col,
                                                              const float* __restrict__ old_w, uint32_t* __restrict__ col,
                                                              float* __restrict__ w, uint32_t* __restrict__ emap,
                                                              uint32_t D) {
  extern __shared__ uint32_t sm[];
  uint32_t* s_new = sm;          // new_row_ptr[r0 .. r1+1]
  uint32_t* s_old = sm + D + 2;  // old start of rows r0 .. r1
  for (uint32_t t = blockIdx.x; t < num_tiles; t += gridDim.x) {
    const uint32_t r0 = tile_row[t], r1 = tile_row[t + 1], k0 = tile_nnz[t], k1 = tile_nnz[t + 1];
    const uint32_t rows = r1 - r0 + 1;  // includes the (possibly partial) row r1
    for (uint32_t j = threadIdx.x; j <= rows; j += NT) s_new[j] = new_row_ptr[r0 + j];
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < rows; j += NT) {
      const uint32_t r = r0 + j;
      s_old[j] = (s_new[j] < s_new[j + 1]) ? old_row_ptr[inv[r]] : 0u;  // rows without entries here are never read
    }
    __syncthreads();
    for (uint32_t p = k0 + threadIdx.x; p < k1; p += NT) {
      // row of entry p among rows r0..r1: last j with s_new[j] <= p
      uint32_t lo = 0, hi = rows;  // answer in [0, rows)
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_new[mid] <= p)
          lo = mid;
        else
          hi = mid;
      }
      const uint32_t src = s_old[lo] + (p - s_new[lo]);
      col[p] = perm[old_col[src]];
      if (w) w[p] = old_w[src];
      if (emap) emap[p] = src;
    }
    __syncthreads();
  }
}

// The input entries of merge-path items [d0, d1) of the input CSR, each
// copied to its place in the relabelled CSR with its id mapped: entry p of
// input row o goes to new_row_ptr[perm[o]] + (p - old_row_ptr[o]). Reads the
// input coalesced, so a chunk can be placed as soon as it has arrived; the
// row pointers must be valid (validate_row_ptr). Ids >= n set bit 2 of *err
// and are written as 0, so no load or store leaves its array.
template <int NT>
__global__ void __launch_bounds__(NT) scatter_entries_kernel(const uint32_t* __restrict__ old_row_ptr,
                                                              const uint32_t* __restrict__ old_col, uint64_t n,
                                                              uint64_t nnz, uint64_t d0, uint64_t d1,
                                                              const uint32_t* __restrict__ perm,
                                                              const uint32_t* __restrict__ new_row_ptr,
                                                              uint32_t* __restrict__ col, unsigned int* err, uint32_t D) {
  extern __shared__ uint32_t sm[];
  __shared__ uint32_t        s_pt[2];
  uint32_t*                  s_old = sm;          // old_row_ptr[i0 + j]
  uint32_t*                  s_dst = sm + D + 2;  // new start of row i0 + j
  unsigned int               bad = 0;
  const uint64_t             tiles = (d1 - d0 + D - 1) / D;
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint64_t a = d0 + t * D, b = min(a + (uint64_t)D, d1);
    if (threadIdx.x < 2) s_pt[threadIdx.x] = merge_path_row(old_row_ptr, n, nnz, threadIdx.x ? b : a);
    __syncthreads();
    const uint32_t i0 = s_pt[0], i1 = s_pt[1];
    const uint64_t k0 = a - i0, k1 = b - i1;
    // rows i0 .. min(i1, n - 1) hold this tile's entries (at most D + 1 rows)
    const uint32_t rows = (i1 < n ? i1 : (uint32_t)(n - 1)) - i0 + 1;
    for (uint32_t j = threadIdx.x; j < rows; j += NT) {
      s_old[j] = old_row_ptr[i0 + j];
      s_dst[j] = new_row_ptr[perm[i0 + j]];
    }
    __syncthreads();
    for (uint64_t p = k0 + threadIdx.x; p < k1; p += NT) {
      uint32_t lo = 0, hi = rows;  // last j with s_old[j] <= p
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_old[mid] <= p)
          lo = mid;
        else
          hi = mid;
      }
      uint32_t c = __ldcs(old_col + p);
      if ((uint64_t)c >= n) {
        bad |= 4u;
        c = 0u;
      }
      col[s_dst[lo] + (p - s_old[lo])] = perm[c];
    }
    __syncthreads();
  }
  bad = __reduce_or_sync(kFullMask, bad);
  if ((threadIdx.x & 31) == 0 && bad) atomicOr(err, bad);
}

// The row half of the relabelling: allocates *out's arrays (row_ptr, col,
// perm, inv, and w / emap when with_weights) and computes the id maps and the
// new row pointers. The entries are placed afterwards, all at once
// (permute_entries_kernel) or chunk by chunk (scatter_entries).
cudaError_t relabel_rows(const uint32_t* d_row_ptr, uint64_t n, uint64_t nnz, int sms, bool with_weights,
                         bool clear_entries, Relabelled* out, cudaStream_t s) {
  cudaError_t e;
  uint32_t *cnt = nullptr, *cnt_sorted = nullptr, *ids = nullptr, *new_len = nullptr;
  void*     tmp = nullptr;
  size_t    tmp_bytes = 0, scan_bytes = 0;
  auto      cleanup = [&]() {
    pool_free(cnt, s);
    pool_free(cnt_sorted, s);
    pool_free(ids, s);
    pool_free(new_len, s);
    pool_free(tmp, s);
  };
#define RK(x)                \
  do {                       \
    if ((e = (x)) != cudaSuccess) { \
      cleanup();             \
      return e;              \
    }                        \
  } while (0)
  const int grid = sms * 8;
  RK(pool_alloc_n(&cnt, n + 1, s));
  RK(pool_alloc_n(&cnt_sorted, n + 1, s));
  RK(pool_alloc_n(&ids, n + 1, s));
  RK(pool_alloc_n(&new_len, n + 1, s));
  RK(pool_alloc_n(&out->inv, n + kPad, s));
  RK(pool_alloc_n(&out->perm, n + kPad, s));
  RK(pool_alloc_n(&out->row_ptr, n + 1 + kPad, s));
  RK(pool_alloc_n(&out->col, nnz + kPad, s));
  RK(cudaMemsetAsync(out->row_ptr, 0, (n + 1 + kPad) * sizeof(uint32_t), s));
  if (clear_entries)
    RK(cudaMemsetAsync(out->col, 0, (nnz + kPad) * sizeof(uint32_t), s));
  else  // every entry is written by the scatter; only the padding is cleared here
    RK(cudaMemsetAsync(out->col + nnz, 0, kPad * sizeof(uint32_t), s));
  if (with_weights) {
    RK(pool_alloc_n(&out->w, nnz + kPad, s));
    RK(cudaMemsetAsync(out->w, 0, (nnz + kPad) * sizeof(float), s));
    RK(pool_alloc_n(&out->emap, nnz + kPad, s));
    RK(cudaMemsetAsync(out->emap, 0, (nnz + kPad) * sizeof(uint32_t), s));
  }
  row_length_kernel<<<grid, 256, 0, s>>>(d_row_ptr, n, cnt);
  RK(cudaGetLastError());
  iota_kernel<<<grid, 256, 0, s>>>(ids, n);
  RK(cudaGetLastError());
  // stable descending sort of vertex ids by gather count
  RK(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, cnt, cnt_sorted, ids, out->inv, (int64_t)n, 0, 32, s));
  RK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, new_len, out->row_ptr, (int64_t)(n + 1), s));
  if (scan_bytes > tmp_bytes) tmp_bytes = scan_bytes;
  RK(pool_alloc(&tmp, tmp_bytes, s));
  size_t b1 = tmp_bytes;
  RK(cub::DeviceRadixSort::SortPairsDescending(tmp, b1, cnt, cnt_sorted, ids, out->inv, (int64_t)n, 0, 32, s));
  invert_kernel<<<grid, 256, 0, s>>>(out->inv, d_row_ptr, n, out->perm, new_len);
  RK(cudaGetLastError());
  RK(cudaMemsetAsync(new_len + n, 0, sizeof(uint32_t), s));
  size_t b2 = tmp_bytes;
  RK(cub::DeviceScan::ExclusiveSum(tmp, b2, new_len, out->row_ptr, (int64_t)(n + 1), s));
  cleanup();
#undef RK
  return cudaSuccess;
}

cudaError_t scatter_entries(const uint32_t* d_row_ptr, const uint32_t* d_col, uint64_t n, uint64_t nnz, uint64_t d0,
                            uint64_t d1, const Relabelled& out, unsigned int* d_err, int sms, cudaStream_t s) {
  if (d1 <= d0 || n == 0) return cudaSuccess;
  const uint32_t D = 2048;
  const size_t   smem = (size_t)(2 * D + 4) * sizeof(uint32_t);
  const uint64_t tiles = (d1 - d0 + D - 1) / D, cap = (uint64_t)sms * 4;
  scatter_entries_kernel<kSweepThreads><<<(unsigned)(tiles < cap ? tiles : cap), kSweepThreads, smem, s>>>(
      d_row_ptr, d_col, n, nnz, d0, d1, out.perm, out.row_ptr, out.col, d_err, D);
  return cudaGetLastError();
}

// Builds the relabelled copy. On success *out holds freshly allocated
// row_ptr / col / (weights) / perm / inv arrays padded for 16-byte bulk loads.
cudaError_t build_relabelled(const uint32_t* d_row_ptr, const uint32_t* d_col, const float* d_w, uint64_t n,
                             uint64_t nnz, int sms, Relabelled* out, cudaStream_t s) {
  cudaError_t e = relabel_rows(d_row_ptr, n, nnz, sms, d_w != nullptr, true, out, s);
  if (e != cudaSuccess) return e;
  // entries: tile the new CSR and copy each tile's entries
  const uint32_t D = 2048;
  Tiling         nt{};
  if ((e = build_tiling(out->row_ptr, n, nnz, D, &nt, s)) == cudaSuccess) {
    const size_t smem = (size_t)(2 * D + 4) * sizeof(uint32_t);
    permute_entries_kernel<kSweepThreads><<<sms * 4, kSweepThreads, smem, s>>>(
        out->row_ptr, nt.tile_row, nt.tile_nnz, nt.num_tiles, out->inv, out->perm, d_row_ptr, d_col, d_w, out->col,
        out->w, out->emap, D);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  pool_free(nt.tile_row, s);
  pool_free(nt.tile_nnz, s);
  return e;
}

// ---------------------------------------------------------------------------
// Transposed CSR (out-rows), for the adjoint solve
// ---------------------------------------------------------------------------
// Row of each entry: the last row whose start is <= k.
__global__ void entry_row_kernel(const uint32_t* __restrict__ row_ptr, uint64_t n, uint64_t nnz,
                                 uint32_t* __restrict__ erow) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
    uint64_t lo = 0, hi = n;  // row_ptr[lo] <= k < row_ptr[hi]
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) >> 1;
      if (row_ptr[mid] <= k)
        lo = mid;
      else
        hi = mid;
    }
    erow[k] = (uint32_t)lo;
  }
}

__global__ void count_cols_kernel(const uint32_t* __restrict__ col, uint64_t nnz, uint32_t* __restrict__ cnt) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) atomicAdd(cnt + col[k], 1u);
}

// Out-entry e is forward entry fwd[e]: its destination row and weight.
__global__ void transpose_fill_kernel(const uint32_t* __restrict__ fwd, const uint32_t* __restrict__ erow,
                                      const float* __restrict__ w, uint64_t nnz, uint32_t* __restrict__ tcol,
                                      float* __restrict__ tw) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
    const uint32_t k = fwd[e];
    tcol[e] = erow[k];
    tw[e] = w ? w[k] : 1.0f;
  }
}

// s_j = sum of the weights of out-row j, in entry order, in FP64.
__global__ void out_weight_kernel(const uint32_t* __restrict__ trow, const float* __restrict__ tw, uint64_t n,
                                  float* __restrict__ s) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
    double acc = 0.0;
    for (uint32_t e = trow[j]; e < trow[j + 1]; ++e) acc += (double)tw[e];
    s[j] = (float)acc;
  }
}

cudaError_t build_transpose(const uint32_t* d_row_ptr, const uint32_t* d_col, const float* d_w, uint64_t n, uint64_t nnz,
                            int sms, Transposed* out, cudaStream_t s) {
  cudaError_t e;
  uint32_t *ids = nullptr, *keys = nullptr, *cnt = nullptr;
  void*     tmp = nullptr;
  size_t    sort_bytes = 0, scan_bytes = 0;
  auto      cleanup = [&]() {
    pool_free(ids, s);
    pool_free(keys, s);
    pool_free(cnt, s);
    pool_free(tmp, s);
  };
#define TK(x)                       \
  do {                              \
    if ((e = (x)) != cudaSuccess) { \
      cleanup();                    \
      return e;                     \
    }                               \
  } while (0)
  const int grid = sms * 8;
  TK(pool_alloc_n(&out->erow, nnz + kPad, s));
  uint32_t* erow = out->erow;
  TK(pool_alloc_n(&ids, nnz + kPad, s));
  TK(pool_alloc_n(&keys, nnz + kPad, s));
  TK(pool_alloc_n(&cnt, n + 1, s));
  TK(pool_alloc_n(&out->row_ptr, n + 1 + kPad, s));
  TK(pool_alloc_n(&out->col, nnz + kPad, s));
  TK(pool_alloc_n(&out->w, nnz + kPad, s));
  TK(pool_alloc_n(&out->fwd, nnz + kPad, s));
  TK(pool_alloc_n(&out->s, n + kPad, s));
  TK(cudaMemsetAsync(out->row_ptr, 0, (n + 1 + kPad) * sizeof(uint32_t), s));
  TK(cudaMemsetAsync(out->col, 0, (nnz + kPad) * sizeof(uint32_t), s));
  TK(cudaMemsetAsync(out->w, 0, (nnz + kPad) * sizeof(float), s));
  TK(cudaMemsetAsync(out->fwd, 0, (nnz + kPad) * sizeof(uint32_t), s));
  TK(cudaMemsetAsync(out->s, 0, (n + kPad) * sizeof(float), s));
  TK(cudaMemsetAsync(cnt, 0, (n + 1) * sizeof(uint32_t), s));
  if (nnz) {
    entry_row_kernel<<<grid, 256, 0, s>>>(d_row_ptr, n, nnz, erow);
    TK(cudaGetLastError());
    iota_kernel<<<grid, 256, 0, s>>>(ids, nnz);
    TK(cudaGetLastError());
    count_cols_kernel<<<grid, 256, 0, s>>>(d_col, nnz, cnt);
    TK(cudaGetLastError());
  }
  // stable sort of the entries by column: out-row order, entries of one
  // out-row in forward entry order
  int bits = 1;
  while (bits < 32 && (1ull << bits) < n) ++bits;
  TK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, d_col, keys, ids, out->fwd, (int64_t)nnz, 0, bits, s));
  TK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt, out->row_ptr, (int64_t)(n + 1), s));
  TK(pool_alloc(&tmp, sort_bytes > scan_bytes ? sort_bytes : scan_bytes, s));
  if (nnz) TK(cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, d_col, keys, ids, out->fwd, (int64_t)nnz, 0, bits, s));
  TK(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, cnt, out->row_ptr, (int64_t)(n + 1), s));
  if (nnz) {
    transpose_fill_kernel<<<grid, 256, 0, s>>>(out->fwd, erow, d_w, nnz, out->col, out->w);
    TK(cudaGetLastError());
  }
  out_weight_kernel<<<grid, 256, 0, s>>>(out->row_ptr, out->w, n, out->s);
  TK(cudaGetLastError());
  TK(cudaStreamSynchronize(s));
  cleanup();
#undef TK
  return cudaSuccess;
}

}  // namespace nwgpu
