// Device graph construction: CSR from an edge list, and seeded edge-list
// generators (RMAT, 4-neighbour grid).
//
// nwgpu_csr_from_edges does on the device what the reference's build steps do
// on the host (include/nwgraph/build.hpp): fill_directed (:209-232) indexes
// the edges by one endpoint and lists the other; fill_undirected (:235-272)
// lists every edge in both directions; uniq (:394-402) drops repeated
// (row, col) pairs; remove_self_loops (:404-410) drops u == v edges; the
// degree vector is the bench's count of column occurrences
// (bench/gapbs/common.hpp:110-121). Here the edges become packed 64-bit
// (row, col) keys; a radix sort (rows come out sorted by column, as with
// fill(..., sort_adjacency = true)) and a unique pass do uniq on the edge
// list; undirected lists then get the swapped keys appended and sorted again
// (so, as in the reference, (u, v) and (v, u) both listed give two entries
// per row unless the entries are made unique too); one binary search per row
// gives the row pointers, and a histogram the degrees.
//
// The generators reproduce the host builder's samples exactly (graphgen.cpp:
// splitmix64's finaliser as a counter-based hash of (seed, sample, level),
// 32-bit thresholds per level), so RMAT edges generated and built here give
// the same CSR as nwgen_rmat.
#include <cmath>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include "common.cuh"
#include "handle.h"

namespace nwgpu {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
uint64_t mix64_host(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Packed key of entry (row, col): row << cbits | col. Dropped edges get the
// all-ones key of 2 * cbits bits, which sorts after every real key (a real
// key can equal it only as the self-loop of vertex 2^cbits - 1, which is
// dropped too).
__global__ void edge_keys_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t m,
                                 uint64_t n, int by_source, int drop_loops, int cbits, uint64_t* __restrict__ keys,
                                 unsigned int* __restrict__ err, unsigned long long* __restrict__ dropped) {
  const uint64_t sent = (cbits == 32) ? ~0ull : ((1ull << (2 * cbits)) - 1ull);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned int   bad = 0;
  unsigned long long drop = 0;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const uint32_t u = src[e], v = dst[e];
    const bool     invalid = (uint64_t)u >= n || (uint64_t)v >= n;
    const bool     gone = invalid || (drop_loops && u == v);
    bad |= invalid ? 1u : 0u;
    const uint64_t row = by_source ? u : v, col = by_source ? v : u;
    keys[e] = gone ? sent : ((row << cbits) | col);
    drop += gone ? 1u : 0u;
  }
  bad = __reduce_or_sync(kFullMask, bad);
  for (int o = 16; o; o >>= 1) drop += __shfl_xor_sync(kFullMask, drop, o);
  if ((threadIdx.x & 31) == 0) {
    if (bad) atomicOr(err, bad);
    if (drop) atomicAdd(dropped, drop);
  }
}

// keys[m + k] = keys[k] with row and column swapped (fill_undirected's second copy).
__global__ void swap_keys_kernel(uint64_t* __restrict__ keys, uint64_t m, int cbits) {
  const uint64_t mask = (cbits == 32) ? 0xFFFFFFFFull : ((1ull << cbits) - 1ull);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride) {
    const uint64_t x = keys[k];
    keys[m + k] = ((x & mask) << cbits) | (x >> cbits);
  }
}

// row_ptr[r] = first entry whose row is >= r (r = 0..n).
__global__ void row_bounds_kernel(const uint64_t* __restrict__ keys, uint64_t nnz, uint64_t n, int cbits,
                                  uint32_t* __restrict__ row_ptr) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += stride) {
    const uint64_t want = r << cbits;
    uint64_t       lo = 0, hi = nnz;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (keys[mid] < want)
        lo = mid + 1;
      else
        hi = mid;
    }
    row_ptr[r] = (uint32_t)lo;
  }
}

__global__ void key_cols_kernel(const uint64_t* __restrict__ keys, uint64_t nnz, int cbits, uint32_t* __restrict__ col,
                                uint32_t* __restrict__ deg) {
  const uint64_t mask = (cbits == 32) ? 0xFFFFFFFFull : ((1ull << cbits) - 1ull);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
    const uint32_t c = (uint32_t)(keys[k] & mask);
    col[k] = c;
    if (deg) atomicAdd(deg + c, 1u);
  }
}

// graphgen.cpp's rmat_sample: `scale` levels, two 32-bit draws per 64-bit hash.
__global__ void rmat_edges_kernel(int scale, uint64_t m, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t key0,
                                  uint64_t fold, uint32_t* __restrict__ src, uint32_t* __restrict__ dst) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const uint64_t key = key0 ^ (e * 0xD6E8FEB86659FD93ull);
    uint32_t       s = 0, d = 0;
    uint64_t       h = 0;
    for (int l = 0; l < scale; ++l) {
      if ((l & 1) == 0) h = mix64(key + (uint64_t)(l >> 1));
      const uint32_t r = (l & 1) ? (uint32_t)(h >> 32) : (uint32_t)h;
      const uint32_t sb = r >= tab ? 1u : 0u;
      const uint32_t db = (r >= ta && r < tab) || r >= tabc ? 1u : 0u;
      s = (s << 1) | sb;
      d = (d << 1) | db;
    }
    src[e] = fold ? (uint32_t)(s % fold) : s;
    dst[e] = fold ? (uint32_t)(d % fold) : d;
  }
}

// Horizontal edges (v, v + 1) first, then vertical (v, v + side).
__global__ void grid_edges_kernel(uint64_t side, uint32_t* __restrict__ src, uint32_t* __restrict__ dst) {
  const uint64_t h = side * (side - 1), m = 2 * h;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    uint64_t u, v;
    if (e < h) {
      const uint64_t r = e / (side - 1), q = e % (side - 1);
      u = r * side + q;
      v = u + 1;
    } else {
      u = e - h;
      v = u + side;
    }
    src[e] = (uint32_t)u;
    dst[e] = (uint32_t)v;
  }
}

int bit_width(uint64_t x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

struct Scratch {
  cudaStream_t       s;
  std::vector<void*> ptrs;
  template <class T>
  cudaError_t get(T** p, uint64_t count) {
    cudaError_t e = pool_alloc_n(p, count + kPad, s);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
  ~Scratch() {
    for (void* p : ptrs) pool_free(p, s);
    cudaStreamSynchronize(s);
  }
};

}  // namespace
}  // namespace nwgpu

using namespace nwgpu;

extern "C" {

int nwgpu_csr_from_edges(const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n, uint32_t flags,
                         uint32_t* row_ptr, uint32_t* col, uint64_t col_capacity, uint64_t* nnz_out, uint32_t* degrees,
                         void* stream) {
  clear_error();
  if (!row_ptr || !nnz_out) return fail(NWGPU_ERR_INVALID_ARG, "row_ptr / nnz is NULL");
  if (m && (!src || !dst)) return fail(NWGPU_ERR_INVALID_ARG, "src / dst is NULL with m > 0");
  if (n == 0 || n >= 0xFFFFFFF0ull) return fail(NWGPU_ERR_INVALID_ARG, "n = %llu outside [1, 2^32 - 16)", (unsigned long long)n);
  const bool     dev = (flags & NWGPU_EDGES_DEVICE_PTRS) != 0;
  const bool     undirected = (flags & NWGPU_EDGES_UNDIRECTED) != 0;
  const uint64_t total = undirected ? 2 * m : m;
  if (total >= 0xFFFFFFF0ull)
    return fail(NWGPU_ERR_INVALID_ARG, "%llu entries before clean-up do not fit uint32 row pointers",
                (unsigned long long)total);
  int dev_id, sms;
  int rc = check_device(&dev_id, &sms);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  Scratch      sc{s, {}};
  const int    cbits = bit_width(n - 1) ? bit_width(n - 1) : 1;
  const int    end_bit = 2 * cbits;
  const uint32_t *d_src = src, *d_dst = dst;
  if (!dev && m) {
    uint32_t *a = nullptr, *b = nullptr;
    CK(sc.get(&a, m), "cudaMalloc(edges)");
    CK(sc.get(&b, m), "cudaMalloc(edges)");
    CK(cudaMemcpyAsync(a, src, m * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "upload edges");
    CK(cudaMemcpyAsync(b, dst, m * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "upload edges");
    d_src = a;
    d_dst = b;
  }
  uint64_t *keys = nullptr, *sorted = nullptr;
  unsigned int*       d_err = nullptr;
  unsigned long long* d_drop = nullptr;
  uint64_t*           d_nsel = nullptr;
  CK(sc.get(&keys, total), "cudaMalloc(keys)");
  CK(sc.get(&sorted, total), "cudaMalloc(keys)");
  CK(sc.get(&d_err, 1), "cudaMalloc(flags)");
  CK(sc.get(&d_drop, 1), "cudaMalloc(flags)");
  CK(sc.get(&d_nsel, 1), "cudaMalloc(flags)");
  CK(cudaMemsetAsync(d_err, 0, sizeof(unsigned int), s), "memset");
  CK(cudaMemsetAsync(d_drop, 0, sizeof(unsigned long long), s), "memset");
  if (m) {
    edge_keys_kernel<<<sms * 8, 256, 0, s>>>(d_src, d_dst, m, n, (flags & NWGPU_EDGES_BY_SOURCE) ? 1 : 0,
                                              (flags & NWGPU_EDGES_REMOVE_SELF_LOOPS) ? 1 : 0, cbits, keys, d_err,
                                              d_drop);
    CK(cudaGetLastError(), "edge keys");
  }
  unsigned int       h_err = 0;
  unsigned long long h_drop = 0;
  CK(cudaMemcpyAsync(&h_err, d_err, sizeof(h_err), cudaMemcpyDeviceToHost, s), "copy flags");
  CK(cudaMemcpyAsync(&h_drop, d_drop, sizeof(h_drop), cudaMemcpyDeviceToHost, s), "copy flags");
  CK(cudaStreamSynchronize(s), "edge keys");
  if (h_err) return fail(NWGPU_ERR_INVALID_GRAPH, "edge endpoint >= n = %llu", (unsigned long long)n);
  size_t sort_bytes = 0, uniq_bytes = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, keys, sorted, (int64_t)total, 0, end_bit, s), "sort size");
  CK(cub::DeviceSelect::Unique(nullptr, uniq_bytes, sorted, keys, d_nsel, (int64_t)total, s), "unique size");
  void* tmp = nullptr;
  CK(sc.get(reinterpret_cast<unsigned char**>(&tmp), sort_bytes > uniq_bytes ? sort_bytes : uniq_bytes), "cudaMalloc(tmp)");
  // sorted [0, count) of `in` into `out`; optionally unique back into `in`
  uint64_t* cur = keys;   // holds the current key list
  uint64_t* other = sorted;
  uint64_t  count = m;
  auto      sort_unique = [&](bool unique) -> int {
    if (count) CK(cub::DeviceRadixSort::SortKeys(tmp, sort_bytes, cur, other, (int64_t)count, 0, end_bit, s), "sort");
    std::swap(cur, other);
    if (unique && count) {
      CK(cub::DeviceSelect::Unique(tmp, uniq_bytes, cur, other, d_nsel, (int64_t)count, s), "unique");
      CK(cudaMemcpyAsync(&count, d_nsel, sizeof(uint64_t), cudaMemcpyDeviceToHost, s), "copy count");
      CK(cudaStreamSynchronize(s), "unique");
      std::swap(cur, other);
    }
    return NWGPU_OK;
  };
  // the edge list: dropped edges sort last and are cut off; uniq
  if ((rc = sort_unique((flags & NWGPU_EDGES_UNIQUE) != 0))) return rc;
  if (!(flags & NWGPU_EDGES_UNIQUE)) count = m - h_drop;
  else if (h_drop) count -= 1;  // the one remaining all-ones key of the dropped edges
  if (undirected) {
    if (count) {
      swap_keys_kernel<<<sms * 8, 256, 0, s>>>(cur, count, cbits);
      CK(cudaGetLastError(), "swap keys");
    }
    count *= 2;
    if ((rc = sort_unique((flags & NWGPU_EDGES_UNIQUE_ENTRIES) != 0))) return rc;
  } else if (flags & NWGPU_EDGES_UNIQUE_ENTRIES) {
    if ((rc = sort_unique(true))) return rc;
  }
  const uint64_t  nnz = count;
  const uint64_t* final_keys = cur;
  *nnz_out = nnz;
  if (nnz > col_capacity || (nnz && !col))
    return fail(NWGPU_ERR_INVALID_ARG, "col holds %llu entries, the graph has %llu", (unsigned long long)col_capacity,
                (unsigned long long)nnz);
  // Row pointers, columns and degrees (device staging when the outputs are host arrays).
  uint32_t *o_rp = row_ptr, *o_col = col, *o_deg = degrees;
  if (!dev) {
    CK(sc.get(&o_rp, n + 1), "cudaMalloc(row_ptr)");
    CK(sc.get(&o_col, nnz), "cudaMalloc(col)");
    if (degrees) CK(sc.get(&o_deg, n), "cudaMalloc(degrees)");
  }
  if (o_deg) CK(cudaMemsetAsync(o_deg, 0, n * sizeof(uint32_t), s), "memset degrees");
  row_bounds_kernel<<<sms * 8, 256, 0, s>>>(final_keys, nnz, n, cbits, o_rp);
  CK(cudaGetLastError(), "row bounds");
  if (nnz) {
    key_cols_kernel<<<sms * 8, 256, 0, s>>>(final_keys, nnz, cbits, o_col, o_deg);
    CK(cudaGetLastError(), "columns");
  }
  if (!dev) {
    CK(cudaMemcpyAsync(row_ptr, o_rp, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy row_ptr");
    if (nnz) CK(cudaMemcpyAsync(col, o_col, nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy col");
    if (degrees) CK(cudaMemcpyAsync(degrees, o_deg, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy degrees");
  }
  CK(cudaStreamSynchronize(s), "csr build");
  return NWGPU_OK;
}

int nwgpu_rmat_edges(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed, uint64_t n, uint32_t* src,
                     uint32_t* dst, void* stream) {
  clear_error();
  if (scale < 1 || scale > 31) return fail(NWGPU_ERR_INVALID_ARG, "scale %u outside [1, 31]", scale);
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) return fail(NWGPU_ERR_INVALID_ARG, "bad quadrant probabilities");
  if (n > (1ull << scale)) return fail(NWGPU_ERR_INVALID_ARG, "n = %llu > 2^scale", (unsigned long long)n);
  if (m && (!src || !dst)) return fail(NWGPU_ERR_INVALID_ARG, "src / dst is NULL");
  int dev_id, sms;
  int rc = check_device(&dev_id, &sms);
  if (rc) return rc;
  auto thr = [](double x) -> uint32_t {
    const double v = std::floor(x * 4294967296.0);
    return v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
  };
  if (m) {
    rmat_edges_kernel<<<sms * 8, 256, 0, (cudaStream_t)stream>>>((int)scale, m, thr(a), thr(a + b), thr(a + b + c),
                                                                  mix64_host(seed), n == (1ull << scale) ? 0 : n, src, dst);
    CK(cudaGetLastError(), "rmat edges");
  }
  return NWGPU_OK;
}

int nwgpu_grid_edges(uint64_t side, uint32_t* src, uint32_t* dst, void* stream) {
  clear_error();
  if (side < 1 || side * side >= 0xFFFFFFF0ull) return fail(NWGPU_ERR_INVALID_ARG, "side %llu", (unsigned long long)side);
  if (side > 1 && (!src || !dst)) return fail(NWGPU_ERR_INVALID_ARG, "src / dst is NULL");
  int dev_id, sms;
  int rc = check_device(&dev_id, &sms);
  if (rc) return rc;
  if (side > 1) {
    grid_edges_kernel<<<sms * 8, 256, 0, (cudaStream_t)stream>>>(side, src, dst);
    CK(cudaGetLastError(), "grid edges");
  }
  return NWGPU_OK;
}

}  // extern "C"
