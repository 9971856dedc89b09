// Seeded synthetic graph builder for the PageRank engine's inputs.
//
// The reference ships no RMAT generator (include/nwgraph/generators/ has only
// configuration_model.hpp; GAP's generator lives in the empty submodule
// bench/gapbs-reference). This builder writes the CSR that both the reference
// CPU path and the GPU engine consume, so both sum over identical rows.
//
// RMAT: m = edge_factor * 2^scale samples; sample e descends `scale` levels,
// picking quadrant (0,0),(0,1),(1,0),(1,1) with probabilities a,b,c,d from a
// counter-based hash of (seed, e, level) -- splitmix64's finaliser, 32-bit
// resolution per level -- so the result does not depend on the thread count.
// Clean-up as a symmetrised simple graph: drop self-loops, add the reverse of
// every edge, sort each row ascending and drop duplicates. No relabelling.
// The CSR is adjacency<1> (row i = in-neighbours of i); for these symmetric
// graphs it equals adjacency<0>.
//
// Grid: floor(sqrt(n))^2 vertices, 4-neighbour lattice, rows sorted.
//
// Exported through a C ABI (include/nwgraph_gen.h); buffers are malloc'd here
// and released with nwgen_free.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/nwgraph_gen.h"

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int pick_threads(int requested) {
  if (requested > 0) return requested;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

template <class F>
void parallel_chunks(uint64_t count, int nthreads, F&& f) {
  if (count == 0) return;
  int nt = (int)std::min<uint64_t>((uint64_t)nthreads, count);
  if (nt <= 1) {
    f(0, count, 0);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) {
    uint64_t lo = count * t / nt, hi = count * (t + 1) / nt;
    pool.emplace_back([=, &f] { f(lo, hi, t); });
  }
  for (auto& th : pool) th.join();
}

struct RmatParams {
  int      scale;
  uint64_t m;
  uint32_t ta, tab, tabc;  // cumulative quadrant thresholds on 32-bit draws
  uint64_t seed;
};

inline void rmat_sample(const RmatParams& p, uint64_t e, uint32_t& u, uint32_t& v) {
  uint32_t src = 0, dst = 0;
  uint64_t key = mix64(p.seed) ^ (e * 0xD6E8FEB86659FD93ull);
  uint64_t h = 0;
  for (int l = 0; l < p.scale; ++l) {
    if ((l & 1) == 0) h = mix64(key + (uint64_t)(l >> 1));
    uint32_t r = (l & 1) ? (uint32_t)(h >> 32) : (uint32_t)h;
    uint32_t sb = 0, db = 0;
    if (r < p.ta) {
    } else if (r < p.tab) {
      db = 1;
    } else if (r < p.tabc) {
      sb = 1;
    } else {
      sb = 1;
      db = 1;
    }
    src = (src << 1) | sb;
    dst = (dst << 1) | db;
  }
  u = src;
  v = dst;
}

// Turn per-row candidate lists into a sorted, duplicate-free CSR.
int finish_csr(uint64_t n, std::vector<uint32_t>& off, std::vector<uint32_t>& tmp, int nt, nwgen_csr* out) {
  std::vector<uint32_t> newdeg(n);
  parallel_chunks(n, nt, [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t i = lo; i < hi; ++i) {
      uint32_t* b = tmp.data() + off[i];
      uint32_t* e = tmp.data() + off[i + 1];
      std::sort(b, e);
      newdeg[i] = (uint32_t)(std::unique(b, e) - b);
    }
  });
  uint32_t* row_ptr = (uint32_t*)std::malloc((n + 1) * sizeof(uint32_t));
  if (!row_ptr) return -2;
  uint64_t acc = 0;
  row_ptr[0] = 0;
  for (uint64_t i = 0; i < n; ++i) {
    acc += newdeg[i];
    if (acc > 0xFFFFFFFFull) {
      std::free(row_ptr);
      return -3;  // nnz must fit default_index_t (uint32), util/defaults.hpp:24
    }
    row_ptr[i + 1] = (uint32_t)acc;
  }
  uint32_t* col = (uint32_t*)std::malloc((acc ? acc : 1) * sizeof(uint32_t));
  if (!col) {
    std::free(row_ptr);
    return -2;
  }
  parallel_chunks(n, nt, [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t i = lo; i < hi; ++i)
      std::memcpy(col + row_ptr[i], tmp.data() + off[i], (size_t)newdeg[i] * sizeof(uint32_t));
  });
  out->n = n;
  out->nnz = acc;
  out->row_ptr = row_ptr;
  out->col = col;
  return 0;
}

}  // namespace

extern "C" {

int nwgen_rmat(int scale, double edge_factor, double a, double b, double c, uint64_t seed, int nthreads,
               nwgen_csr* out) {
  if (!out || scale < 1 || scale > 31 || edge_factor <= 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
  std::memset(out, 0, sizeof(*out));
  const int      nt = pick_threads(nthreads);
  const uint64_t n = 1ull << scale;
  RmatParams     p;
  p.scale = scale;
  p.m = (uint64_t)std::llround(edge_factor * (double)n);
  auto thr = [](double x) -> uint32_t {
    double v = std::floor(x * 4294967296.0);
    return v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
  };
  p.ta = thr(a);
  p.tab = thr(a + b);
  p.tabc = thr(a + b + c);
  p.seed = seed;

  // Pass 1: row counts (each non-loop sample adds u->v and v->u).
  std::vector<uint32_t> cnt(n, 0);
  parallel_chunks(p.m, nt, [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t e = lo; e < hi; ++e) {
      uint32_t u, v;
      rmat_sample(p, e, u, v);
      if (u == v) continue;
      std::atomic_ref<uint32_t>(cnt[u]).fetch_add(1, std::memory_order_relaxed);
      std::atomic_ref<uint32_t>(cnt[v]).fetch_add(1, std::memory_order_relaxed);
    }
  });
  std::vector<uint32_t> off(n + 1);
  uint64_t              total = 0;
  for (uint64_t i = 0; i < n; ++i) {
    off[i] = (uint32_t)total;
    total += cnt[i];
    if (total > 0xFFFFFFFFull) return -3;
  }
  off[n] = (uint32_t)total;
  // Pass 2: scatter (samples are regenerated from the hash, not stored).
  std::vector<uint32_t> cur(off.begin(), off.end() - 1);
  std::vector<uint32_t> tmp(total ? total : 1);
  parallel_chunks(p.m, nt, [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t e = lo; e < hi; ++e) {
      uint32_t u, v;
      rmat_sample(p, e, u, v);
      if (u == v) continue;
      uint32_t pu = std::atomic_ref<uint32_t>(cur[u]).fetch_add(1, std::memory_order_relaxed);
      tmp[pu] = v;
      uint32_t pv = std::atomic_ref<uint32_t>(cur[v]).fetch_add(1, std::memory_order_relaxed);
      tmp[pv] = u;
    }
  });
  std::vector<uint32_t>().swap(cur);
  std::vector<uint32_t>().swap(cnt);
  return finish_csr(n, off, tmp, nt, out);
}

int nwgen_grid(uint64_t n_target, nwgen_csr* out) {
  if (!out || n_target < 1) return -1;
  std::memset(out, 0, sizeof(*out));
  uint64_t side = (uint64_t)std::floor(std::sqrt((double)n_target));
  while ((side + 1) * (side + 1) <= n_target) ++side;
  while (side * side > n_target) --side;
  if (side < 1) side = 1;
  const uint64_t n = side * side;
  uint32_t*      row_ptr = (uint32_t*)std::malloc((n + 1) * sizeof(uint32_t));
  if (!row_ptr) return -2;
  uint64_t acc = 0;
  row_ptr[0] = 0;
  for (uint64_t v = 0; v < n; ++v) {
    uint64_t r = v / side, q = v % side;
    acc += (r > 0) + (q > 0) + (q + 1 < side) + (r + 1 < side);
    row_ptr[v + 1] = (uint32_t)acc;
  }
  uint32_t* col = (uint32_t*)std::malloc((acc ? acc : 1) * sizeof(uint32_t));
  if (!col) {
    std::free(row_ptr);
    return -2;
  }
  for (uint64_t v = 0; v < n; ++v) {
    uint64_t r = v / side, q = v % side, k = row_ptr[v];
    if (r > 0) col[k++] = (uint32_t)(v - side);
    if (q > 0) col[k++] = (uint32_t)(v - 1);
    if (q + 1 < side) col[k++] = (uint32_t)(v + 1);
    if (r + 1 < side) col[k++] = (uint32_t)(v + side);
  }
  out->n = n;
  out->nnz = acc;
  out->row_ptr = row_ptr;
  out->col = col;
  return 0;
}

int nwgen_from_edges(const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n, int symmetrize, int nthreads,
                     nwgen_csr* out) {
  if (!out || (m && (!src || !dst))) return -1;
  std::memset(out, 0, sizeof(*out));
  const int             nt = pick_threads(nthreads);
  std::vector<uint32_t> cnt(n, 0);
  for (uint64_t e = 0; e < m; ++e) {
    if (src[e] >= n || dst[e] >= n) return -1;
    if (symmetrize && src[e] == dst[e]) continue;
    // adjacency<1>: row = destination, entry = source.
    cnt[dst[e]]++;
    if (symmetrize) cnt[src[e]]++;
  }
  std::vector<uint32_t> off(n + 1);
  uint64_t              total = 0;
  for (uint64_t i = 0; i < n; ++i) {
    off[i] = (uint32_t)total;
    total += cnt[i];
  }
  off[n] = (uint32_t)total;
  std::vector<uint32_t> cur(off.begin(), off.end() - 1);
  std::vector<uint32_t> tmp(total ? total : 1);
  for (uint64_t e = 0; e < m; ++e) {
    if (symmetrize && src[e] == dst[e]) continue;
    tmp[cur[dst[e]]++] = src[e];
    if (symmetrize) tmp[cur[src[e]]++] = dst[e];
  }
  return finish_csr(n, off, tmp, nt, out);
}

void nwgen_free(nwgen_csr* g) {
  if (!g) return;
  std::free(g->row_ptr);
  std::free(g->col);
  g->row_ptr = nullptr;
  g->col = nullptr;
}

}  // extern "C"
