// Reference driver: test infrastructure, not part of the product.
//
// Compiles NWGraph's own PageRank headers (read in place from the reference
// tree, never copied) into oracle/_ref/libnwref.so behind a small C ABI so the
// tests and the CPU arm of bench.py can run the reference's code on exactly the
// CSR arrays the GPU engine uploads. Nothing here is linked into the product.
//
// Reference entry points wrapped:
//   nw::graph::page_rank            include/nwgraph/algorithms/page_rank.hpp:89-148 (v11, Gauss-Seidel)
//   nw::graph::page_rank_v10        include/nwgraph/experimental/algorithms/page_rank.hpp:377-432 (Jacobi)
//   nw::graph::page_rank_v1         include/nwgraph/experimental/algorithms/page_rank.hpp:82-119 (serial Jacobi)
//   nw::graph::page_rank_v13        include/nwgraph/experimental/algorithms/page_rank.hpp:552-625 (residual push)
//   nw::graph::bench::build_degrees bench/gapbs/common.hpp:110-121 (out-degree from adjacency<1>)
//   nw::graph::read_mm              include/nwgraph/io/mmio.hpp:171-217 + adjacency<1> fill (build.hpp:209-232)
//   read_mm<directed> edge list     include/nwgraph/io/mmio.hpp:86-103, 171-208
//   edge_list serialize/deserialize include/nwgraph/edge_list.hpp:237-280
//   edge clean-up and fill          remove_self_loops / lexical_sort_by / uniq (build.hpp:58-69, 394-410),
//                                   adjacency<idx>(el, sort_adjacency) (adjacency.hpp:115-129, build.hpp:209-321)
//
// Per-iteration times come from the reference's own pagerank::trace lines
// (page_rank.hpp:42-52, printed at :142), captured from std::cout.
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "nwgraph/adjacency.hpp"
#include "nwgraph/algorithms/page_rank.hpp"
#include "nwgraph/edge_list.hpp"
#include "nwgraph/experimental/algorithms/page_rank.hpp"
#include "nwgraph/io/mmio.hpp"
#include "common.hpp"  // bench/gapbs/common.hpp: build_degrees

namespace {

using Adj1 = nw::graph::adjacency<1>;

struct CoutCapture {
  std::ostringstream buf;
  std::streambuf*    old;
  CoutCapture() : old(std::cout.rdbuf(buf.rdbuf())) {}
  ~CoutCapture() { std::cout.rdbuf(old); }
};

// Parse "iter error time outgoing" trace rows; returns rows parsed.
int parse_trace(const std::string& text, double* errors, double* times, int max_rows) {
  std::istringstream in(text);
  std::string        line;
  int                rows = 0;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    long               it;
    double             err, t;
    if (!(ls >> it >> err >> t)) continue;  // header, life_timer lines
    if (rows < max_rows) {
      if (errors) errors[rows] = err;
      if (times) times[rows] = t;
    }
    ++rows;
  }
  return rows;
}

Adj1 make_adj(const uint32_t* row_ptr, const uint32_t* col, uint64_t n) {
  std::vector<uint32_t> indices(row_ptr, row_ptr + n + 1);
  std::vector<uint32_t> cols(col, col + row_ptr[n]);
  return Adj1(std::move(indices), std::move(cols));
}

struct Loaded {
  Adj1 adj;
};

}  // namespace

extern "C" {

// version: 11 = nw::graph::page_rank, 10 = page_rank_v10, 1 = page_rank_v1 (Real=float).
// Returns the number of sweeps run (trace rows), or -1 on a bad version.
int nwref_page_rank_f32(int version, const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const uint32_t* deg,
                        float* ranks, float damping, float threshold, uint64_t max_iters, int nthreads, double* errors,
                        double* iter_seconds, int max_rows) {
  Adj1                  g = make_adj(row_ptr, col, n);
  std::vector<uint32_t> degrees(deg, deg + n);
  std::vector<float>    pr(n);
  int                   rows = 0;
  {
    tbb::global_control gc(tbb::global_control::max_allowed_parallelism, nthreads > 0 ? nthreads : 1);
    CoutCapture         cap;
    if (version == 11) {
      nw::graph::page_rank(g, degrees, pr, damping, threshold, (size_t)max_iters, (size_t)nthreads);
    } else if (version == 10) {
      nw::graph::page_rank_v10(g, degrees, pr, damping, threshold, (size_t)max_iters, (size_t)nthreads);
    } else if (version == 1) {
      nw::graph::page_rank_v1(g, degrees, pr, damping, threshold, (size_t)max_iters);
    } else if (version == 13) {
      nw::graph::page_rank_v13(g, degrees, pr, damping, threshold, (size_t)max_iters, (size_t)nthreads);
    } else {
      return -1;
    }
    rows = parse_trace(cap.buf.str(), errors, iter_seconds, max_rows);
  }
  std::memcpy(ranks, pr.data(), n * sizeof(float));
  return rows;
}

// page_rank_v1 with Real=double, as test/page_rank_test.cpp:93 calls it.
int nwref_page_rank_v1_f64(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const uint32_t* deg, double* ranks,
                           double damping, double threshold, uint64_t max_iters) {
  Adj1                  g = make_adj(row_ptr, col, n);
  std::vector<uint32_t> degrees(deg, deg + n);
  std::vector<double>   pr(n);
  nw::graph::page_rank_v1(g, degrees, pr, damping, threshold, (size_t)max_iters);
  std::memcpy(ranks, pr.data(), n * sizeof(double));
  return 0;
}

// Out-degree per vertex via the benchmark's build_degrees on adjacency<1>.
int nwref_build_degrees(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, uint32_t* deg, int nthreads) {
  Adj1                g = make_adj(row_ptr, col, n);
  tbb::global_control gc(tbb::global_control::max_allowed_parallelism, nthreads > 0 ? nthreads : 1);
  CoutCapture         cap;
  auto                d = nw::graph::bench::build_degrees(g);
  std::memcpy(deg, d.data(), n * sizeof(uint32_t));
  return 0;
}

// Build adjacency<1> from a directed edge list with the reference's fill
// (build.hpp:209-232) and copy its CSR out. row_ptr has n+1 entries, col has m.
int nwref_fill_adj1(const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n, uint32_t* row_ptr, uint32_t* col) {
  nw::graph::edge_list<nw::graph::directedness::directed> el(n);
  el.open_for_push_back();
  for (uint64_t e = 0; e < m; ++e) el.push_back(src[e], dst[e]);
  el.close_for_push_back();
  CoutCapture cap;
  Adj1        g(el);
  if (g.size() != n || g.indices_.back() != m) return -1;
  std::memcpy(row_ptr, g.indices_.data(), (n + 1) * sizeof(uint32_t));
  std::memcpy(col, std::get<0>(g.to_be_indexed_).data(), m * sizeof(uint32_t));
  return 0;
}

// Edge list -> CSR with the reference's own clean-up steps and fill, rows
// sorted (sort_adjacency = true). flags: 1 by source (adjacency<0>), 2
// undirected edge list (fill_undirected), 4 remove_self_loops, 8 lexical sort
// + uniq. Returns -1 if col_cap is too small (nnz still set).
}  // extern "C"
template <nw::graph::directedness D, int idx>
int build_csr(const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n, int flags, uint32_t* row_ptr,
              uint32_t* col, uint64_t col_cap, uint64_t* nnz) {
  nw::graph::edge_list<D> el(n);
  el.open_for_push_back();
  for (uint64_t e = 0; e < m; ++e) el.push_back(src[e], dst[e]);
  el.close_for_push_back();
  CoutCapture cap;
  if (flags & 4) nw::graph::remove_self_loops(el);
  if (flags & 8) {
    nw::graph::lexical_sort_by<0>(el);
    nw::graph::uniq(el);
  }
  nw::graph::adjacency<idx> g(el, true);
  *nnz = g.indices_.back();
  if (g.indices_.size() != n + 1 || *nnz > col_cap) return -1;
  std::memcpy(row_ptr, g.indices_.data(), (n + 1) * sizeof(uint32_t));
  std::memcpy(col, std::get<0>(g.to_be_indexed_).data(), *nnz * sizeof(uint32_t));
  return 0;
}
extern "C" {

int nwref_build_csr(const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n, int flags, uint32_t* row_ptr,
                    uint32_t* col, uint64_t col_cap, uint64_t* nnz) {
  using nw::graph::directedness;
  const bool by_source = flags & 1, undirected = flags & 2;
  if (undirected)
    return by_source ? build_csr<directedness::undirected, 0>(src, dst, m, n, flags, row_ptr, col, col_cap, nnz)
                     : build_csr<directedness::undirected, 1>(src, dst, m, n, flags, row_ptr, col, col_cap, nnz);
  return by_source ? build_csr<directedness::directed, 0>(src, dst, m, n, flags, row_ptr, col, col_cap, nnz)
                   : build_csr<directedness::directed, 1>(src, dst, m, n, flags, row_ptr, col, col_cap, nnz);
}

// The edge list read_mm<directed> builds, in its order. Returns -1 if cap is
// too small (m still set).
int nwref_read_mm_edges(const char* path, uint32_t* src, uint32_t* dst, uint64_t cap, uint64_t* m, uint64_t* n) {
  CoutCapture cap_out;
  auto        el = nw::graph::read_mm<nw::graph::directedness::directed>(std::string(path));
  *m             = el.size();
  *n             = el.num_vertices()[0];
  if (*m > cap) return -1;
  uint64_t e = 0;
  for (auto&& [u, v] : el) {
    src[e] = u;
    dst[e] = v;
    ++e;
  }
  return 0;
}

// edge_list<directed>::serialize of the given edges.
int nwref_write_nw_edges(const char* path, const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n) {
  nw::graph::edge_list<nw::graph::directedness::directed> el(n);
  el.open_for_push_back();
  for (uint64_t e = 0; e < m; ++e) el.push_back(src[e], dst[e]);
  el.close_for_push_back();
  el.serialize(std::string(path));
  return 0;
}

// edge_list<directed>::deserialize, as load_graph does for "NW" files.
int nwref_read_nw_edges(const char* path, uint32_t* src, uint32_t* dst, uint64_t cap, uint64_t* m, uint64_t* n) {
  CoutCapture                                              cap_out;
  nw::graph::edge_list<nw::graph::directedness::directed> el(0);
  el.deserialize(std::string(path));
  *m = el.size();
  *n = el.num_vertices()[0];
  if (*m > cap) return -1;
  uint64_t e = 0;
  for (auto&& [u, v] : el) {
    src[e] = u;
    dst[e] = v;
    ++e;
  }
  return 0;
}

// What adjacency<1>::serialize (adjacency.hpp:180-184) writes for the CSR.
// That member does not compile in the reference (it is const and calls the
// non-const indexed_struct_of_arrays::serialize), so this makes its two calls
// directly on a non-const graph.
int nwref_write_adj1(const char* path, const uint32_t* row_ptr, const uint32_t* col, uint64_t n) {
  Adj1          g = make_adj(row_ptr, col, n);
  std::ofstream out(path, std::ofstream::binary);
  static_cast<const nw::graph::unipartite_graph_base&>(g).serialize(out);
  static_cast<nw::graph::indexed_struct_of_arrays<uint32_t, uint32_t>&>(g).serialize(out);
  return out.good() ? 0 : -1;
}

// A resident adjacency<1> + degrees, so timing runs do not re-copy the CSR.
struct Resident {
  Adj1                  adj;
  std::vector<uint32_t> degrees;
};
void* nwref_graph_create(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const uint32_t* deg) {
  return new Resident{make_adj(row_ptr, col, n), std::vector<uint32_t>(deg, deg + n)};
}
void nwref_graph_destroy(void* h) { delete static_cast<Resident*>(h); }
// Same as nwref_page_rank_f32 on a resident graph.
int nwref_graph_page_rank_f32(void* h, int version, float* ranks, float damping, float threshold, uint64_t max_iters,
                              int nthreads, double* errors, double* iter_seconds, int max_rows) {
  auto*              r = static_cast<Resident*>(h);
  const uint64_t     n = r->adj.size();
  std::vector<float> pr(n);
  int                rows = 0;
  {
    tbb::global_control gc(tbb::global_control::max_allowed_parallelism, nthreads > 0 ? nthreads : 1);
    CoutCapture         cap;
    if (version == 11)
      nw::graph::page_rank(r->adj, r->degrees, pr, damping, threshold, (size_t)max_iters, (size_t)nthreads);
    else if (version == 10)
      nw::graph::page_rank_v10(r->adj, r->degrees, pr, damping, threshold, (size_t)max_iters, (size_t)nthreads);
    else
      return -1;
    rows = parse_trace(cap.buf.str(), errors, iter_seconds, max_rows);
  }
  std::memcpy(ranks, pr.data(), n * sizeof(float));
  return rows;
}

// Read a MatrixMarket file with read_mm<directed> and build adjacency<1>.
// Returns an opaque handle; query sizes then copy the arrays out.
void* nwref_load_mm(const char* path, uint64_t* n, uint64_t* nnz) {
  CoutCapture cap;
  auto        el = nw::graph::read_mm<nw::graph::directedness::directed>(std::string(path));
  auto*       h  = new Loaded{Adj1(el)};
  *n             = h->adj.size();
  *nnz           = h->adj.indices_.back();
  return h;
}
void nwref_copy_csr(void* handle, uint32_t* row_ptr, uint32_t* col) {
  auto* h = static_cast<Loaded*>(handle);
  std::memcpy(row_ptr, h->adj.indices_.data(), h->adj.indices_.size() * sizeof(uint32_t));
  std::memcpy(col, std::get<0>(h->adj.to_be_indexed_).data(), std::get<0>(h->adj.to_be_indexed_).size() * sizeof(uint32_t));
}
void nwref_free(void* handle) { delete static_cast<Loaded*>(handle); }

}  // extern "C"
