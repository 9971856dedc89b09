/**
 * nwgraph_gpu/page_rank.hpp -- C++20 drop-in for nw::graph::page_rank on B200.
 *
 * Same call surface as the reference:
 *
 *   nw::graph::page_rank(graph, degrees, page_rank, damping_factor, threshold, max_iters, num_threads)
 *     include/nwgraph/algorithms/page_rank.hpp:89-91
 *   nw::graph::gpu::page_rank(graph, degrees, page_rank, damping_factor, threshold, max_iters, num_threads)
 *     this header
 *
 * so a caller switches by changing the namespace. Semantics are those of
 * page_rank_v10 (include/nwgraph/experimental/algorithms/page_rank.hpp:377-432):
 * Jacobi sweeps, FP32 scores, FP64 L1 error, stop after the first sweep whose
 * error is below threshold or after max_iters sweeps; page_rank is fully
 * overwritten; num_threads is unused, as in the reference.
 *
 * Differences a caller can observe:
 *  - Graph must expose NWGraph's public CSR members: contiguous uint32
 *    indices_ and std::get<0>(to_be_indexed_) (include/nwgraph/containers/compressed.hpp:71-73),
 *    which nw::graph::adjacency<idx> does; Real must be float.
 *  - Errors throw std::runtime_error (the reference has no error path); there
 *    is no CPU fallback.
 *  - The CSR is uploaded on the first call for a graph and kept resident in
 *    HBM, keyed by the graph's address, its array addresses, n, nnz, a hash
 *    of all of indices_ and a hash of up to 65,536 evenly spaced column ids
 *    (all of them in graphs of up to 65,536 entries). A graph rebuilt at the
 *    same addresses with other row pointers, or with other column ids at the
 *    sampled positions, is uploaded again. An in-place edit that touches only
 *    unsampled column ids is not seen: after mutating a graph in place, call
 *    nw::graph::gpu::release(graph) (or release_all()) before the next solve.
 *    At most cache_capacity() graphs (default 4) stay resident; the least
 *    recently used one is released first.
 *  - No per-iteration trace is printed (page_rank.hpp:109,142); use
 *    resident_graph::run for per-sweep errors and timing.
 *
 * Link with libnwgpu.so (C ABI in nwgpu.h).
 */
#ifndef NWGRAPH_GPU_PAGE_RANK_HPP
#define NWGRAPH_GPU_PAGE_RANK_HPP

#include <cstddef>
#include <cstdint>
#include <list>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../nwgpu.h"

namespace nw::graph::gpu {

/// A graph whose CSR members are contiguous uint32 arrays (adjacency<idx> and friends).
template <class Graph>
concept gpu_csr_graph = requires(const Graph& g) {
  { g.indices_.data() } -> std::convertible_to<const std::uint32_t*>;
  { std::get<0>(g.to_be_indexed_).data() } -> std::convertible_to<const std::uint32_t*>;
  { g.indices_.size() } -> std::convertible_to<std::size_t>;
  { std::get<0>(g.to_be_indexed_).size() } -> std::convertible_to<std::size_t>;
};

/// Thrown for every nonzero nwgpu status.
class gpu_error : public std::runtime_error {
public:
  gpu_error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int status() const noexcept { return status_; }

private:
  int status_;
};

namespace detail {
inline void check(int status, const char* call) {
  if (status == NWGPU_OK) return;
  char buf[512];
  nwgpu_last_error(buf, sizeof(buf));
  throw gpu_error(status, std::string(call) + ": " + buf);
}
}  // namespace detail

/// RAII owner of one resident CSR (nwgpu_graph handle).
class resident_graph {
public:
  resident_graph(const std::uint32_t* row_ptr, const std::uint32_t* col, std::uint64_t n, std::uint64_t nnz,
                 const float* weights = nullptr, std::uint32_t flags = 0) {
    detail::check(nwgpu_graph_create(row_ptr, col, weights, n, nnz, flags, &h_), "nwgpu_graph_create");
  }
  template <gpu_csr_graph Graph>
  explicit resident_graph(const Graph& g)
      : resident_graph(g.indices_.data(), std::get<0>(g.to_be_indexed_).data(), g.indices_.size() - 1,
                       std::get<0>(g.to_be_indexed_).size()) {}
  resident_graph(const resident_graph&) = delete;
  resident_graph& operator=(const resident_graph&) = delete;
  ~resident_graph() {
    if (h_) nwgpu_graph_destroy(h_);
  }
  nwgpu_graph* handle() const noexcept { return h_; }

  /// One solve; returns the engine's statistics.
  nwgpu_pr_stats run(const std::uint32_t* out_degree, float* ranks, float damping, float threshold,
                     std::uint64_t max_iters, const nwgpu_pr_options* opt = nullptr, double* errors = nullptr,
                     std::uint64_t errors_cap = 0) const {
    nwgpu_pr_stats st{};
    st.errors = errors;
    st.errors_cap = errors_cap;
    detail::check(nwgpu_pr_run(h_, out_degree, ranks, damping, threshold, max_iters, opt, &st), "nwgpu_pr_run");
    return st;
  }

  /// One residual-push solve (page_rank_v13's semantics); returns the engine's statistics.
  nwgpu_pr_stats run_residual(const std::uint32_t* out_degree, float* ranks, float damping, float threshold,
                              std::uint64_t max_iters, const nwgpu_pr_options* opt = nullptr) const {
    nwgpu_pr_stats st{};
    detail::check(nwgpu_pr_residual_run(h_, out_degree, ranks, damping, threshold, max_iters, opt, &st),
                  "nwgpu_pr_residual_run");
    return st;
  }

private:
  nwgpu_graph* h_ = nullptr;
};

namespace detail {
struct cache_key {
  const void*   graph;
  const void*   indices;
  const void*   cols;
  std::uint64_t n, nnz, row_hash, col_hash;
  bool          operator==(const cache_key& o) const {
    return std::tie(graph, indices, cols, n, nnz, row_hash, col_hash) ==
           std::tie(o.graph, o.indices, o.cols, o.n, o.nnz, o.row_hash, o.col_hash);
  }
};

// 64-bit multiply-xor mix of one word into the running hash.
inline std::uint64_t mix64(std::uint64_t h, std::uint64_t v) {
  h = (h ^ v) * 0x9E3779B97F4A7C15ull;
  return h ^ (h >> 29);
}

// All n + 1 row pointers, two per step (about 67 MB at n = 2^24, read once per call).
inline std::uint64_t row_hash(const std::uint32_t* rp, std::uint64_t n) {
  std::uint64_t       h = 0x243F6A8885A308D3ull ^ n;
  const std::uint64_t m = n + 1;
  std::uint64_t       i = 0;
  for (; i + 1 < m; i += 2) h = mix64(h, (std::uint64_t)rp[i] | ((std::uint64_t)rp[i + 1] << 32));
  if (i < m) h = mix64(h, rp[i]);
  return h;
}

// Up to 65,536 evenly spaced column ids plus the last one (every id when nnz <= 65,536).
inline std::uint64_t col_hash(const std::uint32_t* col, std::uint64_t nnz) {
  std::uint64_t h = 0x13198A2E03707344ull ^ nnz;
  if (!nnz) return h;
  const std::uint64_t step = (nnz + 65535) / 65536;
  for (std::uint64_t k = 0; k < nnz; k += step) h = mix64(h, ((std::uint64_t)k << 32) | col[k]);
  return mix64(h, col[nnz - 1]);
}

struct cache_state {
  std::mutex mu;
  std::size_t capacity = 4;
  // most recently used first
  std::list<std::pair<cache_key, std::shared_ptr<resident_graph>>> entries;
};

inline cache_state& cache() {
  static cache_state c;
  return c;
}

template <gpu_csr_graph Graph>
cache_key key_of(const Graph& g) {
  const std::uint64_t  n = g.indices_.size() - 1;
  const auto&          cols = std::get<0>(g.to_be_indexed_);
  return {&g, g.indices_.data(), cols.data(), n, cols.size(), row_hash(g.indices_.data(), n),
          col_hash(cols.data(), cols.size())};
}
}  // namespace detail

/// Number of graphs kept resident by the drop-in calls.
inline std::size_t cache_capacity() {
  std::lock_guard<std::mutex> lock(detail::cache().mu);
  return detail::cache().capacity;
}

/// Keep at most `capacity` graphs (>= 1) resident; releases the least recently used ones beyond it.
inline void set_cache_capacity(std::size_t capacity) {
  auto&                       c = detail::cache();
  std::lock_guard<std::mutex> lock(c.mu);
  c.capacity = capacity ? capacity : 1;
  while (c.entries.size() > c.capacity) c.entries.pop_back();
}

/// The resident copy of graph, uploading it on first use.
template <gpu_csr_graph Graph>
std::shared_ptr<resident_graph> resident(const Graph& graph) {
  if (graph.indices_.empty()) throw gpu_error(NWGPU_ERR_INVALID_ARG, "graph has no indices_ (not even indices_[0])");
  const auto                  key = detail::key_of(graph);
  auto&                       c = detail::cache();
  std::lock_guard<std::mutex> lock(c.mu);
  for (auto it = c.entries.begin(); it != c.entries.end(); ++it)
    if (it->first == key) {
      c.entries.splice(c.entries.begin(), c.entries, it);  // most recently used
      return c.entries.front().second;
    }
  // an entry for the same graph object or the same arrays is stale (mutated or rebuilt in place)
  c.entries.remove_if([&](const auto& e) {
    return e.first.graph == key.graph || e.first.indices == key.indices || e.first.cols == key.cols;
  });
  auto r = std::make_shared<resident_graph>(graph);
  c.entries.emplace_front(key, r);
  while (c.entries.size() > c.capacity) c.entries.pop_back();
  return r;
}

/// Free the resident copy of graph (after mutating it, or to return HBM).
template <class Graph>
void release(const Graph& graph) {
  auto&                       c = detail::cache();
  std::lock_guard<std::mutex> lock(c.mu);
  c.entries.remove_if([&](const auto& e) { return e.first.graph == (const void*)&graph; });
}

inline void release_all() {
  auto&                       c = detail::cache();
  std::lock_guard<std::mutex> lock(c.mu);
  c.entries.clear();
}

/**
 * Drop-in for nw::graph::page_rank (include/nwgraph/algorithms/page_rank.hpp:89-148).
 * degrees[j] is the out-degree of j (bench/gapbs/common.hpp:110-121); page_rank
 * must already hold graph.size() entries, as in the reference.
 */
template <gpu_csr_graph Graph, typename Real>
void page_rank(const Graph& graph, const std::vector<typename Graph::vertex_id_type>& degrees,
               std::vector<Real>& page_rank, Real damping_factor, Real threshold, std::size_t max_iters,
               std::size_t num_threads) {
  static_assert(std::is_same_v<Real, float>, "the B200 engine computes FP32 scores (Real = float)");
  static_assert(sizeof(typename Graph::vertex_id_type) == 4, "vertex ids must be 32-bit (default_vertex_id_type)");
  (void)num_threads;  // unused, as in the reference
  const std::size_t n = graph.indices_.size() - 1;
  if (degrees.size() != n) throw gpu_error(NWGPU_ERR_INVALID_ARG, "degrees.size() != graph.size()");
  if (page_rank.size() != n) throw gpu_error(NWGPU_ERR_INVALID_ARG, "page_rank.size() != graph.size()");
  auto g = resident(graph);
  g->run(reinterpret_cast<const std::uint32_t*>(degrees.data()), page_rank.data(), damping_factor, threshold,
         max_iters);
}

/**
 * Drop-in for nw::graph::page_rank_v10 (include/nwgraph/experimental/algorithms/
 * page_rank.hpp:377-432), the Jacobi solve the engine implements: the same
 * call as page_rank above.
 */
template <gpu_csr_graph Graph, typename Real>
void page_rank_v10(const Graph& graph, const std::vector<typename Graph::vertex_id_type>& degrees,
                   std::vector<Real>& page_rank, Real damping_factor, Real threshold, std::size_t max_iters,
                   std::size_t num_threads) {
  gpu::page_rank(graph, degrees, page_rank, damping_factor, threshold, max_iters, num_threads);
}

/**
 * Drop-in for nw::graph::page_rank_v13 (include/nwgraph/experimental/algorithms/
 * page_rank.hpp:552-625), the residual-push PageRank: ranks start at 0, every
 * residual at 1 - d, residuals above threshold are pushed each iteration;
 * the ranks are not normalised, as in the reference.
 */
template <gpu_csr_graph Graph, typename Real>
void page_rank_v13(const Graph& graph, const std::vector<typename Graph::vertex_id_type>& degrees,
                   std::vector<Real>& page_rank, Real damping_factor, Real threshold, std::size_t max_iters,
                   std::size_t num_threads) {
  static_assert(std::is_same_v<Real, float>, "the B200 engine computes FP32 scores (Real = float)");
  static_assert(sizeof(typename Graph::vertex_id_type) == 4, "vertex ids must be 32-bit (default_vertex_id_type)");
  (void)num_threads;
  const std::size_t n = graph.indices_.size() - 1;
  if (degrees.size() != n) throw gpu_error(NWGPU_ERR_INVALID_ARG, "degrees.size() != graph.size()");
  if (page_rank.size() != n) throw gpu_error(NWGPU_ERR_INVALID_ARG, "page_rank.size() != graph.size()");
  auto g = resident(graph);
  g->run_residual(reinterpret_cast<const std::uint32_t*>(degrees.data()), page_rank.data(), damping_factor,
                  threshold, max_iters);
}

}  // namespace nw::graph::gpu

#endif  // NWGRAPH_GPU_PAGE_RANK_HPP
