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
 *    HBM, keyed by the graph's address, its array addresses, n, nnz and a
 *    sampled hash of indices_. After mutating a graph in place, call
 *    nw::graph::gpu::release(graph) (or release_all()) before the next solve.
 *  - No per-iteration trace is printed (page_rank.hpp:109,142); use
 *    resident_graph::run for per-sweep errors and timing.
 *
 * Link with libnwgpu.so (C ABI in nwgpu.h).
 */
#ifndef NWGRAPH_GPU_PAGE_RANK_HPP
#define NWGRAPH_GPU_PAGE_RANK_HPP

#include <cstddef>
#include <cstdint>
#include <map>
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
  std::uint64_t n, nnz, sample_hash;
  bool          operator<(const cache_key& o) const {
    return std::tie(graph, indices, cols, n, nnz, sample_hash) <
           std::tie(o.graph, o.indices, o.cols, o.n, o.nnz, o.sample_hash);
  }
};

// FNV-1a over up to 4096 evenly spaced row pointers plus the last one.
inline std::uint64_t sample_hash(const std::uint32_t* rp, std::uint64_t n) {
  std::uint64_t       h = 1469598103934665603ull;
  const std::uint64_t step = n / 4096 + 1;
  auto                mix = [&](std::uint64_t v) {
    h ^= v;
    h *= 1099511628211ull;
  };
  for (std::uint64_t i = 0; i <= n; i += step) mix(rp[i]);
  mix(rp[n]);
  return h;
}

inline std::mutex& cache_mutex() {
  static std::mutex m;
  return m;
}
inline std::map<cache_key, std::shared_ptr<resident_graph>>& cache() {
  static std::map<cache_key, std::shared_ptr<resident_graph>> c;
  return c;
}

template <gpu_csr_graph Graph>
cache_key key_of(const Graph& g) {
  const std::uint64_t n = g.indices_.size() - 1;
  return {&g, g.indices_.data(), std::get<0>(g.to_be_indexed_).data(), n, std::get<0>(g.to_be_indexed_).size(),
          sample_hash(g.indices_.data(), n)};
}
}  // namespace detail

/// The resident copy of graph, uploading it on first use.
template <gpu_csr_graph Graph>
std::shared_ptr<resident_graph> resident(const Graph& graph) {
  if (graph.indices_.empty()) throw gpu_error(NWGPU_ERR_INVALID_ARG, "graph has no indices_ (not even indices_[0])");
  auto                        key = detail::key_of(graph);
  std::lock_guard<std::mutex> lock(detail::cache_mutex());
  auto&                       c = detail::cache();
  auto                        it = c.find(key);
  if (it != c.end()) return it->second;
  // drop stale entries of the same graph object (mutated in place)
  for (auto i = c.begin(); i != c.end();) i = (i->first.graph == key.graph) ? c.erase(i) : std::next(i);
  auto r = std::make_shared<resident_graph>(graph);
  c.emplace(key, r);
  return r;
}

/// Free the resident copy of graph (after mutating it, or to return HBM).
template <class Graph>
void release(const Graph& graph) {
  std::lock_guard<std::mutex> lock(detail::cache_mutex());
  auto&                       c = detail::cache();
  for (auto i = c.begin(); i != c.end();) i = (i->first.graph == (const void*)&graph) ? c.erase(i) : std::next(i);
}

inline void release_all() {
  std::lock_guard<std::mutex> lock(detail::cache_mutex());
  detail::cache().clear();
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
