// Drop-in check against the reference's own graph type (test infrastructure).
//
// Builds NWGraph's nw::graph::adjacency<1> (include/nwgraph/adjacency.hpp:194-195)
// from a MatrixMarket file with read_mm (include/nwgraph/io/mmio.hpp:171-217),
// computes degrees with the benchmark's build_degrees (bench/gapbs/common.hpp:110-121),
// then runs the reference's page_rank_v10 and the B200 engine's
// nw::graph::gpu::page_rank with the identical argument list and compares.
// Compiled by oracle/Makefile (target dropin) where the reference tree exists;
// the binary links libnwgpu.so and runs on a GPU host.
//
//   dropin_ref <file.mtx> [max_iters] [o2]
//
// exit 0 when max-abs <= 1e-6 and L1 <= 1e-5 after max_iters sweeps. With
// "o2" it also checks the drop-in against the production solver,
// nw::graph::page_rank (v11, include/nwgraph/algorithms/page_rank.hpp:89-148,
// Gauss-Seidel on all host threads), on the same adjacency<1>:
//   * converged: both at 100 sweeps, threshold 0: max-abs <= 1e-7 (the
//     reference's serial FP32 sums over hub rows drift by several 1e-9);
//   * the top-100 vertices in the same order, apart from ties within 1e-6;
//   * the threshold-1e-4 runs (at most 1000 sweeps): the sweep counts of v11
//     (from its own trace lines, :142), of page_rank_v10 and of the engine are
//     printed; the engine's must equal page_rank_v10's.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "common.hpp"
#include "nwgraph/adjacency.hpp"
#include "nwgraph/algorithms/page_rank.hpp"
#include "nwgraph/experimental/algorithms/page_rank.hpp"
#include "nwgraph/io/mmio.hpp"
#include "nwgraph_gpu/page_rank.hpp"

namespace {

// Sweeps a reference solve ran: its trace rows "iter error time ..." (page_rank.hpp:142).
template <class F>
int traced_sweeps(F&& solve) {
  std::ostringstream buf;
  std::streambuf*    old = std::cout.rdbuf(buf.rdbuf());
  solve();
  std::cout.rdbuf(old);
  std::istringstream in(buf.str());
  std::string        line;
  int                rows = 0;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    long               it;
    double             err, t;
    if (ls >> it >> err >> t) ++rows;
  }
  return rows;
}

void compare(const std::vector<float>& a, const std::vector<float>& b, double& max_abs, double& l1) {
  max_abs = 0;
  l1 = 0;
  for (std::size_t i = 0; i < a.size(); ++i) {
    double d = std::fabs((double)a[i] - (double)b[i]);
    max_abs = d > max_abs ? d : max_abs;
    l1 += d;
  }
}

std::vector<std::size_t> top(const std::vector<float>& r, std::size_t k) {
  std::vector<std::size_t> idx(r.size());
  std::iota(idx.begin(), idx.end(), 0);
  k = std::min(k, r.size());
  std::stable_sort(idx.begin(), idx.end(), [&](std::size_t x, std::size_t y) { return r[x] > r[y]; });
  idx.resize(k);
  return idx;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::size_t iters = argc > 2 ? std::stoul(argv[2]) : 20;
  const bool        o2 = argc > 3 && std::string(argv[3]) == "o2";
  auto              el = nw::graph::read_mm<nw::graph::directedness::directed>(std::string(argv[1]));
  nw::graph::adjacency<1> graph(el);
  auto                    degrees = nw::graph::bench::build_degrees(graph);

  std::vector<float> cpu(graph.size()), gpu(graph.size());
  nw::graph::page_rank_v10(graph, degrees, cpu, 0.85f, 0.0f, iters, 1);
  nw::graph::gpu::page_rank(graph, degrees, gpu, 0.85f, 0.0f, iters, 1);

  double max_abs = 0, l1 = 0;
  compare(cpu, gpu, max_abs, l1);
  std::printf("dropin_ref n=%zu nnz=%zu sweeps=%zu max_abs=%.3e l1=%.3e\n", (std::size_t)graph.size(),
              (std::size_t)graph.num_edges(), iters, max_abs, l1);
  bool ok = max_abs <= 1e-6 && l1 <= 1e-5;
  if (!o2) return ok ? 0 : 1;

  // (i) converged agreement with the production solver
  std::vector<float> v11(graph.size()), eng(graph.size());
  traced_sweeps([&] { nw::graph::page_rank(graph, degrees, v11, 0.85f, 0.0f, 100, 1); });
  nw::graph::gpu::page_rank(graph, degrees, eng, 0.85f, 0.0f, 100, 1);
  double c_max = 0, c_l1 = 0;
  compare(v11, eng, c_max, c_l1);
  // (ii) top-100 order, ties within 1e-6 of v11's value at that position allowed
  const auto t11 = top(v11, 100), te = top(eng, 100);
  int        order_breaks = 0;
  for (std::size_t i = 0; i < t11.size(); ++i)
    if (t11[i] != te[i] && std::fabs((double)v11[t11[i]] - (double)v11[te[i]]) > 1e-6) ++order_breaks;
  // (iii) threshold-1e-4 runs: sweep counts
  std::vector<float> tmp(graph.size());
  const int          it11 = traced_sweeps([&] { nw::graph::page_rank(graph, degrees, tmp, 0.85f, 1e-4f, 1000, 1); });
  const int it10 = traced_sweeps([&] { nw::graph::page_rank_v10(graph, degrees, tmp, 0.85f, 1e-4f, 1000, 1); });
  auto      res = nw::graph::gpu::resident(graph);
  const auto st = res->run(reinterpret_cast<const std::uint32_t*>(degrees.data()), tmp.data(), 0.85f, 1e-4f, 1000);
  std::printf("dropin_ref_o2 converged_max_abs=%.3e converged_l1=%.3e top100_order_breaks=%d "
              "thr_sweeps_v11=%d thr_sweeps_v10=%d thr_sweeps_engine=%llu\n",
              c_max, c_l1, order_breaks, it11, it10, (unsigned long long)st.iterations);
  ok = ok && c_max <= 1e-7 && order_breaks == 0 && (unsigned long long)it10 == (unsigned long long)st.iterations &&
       st.converged && it11 > 0;
  nw::graph::gpu::release_all();
  return ok ? 0 : 1;
}
