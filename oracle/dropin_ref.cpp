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
//   dropin_ref <file.mtx> [max_iters]   exit 0 when max-abs <= 1e-6 and L1 <= 1e-5
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "common.hpp"
#include "nwgraph/adjacency.hpp"
#include "nwgraph/experimental/algorithms/page_rank.hpp"
#include "nwgraph/io/mmio.hpp"
#include "nwgraph_gpu/page_rank.hpp"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::size_t iters = argc > 2 ? std::stoul(argv[2]) : 20;
  auto              el = nw::graph::read_mm<nw::graph::directedness::directed>(std::string(argv[1]));
  nw::graph::adjacency<1> graph(el);
  auto                    degrees = nw::graph::bench::build_degrees(graph);

  std::vector<float> cpu(graph.size()), gpu(graph.size());
  nw::graph::page_rank_v10(graph, degrees, cpu, 0.85f, 0.0f, iters, 1);
  nw::graph::gpu::page_rank(graph, degrees, gpu, 0.85f, 0.0f, iters, 1);

  double max_abs = 0, l1 = 0;
  for (std::size_t i = 0; i < cpu.size(); ++i) {
    double d = std::fabs((double)cpu[i] - (double)gpu[i]);
    max_abs = d > max_abs ? d : max_abs;
    l1 += d;
  }
  std::printf("dropin_ref n=%zu nnz=%zu sweeps=%zu max_abs=%.3e l1=%.3e\n", (std::size_t)graph.size(),
              (std::size_t)graph.num_edges(), iters, max_abs, l1);
  return (max_abs <= 1e-6 && l1 <= 1e-5) ? 0 : 1;
}
