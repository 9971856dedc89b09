// Drop-in test of include/nwgraph_gpu/page_rank.hpp: the same call a user of
// nw::graph::page_rank makes (include/nwgraph/algorithms/page_rank.hpp:89-91),
// with the namespace switched to nw::graph::gpu.
//
//   dropin_test <dir>  reads <dir>/row_ptr.u32, col.u32, deg.u32, runs
//   gpu::page_rank(graph, degrees, ranks, 0.85f, 0.0f, 20, 1) twice (the second
//   call reuses the resident CSR), writes <dir>/ranks.f32, and checks the error
//   path. Exit status 0 on success.
//
// The graph type is a stand-in with NWGraph's public CSR members
// (indices_, to_be_indexed_ as in include/nwgraph/containers/compressed.hpp:71-73),
// so this test needs no reference headers on the GPU host.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <tuple>
#include <vector>

#include "nwgraph_gpu/page_rank.hpp"

struct csr_graph {
  using vertex_id_type = std::uint32_t;
  std::vector<std::uint32_t>              indices_;
  std::tuple<std::vector<std::uint32_t>> to_be_indexed_;
  std::size_t                             size() const { return indices_.size() - 1; }
};

template <class T>
std::vector<T> read_all(const std::string& path) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) throw std::runtime_error("cannot open " + path);
  std::size_t bytes = (std::size_t)in.tellg();
  std::vector<T> v(bytes / sizeof(T));
  in.seekg(0);
  in.read(reinterpret_cast<char*>(v.data()), (std::streamsize)bytes);
  return v;
}

int main(int argc, char** argv) {
  if (argc != 2) {
    std::fprintf(stderr, "usage: %s <dir>\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  csr_graph g;
  g.indices_ = read_all<std::uint32_t>(dir + "/row_ptr.u32");
  std::get<0>(g.to_be_indexed_) = read_all<std::uint32_t>(dir + "/col.u32");
  std::vector<std::uint32_t> degrees = read_all<std::uint32_t>(dir + "/deg.u32");
  std::vector<float>         ranks(g.size());

  nw::graph::gpu::page_rank(g, degrees, ranks, 0.85f, 0.0f, 20, 1);
  std::vector<float> again(g.size());
  nw::graph::gpu::page_rank(g, degrees, again, 0.85f, 0.0f, 20, 1);  // resident CSR reused
  if (std::memcmp(ranks.data(), again.data(), ranks.size() * sizeof(float)) != 0) {
    std::fprintf(stderr, "second call differs\n");
    return 1;
  }
  bool threw = false;
  try {
    std::vector<std::uint32_t> short_deg(degrees.begin(), degrees.end() - 1);
    nw::graph::gpu::page_rank(g, short_deg, ranks, 0.85f, 0.0f, 20, 1);
  } catch (const nw::graph::gpu::gpu_error& e) {
    threw = e.status() == NWGPU_ERR_INVALID_ARG;
  }
  if (!threw) {
    std::fprintf(stderr, "size mismatch did not throw\n");
    return 1;
  }
  // page_rank_v10 is the same Jacobi solve; page_rank_v13 the residual push
  std::vector<float> v10(g.size()), v13(g.size());
  nw::graph::gpu::page_rank_v10(g, degrees, v10, 0.85f, 0.0f, 20, 1);
  if (std::memcmp(ranks.data(), v10.data(), ranks.size() * sizeof(float)) != 0) {
    std::fprintf(stderr, "page_rank_v10 differs from page_rank\n");
    return 1;
  }
  nw::graph::gpu::page_rank_v13(g, degrees, v13, 0.85f, 1e-4f, 100, 1);
  nw::graph::gpu::release(g);

  // Graphs rebuilt in a loop with the same row pointers (same degree sequence
  // of rows) but other column ids, usually at the same addresses: the cached
  // call must solve the current graph, exactly as a fresh upload does.
  nw::graph::gpu::set_cache_capacity(2);
  const std::size_t n = g.size();
  for (std::uint32_t round = 1; round <= 4; ++round) {
    csr_graph h;
    h.indices_ = g.indices_;
    std::get<0>(h.to_be_indexed_) = std::get<0>(g.to_be_indexed_);
    for (auto& c : std::get<0>(h.to_be_indexed_)) c = (std::uint32_t)((c + 7919ull * round) % n);  // other neighbours
    std::vector<std::uint32_t> hdeg(n, 0);
    for (auto c : std::get<0>(h.to_be_indexed_)) ++hdeg[c];
    std::vector<float> cached(n), fresh(n);
    nw::graph::gpu::page_rank(h, hdeg, cached, 0.85f, 0.0f, 20, 1);
    nw::graph::gpu::resident_graph direct(h);
    direct.run(hdeg.data(), fresh.data(), 0.85f, 0.0f, 20);
    if (std::memcmp(cached.data(), fresh.data(), n * sizeof(float)) != 0) {
      std::fprintf(stderr, "rebuilt graph %u: the cached call solved a stale graph\n", round);
      return 1;
    }
    if (std::memcmp(cached.data(), ranks.data(), n * sizeof(float)) == 0) {
      std::fprintf(stderr, "rebuilt graph %u: ranks equal the original graph's\n", round);
      return 1;
    }
  }
  nw::graph::gpu::release_all();
  std::ofstream out(dir + "/ranks.f32", std::ios::binary);
  out.write(reinterpret_cast<const char*>(ranks.data()), (std::streamsize)(ranks.size() * sizeof(float)));
  std::ofstream out13(dir + "/ranks_v13.f32", std::ios::binary);
  out13.write(reinterpret_cast<const char*>(v13.data()), (std::streamsize)(v13.size() * sizeof(float)));
  std::printf("dropin ok n=%zu\n", g.size());
  return 0;
}
