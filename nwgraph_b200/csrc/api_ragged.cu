// C ABI: ragged batches of independent graphs (nwgpu_batch_create,
// nwgpu_pr_ragged, nwgpu_batch_destroy; include/nwgpu.h).
//
// No counterpart in the reference, whose page_rank (page_rank.hpp:92-147)
// takes one graph: each graph of a batch gets exactly that solve (Jacobi,
// leak semantics, init 1/n_g, base (1-d)/n_g, FP64 L1 stopping test), but all
// graphs advance together in one sweep loop. Each graph keeps its local CSR;
// 64-bit per-graph bases locate its slices of the batch arrays, so a batch is
// limited only by device memory, not by 32-bit totals. The merge-path tiles of
// a graph never cross into the next graph, so every tile's L1 change belongs
// to one graph and the per-graph errors are sums of tile residuals in tile
// order. Graphs that stopped keep their ranks: each sweep walks a list of the
// running graphs' tiles, rebuilt after every sweep by the convergence kernel.
//
// Large graphs (at least 2^22 entries; NWGPU_RAGGED_SOLO_ENTRIES sets the
// bound, 0 keeps every graph in the batch) are solved alone by the
// single-graph engine (relabelled, degree-binned sweep), which sweeps them
// about twice as fast as the merge-path batch sweep; launching them one by one
// costs little next to their size, and they are spread round robin over a
// few streams (NWGPU_RAGGED_SOLO_STREAMS, default 4) so the short sweeps of
// the smaller ones overlap. In the batch they are empty members (no
// rows, no tiles); their handles read and write their slices of the batch's
// degree and rank arrays. Whether a graph is solved alone depends only on its
// own size, so a graph gets the same result in any batch.
//
// The graphs kept in the batch are solved together as one union graph by
// default (ragged_union.cu): their CSRs become diagonal blocks of one CSR,
// relabelled and swept by the degree-binned kernel in kModeRagged, each graph
// stopping at its own first sweep below the threshold and its rows then left
// alone. Every graph gets, sweep for sweep, a single-graph handle's ranks bit
// for bit. NWGPU_RAGGED_UNION=0 keeps the merge-path batch sweep; it is also
// used when the union's vertex or entry count does not fit 32-bit ids.
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "handle.h"
#include "ragged_union.h"

namespace nwgpu {

constexpr uint64_t kRaggedSoloEntries = 1ull << 22;
constexpr long     kRaggedSoloStreams = 4;  // NWGPU_RAGGED_SOLO_STREAMS

struct RaggedSolo {
  uint32_t     g = 0;  // the graph's index in the batch
  uint64_t     v0 = 0, n = 0, nnz = 0;
  nwgpu_graph* h = nullptr;
};

// A group of the graphs kept in a batch solved as one union graph: the
// union's handle and its per-row and per-part tables, and its solve loop.
struct RaggedUnion {
  nwgpu_graph*    h = nullptr;
  UnionParts      parts{};
  uint32_t*       ids = nullptr;
  uint64_t *      voff = nullptr, *eoff = nullptr;
  uint32_t*       coff = nullptr;       // per part: its first vertex chunk
  double*         chunk_part = nullptr;
  uint32_t*       row_graph = nullptr;  // per internal row: its batch graph
  double*         row_res = nullptr;    // per internal row: |dr| of the last sweep
  cudaGraph_t     cg = nullptr;
  cudaGraphExec_t exec = nullptr;
  float           damping = -1.f;       // the damping and threshold exec was built for
  double          threshold = -1.0;
  BinnedArgs      args{};               // this solve's sweep arguments
};

struct RaggedBatch {
  int          device = 0, sms = 0;
  std::vector<RaggedSolo> solos;  // graphs solved alone (empty members of the batch)
  // The solo graphs run on these streams, round robin, beside the batch's
  // sweep loop: the short sweeps of mid-size graphs overlap one another's
  // launch gaps and finishing kernels.
  std::vector<cudaStream_t> solo_streams;
  std::vector<cudaEvent_t>  solo_done;
  cudaStream_t stream = nullptr;
  uint32_t     num_graphs = 0;
  uint64_t     nv = 0, nnz = 0, nrp = 0;  // vertices, entries, row pointers of the batch
  uint32_t     num_tiles = 0;
  uint64_t     device_bytes = 0;
  std::vector<RaggedGraph> h_graphs;
  std::vector<uint32_t>    h_act;  // staging of the initial tile-list offsets
  RaggedGraph* graphs = nullptr;
  uint32_t *   row_ptr = nullptr, *col = nullptr;
  uint32_t *   tile_row = nullptr, *tile_nnz = nullptr;
  float *      rank = nullptr, *contrib[2] = {nullptr, nullptr};
  uint32_t*    deg = nullptr;
  float *      cpart = nullptr, *epart = nullptr, *base = nullptr;
  double *     res_tile = nullptr, *res_part = nullptr, *err_hist = nullptr;
  uint32_t     err_cap = 4096;
  RaggedState  rs{};
  PrState*     st = nullptr;
  PrState*     h_st = nullptr;
  unsigned int* h_abort = nullptr;
  unsigned int* d_abort = nullptr;
  int          sweep_grid = 1, finish_grid = 1, conv_grid = 1;
  cudaEvent_t  ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t  cg = nullptr;
  cudaGraphExec_t cg_exec = nullptr;
  float        cg_damping = -1.f;
  // The graphs kept in the batch, solved as unions by the degree-binned
  // sweep (none: the merge-path batch sweep instead).
  std::vector<RaggedUnion> unions;

  template <class T>
  cudaError_t alloc(T** p, uint64_t count) {
    const uint64_t bytes = (count + kPad) * sizeof(T);
    cudaError_t    e = pool_alloc((void**)p, bytes, stream);
    if (e == cudaSuccess) {
      device_bytes += bytes;
      e = cudaMemsetAsync(*p, 0, bytes, stream);
    }
    return e;
  }
  ~RaggedBatch() {
    for (cudaStream_t t : solo_streams) cudaStreamSynchronize(t);
    for (RaggedSolo& S : solos) delete S.h;  // not nwgpu_graph_destroy: that clears the caller's last error
    for (RaggedUnion& U : unions) {
      if (U.exec) cudaGraphExecDestroy(U.exec);
      if (U.cg) cudaGraphDestroy(U.cg);
      delete U.h;
      void* up[] = {U.ids, U.voff, U.eoff, U.coff, U.chunk_part, U.row_graph, U.row_res};
      for (void* p : up) pool_free(p, stream);
    }
    for (cudaEvent_t ev : solo_done) cudaEventDestroy(ev);
    for (cudaStream_t t : solo_streams) cudaStreamDestroy(t);
    if (stream) cudaStreamSynchronize(stream);
    if (cg_exec) cudaGraphExecDestroy(cg_exec);
    if (cg) cudaGraphDestroy(cg);
    void* ptrs[] = {graphs,   row_ptr,  col,      tile_row, tile_nnz, rank,     contrib[0], contrib[1],
                    deg,      cpart,    epart,    base,       res_tile, res_part, err_hist, rs.done,    rs.iters,
                    rs.err,   rs.conv,  rs.act_off, rs.act_list, st};
    for (void* p : ptrs) pool_free(p, stream);
    if (stream) cudaStreamSynchronize(stream);
    host_block_put(h_st);  // the stream is idle: no copy still targets them
    host_block_put(h_abort);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

SweepArgs ragged_args(const RaggedBatch* b, float damping) {
  SweepArgs a = {};
  a.row_ptr = b->row_ptr;
  a.col = b->col;
  a.tile_row = b->tile_row;
  a.tile_nnz = b->tile_nnz;
  a.num_tiles = b->num_tiles;
  a.tile_items = kRaggedTileItems;
  a.contrib0 = b->contrib[0];
  a.contrib1 = b->contrib[1];
  a.rank = b->rank;
  a.deg = b->deg;
  a.cpart = b->cpart;
  a.epart = b->epart;
  a.res_part = b->res_part;
  a.sweep_grid = (uint32_t)b->sweep_grid;
  a.st = b->st;
  a.err_hist = b->err_hist;
  a.err_cap = b->err_cap;
  a.abort_word = b->d_abort;
  a.damping = damping;
  // gathers allocate in L1 (every id counts as hot) unless NWGPU_RAGGED_GATHER=l2
  const char* gm = getenv("NWGPU_RAGGED_GATHER");
  a.hot_ids = (gm && !strcmp(gm, "l2")) ? 0u : 0xFFFFFFFFu;
  a.graphs = b->graphs;
  a.graph_base = b->base;
  a.res_tile = b->res_tile;
  a.act_off = b->rs.act_off;
  a.act_list = b->rs.act_list;
  a.num_graphs = b->num_graphs;
  return a;
}

int build_ragged_graph(RaggedBatch* b, const SweepArgs& proto) {
  if (b->cg_exec) {
    cudaGraphExecDestroy(b->cg_exec);
    b->cg_exec = nullptr;
  }
  if (b->cg) {
    cudaGraphDestroy(b->cg);
    b->cg = nullptr;
  }
  CK(cudaGraphCreate(&b->cg, 0), "cudaGraphCreate");
  cudaGraphNode_t arm;
  CK(add_pr_arm_node(b->cg, b->st, &arm), "cudaGraphAddKernelNode(arm)");
  cudaGraphConditionalHandle cond;
  CK(cudaGraphConditionalHandleCreate(&cond, b->cg, 1u, cudaGraphCondAssignDefault), "cudaGraphConditionalHandleCreate");
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wnode;
  CK(cudaGraphAddNode(&wnode, b->cg, &arm, 1, &cp), "cudaGraphAddNode(while)");
  SweepArgs a = proto;
  a.cond = cond;
  a.use_cond = 1;
  CK(add_ragged_nodes(cp.conditional.phGraph_out[0], a, b->sweep_grid, b->finish_grid, b->num_graphs, b->rs,
                      b->conv_grid),
     "cudaGraphAddKernelNode(ragged)");
  CK(cudaGraphInstantiate(&b->cg_exec, b->cg, 0), "cudaGraphInstantiate");
  b->cg_damping = proto.damping;
  return NWGPU_OK;
}

// The graphs kept in the batch (all but the solo graphs), in batch order, cut
// into unions of at most NWGPU_RAGGED_UNION_VERTICES vertices (default 2^23:
// a union's contributions, 32 MB, stay in L2 while its sweep gathers them):
// each one relabelled CSR over its graphs' vertices, graph after graph, swept
// by the degree-binned kernel in kModeRagged. Built unless
// NWGPU_RAGGED_UNION=0; a union whose binned plan cannot be built (an
// NWGPU_SWEEP naming a merge-path sweep) sends the batch back to its
// merge-path sweep.
int build_union(RaggedBatch* b, const std::vector<uint32_t>& ids, const std::vector<uint64_t>& voff,
                const std::vector<uint64_t>& eoff, int sms, RaggedUnion* U) {
  const uint64_t m = ids.size(), n = voff.back(), nnz = eoff.back();
  cudaStream_t   s = b->stream;
  CK(b->alloc(&U->ids, m), "cudaMalloc(union)");
  CK(b->alloc(&U->voff, m + 1), "cudaMalloc(union)");
  CK(b->alloc(&U->eoff, m + 1), "cudaMalloc(union)");
  CK(cudaMemcpyAsync(U->ids, ids.data(), m * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "upload union");
  CK(cudaMemcpyAsync(U->voff, voff.data(), (m + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s), "upload union");
  CK(cudaMemcpyAsync(U->eoff, eoff.data(), (m + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s), "upload union");
  std::vector<uint32_t> coff(m + 1, 0u);
  for (uint64_t j = 0; j < m; ++j)
    coff[j + 1] = coff[j] + (uint32_t)((voff[j + 1] - voff[j] + kUnionChunk - 1) / kUnionChunk);
  CK(b->alloc(&U->coff, m + 1), "cudaMalloc(union)");
  CK(b->alloc(&U->chunk_part, (uint64_t)coff[m] + 1), "cudaMalloc(union)");
  CK(cudaMemcpyAsync(U->coff, coff.data(), (m + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "upload union");
  const UnionParts p{U->ids, U->voff, U->eoff, U->coff, U->chunk_part, (uint32_t)m, coff[m], n, nnz};
  uint32_t *       rp = nullptr, *col = nullptr;
  CK(pool_alloc_n(&rp, n + 1 + kPad, s), "cudaMalloc(union CSR)");
  CK(pool_alloc_n(&col, nnz + kPad, s), "cudaMalloc(union CSR)");
  // The union's launch shape and hub tiers are tuned like a solo graph's
  // (bitwise-neutral); NWGPU_RAGGED_UNION_TUNE=0 keeps the defaults.
  const char*    tune_env = getenv("NWGPU_RAGGED_UNION_TUNE");
  const uint32_t tune = (tune_env && !strcmp(tune_env, "0")) ? 0u : kGraphTuneShapes;
  cudaError_t    e = launch_union_build(b->graphs, b->row_ptr, b->col, p, rp, col, sms, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  int rc = e == cudaSuccess ? nwgpu_graph_create(rp, col, nullptr, n, nnz,
                                                 NWGPU_GRAPH_DEVICE_PTRS | kGraphNoBlockedPlan | tune, &U->h)
                            : cuda_fail(e, "union CSR");
  pool_free(rp, s);
  pool_free(col, s);
  if (rc) return rc;
  if (!U->h->relabelled || !U->h->plan.ok) return NWGPU_OK;  // the caller drops the unions
  CK(b->alloc(&U->row_graph, n), "cudaMalloc(union rows)");
  CK(b->alloc(&U->row_res, n), "cudaMalloc(union rows)");
  CK(launch_union_row_graph(U->h->g.inv, p, U->row_graph, sms, s), "union rows");
  CK(cudaStreamSynchronize(s), "union");
  U->parts = p;
  return NWGPU_OK;
}

int build_unions(RaggedBatch* b, int sms) {
  const char* env = getenv("NWGPU_RAGGED_UNION");
  if (env && !strcmp(env, "0")) return NWGPU_OK;
  const char*    vmax_env = getenv("NWGPU_RAGGED_UNION_VERTICES");
  const long long vm = vmax_env && *vmax_env ? strtoll(vmax_env, nullptr, 10) : (1ll << 23);
  const uint64_t vmax = vm > 1 ? (uint64_t)vm : 2u;
  std::vector<char> solo(b->num_graphs, 0);
  for (const RaggedSolo& S : b->solos) solo[S.g] = 1;
  // groups of consecutive graphs kept in the batch; a last group of fewer than two vertices joins the one before
  std::vector<std::vector<uint32_t>> groups;
  uint64_t                           gv = 0, ge = 0;
  for (uint32_t g = 0; g < b->num_graphs; ++g) {
    if (solo[g]) continue;
    const RaggedGraph& R = b->h_graphs[g];
    if (groups.empty() || gv + R.n > vmax || ge + R.nnz > kMaxEntries) {
      groups.emplace_back();
      gv = ge = 0;
    }
    groups.back().push_back(g);
    gv += R.n;
    ge += R.nnz;
  }
  if (groups.size() >= 2 && gv < 2) {
    std::vector<uint32_t> last = std::move(groups.back());
    groups.pop_back();
    groups.back().insert(groups.back().end(), last.begin(), last.end());
  }
  bool ok = !groups.empty();
  for (const std::vector<uint32_t>& gr : groups) {
    std::vector<uint64_t> voff(1, 0), eoff(1, 0);
    for (uint32_t g : gr) {
      voff.push_back(voff.back() + b->h_graphs[g].n);
      eoff.push_back(eoff.back() + b->h_graphs[g].nnz);
    }
    if (voff.back() < 2 || voff.back() >= 0xFFFFFFF0ull || eoff.back() > kMaxEntries) {
      ok = false;  // a graph too large, or too few vertices: the merge-path sweep
      break;
    }
    b->unions.emplace_back();
    const int rc = build_union(b, gr, voff, eoff, sms, &b->unions.back());
    if (rc) return rc;
    if (!b->unions.back().h->plan.ok) {
      ok = false;
      break;
    }
  }
  if (!ok) {  // the merge-path sweep for every graph kept in the batch
    for (RaggedUnion& U : b->unions) {
      delete U.h;
      void* up[] = {U.ids, U.voff, U.eoff, U.coff, U.chunk_part, U.row_graph, U.row_res};
      for (void* p : up) pool_free(p, b->stream);
    }
    b->unions.clear();
    CK(cudaStreamSynchronize(b->stream), "union");
  }
  return NWGPU_OK;
}

}  // namespace
}  // namespace nwgpu

struct nwgpu_batch : nwgpu::RaggedBatch {};

using namespace nwgpu;

extern "C" {

int nwgpu_batch_create(uint64_t num_graphs, const uint64_t* vertex_offsets, const uint64_t* entry_offsets,
                       const uint32_t* row_ptr, const uint32_t* col, uint32_t flags, nwgpu_batch** out) {
  clear_error();
  if (!out) return fail(NWGPU_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (num_graphs == 0 || num_graphs >= 0x7FFFFFFFull)
    return fail(NWGPU_ERR_INVALID_ARG, "num_graphs = %llu outside [1, 2^31)", (unsigned long long)num_graphs);
  if (!vertex_offsets || !entry_offsets) return fail(NWGPU_ERR_INVALID_ARG, "vertex_offsets / entry_offsets is NULL");
  if (vertex_offsets[0] != 0 || entry_offsets[0] != 0)
    return fail(NWGPU_ERR_INVALID_ARG, "vertex_offsets[0] and entry_offsets[0] must be 0");
  // Per-graph slices and tiles, checked on the host (the offsets are host arrays).
  // Graphs solved alone are empty members: one zero row pointer, no entries.
  const char*              solo_env = getenv("NWGPU_RAGGED_SOLO_ENTRIES");
  const uint64_t           solo_min = solo_env && *solo_env ? strtoull(solo_env, nullptr, 10) : kRaggedSoloEntries;
  std::vector<RaggedGraph> hg(num_graphs);
  std::vector<RaggedSolo>  solos;
  uint64_t                 tiles = 0, pc = 0, ec = 0;  // compacted row pointers and entries
  for (uint64_t g = 0; g < num_graphs; ++g) {
    if (vertex_offsets[g + 1] < vertex_offsets[g] || entry_offsets[g + 1] < entry_offsets[g])
      return fail(NWGPU_ERR_INVALID_ARG, "offsets decrease at graph %llu", (unsigned long long)g);
    const uint64_t n = vertex_offsets[g + 1] - vertex_offsets[g], m = entry_offsets[g + 1] - entry_offsets[g];
    if (n >= 0xFFFFFFF0ull || m >= 0xFFFFFFF0ull)
      return fail(NWGPU_ERR_INVALID_ARG, "graph %llu: n = %llu, nnz = %llu do not fit uint32 local ids",
                  (unsigned long long)g, (unsigned long long)n, (unsigned long long)m);
    RaggedGraph& R = hg[g];
    const bool   solo = solo_min && m >= solo_min;
    R.v0 = vertex_offsets[g];
    R.e0 = ec;
    R.p0 = pc;
    R.n = solo ? 0u : (uint32_t)n;
    R.nnz = solo ? 0u : (uint32_t)m;
    R.tile0 = (uint32_t)tiles;
    R.tiles = (uint32_t)((R.n + R.nnz + kRaggedTileItems - 1) / kRaggedTileItems);
    tiles += R.tiles;
    pc += R.n + 1ull;
    ec += R.nnz;
    if (solo) {
      RaggedSolo S;
      S.g = (uint32_t)g;
      S.v0 = vertex_offsets[g];
      S.n = n;
      S.nnz = m;
      solos.push_back(S);
    }
    if (tiles + num_graphs >= 0xFFFFFFF0ull) return fail(NWGPU_ERR_INVALID_ARG, "batch has too many tiles");
  }
  const uint64_t nv = vertex_offsets[num_graphs], nnz = entry_offsets[num_graphs], nrp = pc;
  if (!row_ptr) return fail(NWGPU_ERR_INVALID_ARG, "row_ptr is NULL");
  if (nnz && !col) return fail(NWGPU_ERR_INVALID_ARG, "col is NULL with entries");
  int dev, sms;
  int rc = check_device(&dev, &sms);
  if (rc) return rc;

  nwgpu_batch* b = new (std::nothrow) nwgpu_batch();
  if (!b) return fail(NWGPU_ERR_OUT_OF_MEMORY, "host allocation failed");
  auto bail = [&](int code) {
    delete b;
    return code;
  };
  b->device = dev;
  b->sms = sms;
  b->num_graphs = (uint32_t)num_graphs;
  b->nv = nv;
  b->nnz = nnz;
  b->nrp = nrp;
  b->num_tiles = (uint32_t)tiles;
  b->h_graphs = std::move(hg);
  b->solos = std::move(solos);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamCreate"));
  const cudaMemcpyKind kind = (flags & NWGPU_GRAPH_DEVICE_PTRS) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const uint64_t       T = tiles, G = num_graphs;
#define BK(call, what)                                    \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return bail(cuda_fail(_e, what)); \
  } while (0)
  BK(b->alloc(&b->graphs, G), "cudaMalloc(graphs)");
  BK(b->alloc(&b->row_ptr, nrp), "cudaMalloc(row_ptr)");
  BK(b->alloc(&b->col, ec), "cudaMalloc(col)");
  BK(cudaMemcpyAsync(b->graphs, b->h_graphs.data(), G * sizeof(RaggedGraph), cudaMemcpyHostToDevice, b->stream),
     "upload graphs");
  // Runs of graphs kept in the batch are contiguous in the input and in the
  // compacted arrays: one copy of row pointers and one of entries per run.
  // A solo graph's row pointer stays the zero the allocation wrote.
  for (uint64_t g0 = 0; g0 < G;) {
    if (b->h_graphs[g0].n == 0 && b->h_graphs[g0].nnz == 0) {
      ++g0;
      continue;
    }
    uint64_t g1 = g0 + 1;
    while (g1 < G && !(b->h_graphs[g1].n == 0 && b->h_graphs[g1].nnz == 0 && solo_min &&
                       entry_offsets[g1 + 1] - entry_offsets[g1] >= solo_min))
      ++g1;
    const uint64_t p_in = vertex_offsets[g0] + g0, p_end = vertex_offsets[g1] + g1;  // row pointers of [g0, g1)
    BK(cudaMemcpyAsync(b->row_ptr + b->h_graphs[g0].p0, row_ptr + p_in, (p_end - p_in) * sizeof(uint32_t), kind,
                       b->stream),
       "upload row_ptr");
    const uint64_t e_in = entry_offsets[g0], e_end = entry_offsets[g1];
    if (e_end > e_in)
      BK(cudaMemcpyAsync(b->col + b->h_graphs[g0].e0, col + e_in, (e_end - e_in) * sizeof(uint32_t), kind, b->stream),
         "upload col");
    g0 = g1;
  }
  // Validate on the device before any kernel indexes with these arrays.
  unsigned int* d_err = nullptr;
  unsigned int  h_err = 0;
  BK(pool_alloc_n(&d_err, 1, b->stream), "cudaMalloc(err)");
  e = cudaMemsetAsync(d_err, 0, sizeof(unsigned int), b->stream);
  if (e == cudaSuccess) e = validate_ragged(b->graphs, b->num_graphs, b->row_ptr, b->col, nrp, ec, d_err, sms, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  pool_free(d_err, b->stream);
  if (e != cudaSuccess) return bail(cuda_fail(e, "validate"));
  if (h_err)
    return bail(fail(NWGPU_ERR_INVALID_GRAPH, "invalid batch CSR:%s%s%s",
                     (h_err & 1u) ? " a graph's row pointers do not start at 0 or end at its nnz;" : "",
                     (h_err & 2u) ? " row pointers decrease;" : "", (h_err & 4u) ? " column id >= the graph's n;" : ""));
  // Tiles and solve buffers.
  BK(b->alloc(&b->tile_row, T + G), "cudaMalloc(tile_row)");
  BK(b->alloc(&b->tile_nnz, T + G), "cudaMalloc(tile_nnz)");
  BK(fill_ragged_tiling(b->graphs, b->num_graphs, b->row_ptr, b->num_tiles, b->tile_row, b->tile_nnz, sms, b->stream),
     "ragged tiling");
  BK(b->alloc(&b->rank, nv), "cudaMalloc(rank)");
  BK(b->alloc(&b->contrib[0], nv), "cudaMalloc(contrib)");
  BK(b->alloc(&b->contrib[1], nv), "cudaMalloc(contrib)");
  BK(b->alloc(&b->deg, nv), "cudaMalloc(deg)");
  BK(b->alloc(&b->cpart, T + 1), "cudaMalloc(cpart)");
  BK(b->alloc(&b->epart, T + 1), "cudaMalloc(epart)");
  BK(b->alloc(&b->res_tile, T + 1), "cudaMalloc(res_tile)");
  BK(b->alloc(&b->base, G), "cudaMalloc(base)");
  BK(b->alloc(&b->rs.done, G), "cudaMalloc(graph state)");
  BK(b->alloc(&b->rs.iters, G), "cudaMalloc(graph state)");
  BK(b->alloc(&b->rs.err, G), "cudaMalloc(graph state)");
  BK(b->alloc(&b->rs.conv, G), "cudaMalloc(graph state)");
  BK(b->alloc(&b->rs.act_off, G + 1), "cudaMalloc(graph state)");
  BK(b->alloc(&b->rs.act_list, T), "cudaMalloc(tile list)");
  BK(b->alloc(&b->err_hist, b->err_cap), "cudaMalloc(err_hist)");
  BK(b->alloc(&b->st, 1), "cudaMalloc(state)");
  // Grids: 4 resident 256-thread CTAs per SM for the sweep; the converge
  // kernel has one warp per graph up to 16 CTAs per SM.
  const uint64_t want = (uint64_t)sms * 4;
  b->sweep_grid = (int)(T == 0 ? 1 : (want < T ? want : T));
  b->finish_grid = (int)(T == 0 ? 1 : (T + 255) / 256);
  const uint64_t cg = (G + 7) / 8, cap = (uint64_t)sms * 16;
  b->conv_grid = (int)(cg < cap ? cg : cap);
  BK(b->alloc(&b->res_part, (uint64_t)b->conv_grid), "cudaMalloc(res_part)");
  BK(host_block_get((void**)&b->h_st), "cudaHostAlloc(state)");
  BK(host_block_get((void**)&b->h_abort), "cudaHostAlloc(abort)");
  BK(cudaHostGetDevicePointer((void**)&b->d_abort, b->h_abort, 0), "cudaHostGetDevicePointer(abort)");
  BK(cudaEventCreate(&b->ev0), "cudaEventCreate");
  BK(cudaEventCreate(&b->ev1), "cudaEventCreate");
  BK(cudaStreamSynchronize(b->stream), "batch create");
#undef BK
  // The unions of the graphs kept in the batch (no merge-path sweep then).
  if ((rc = build_unions(b, sms))) return bail(rc);
  // The graphs solved alone: single-graph handles over the caller's slices.
  // Solo graphs and unions run on a few streams beside each other.
  if (!b->solos.empty() || !b->unions.empty()) {
    const char*  ns_env = getenv("NWGPU_RAGGED_SOLO_STREAMS");
    long         ns = ns_env && *ns_env ? strtol(ns_env, nullptr, 10) : kRaggedSoloStreams;
    const size_t jobs = b->solos.size() + b->unions.size();
    if (ns < 1) ns = 1;
    if ((size_t)ns > jobs) ns = (long)jobs;
    for (long i = 0; i < ns; ++i) {
      cudaStream_t t = nullptr;
      cudaEvent_t  ev = nullptr;
      if ((e = cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking)) != cudaSuccess) return bail(cuda_fail(e, "solo stream"));
      b->solo_streams.push_back(t);
      if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return bail(cuda_fail(e, "solo stream"));
      b->solo_done.push_back(ev);
    }
  }
  // A solo graph's launch shape and hub tiers are tuned (cached per graph
  // signature, so graphs alike are timed once): bitwise-neutral, and a small
  // graph can stage fewer hub contributions per sweep than a large one.
  // NWGPU_RAGGED_SOLO_TUNE=0 keeps the defaults.
  const char*    solo_tune_env = getenv("NWGPU_RAGGED_SOLO_TUNE");
  const uint32_t solo_tune = (solo_tune_env && !strcmp(solo_tune_env, "0")) ? 0u : kGraphTuneShapes;
  for (RaggedSolo& S : b->solos) {
    rc = nwgpu_graph_create(row_ptr + (vertex_offsets[S.g] + S.g), col + entry_offsets[S.g], nullptr, S.n, S.nnz,
                            (flags & NWGPU_GRAPH_DEVICE_PTRS) | solo_tune, &S.h);
    if (rc) {
      char msg[400];
      nwgpu_last_error(msg, sizeof(msg));
      return bail(fail(rc, "graph %u: %s", S.g, msg));
    }
  }
  *out = b;
  return NWGPU_OK;
}

int nwgpu_batch_destroy(nwgpu_batch* b) {
  clear_error();
  delete b;
  return NWGPU_OK;
}

int nwgpu_pr_ragged(nwgpu_batch* b, const uint32_t* out_degree, float* ranks, float damping, float threshold,
                    uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_batch_stats* stats) {
  clear_error();
  if (!b) return fail(NWGPU_ERR_INVALID_ARG, "batch is NULL");
  if (b->nv && (!out_degree || !ranks)) return fail(NWGPU_ERR_INVALID_ARG, "out_degree / ranks is NULL");
  if (!(damping >= 0.0f && damping <= 1.0f)) return fail(NWGPU_ERR_INVALID_ARG, "damping %g outside [0, 1]", (double)damping);
  const nwgpu_pr_options opt = read_options(options);
  if (opt.mode != NWGPU_MODE_PARITY) return fail(NWGPU_ERR_UNSUPPORTED, "mode %u is not supported", opt.mode);
  if (opt.launch > NWGPU_LAUNCH_STREAM) return fail(NWGPU_ERR_INVALID_ARG, "launch %u unknown", opt.launch);
  cudaStream_t   s = opt.stream ? (cudaStream_t)opt.stream : b->stream;
  const uint64_t nv = b->nv, G = b->num_graphs;
  const bool     dptr = opt.device_ptrs != 0;
  *(volatile unsigned int*)b->h_abort = 0u;
  if (nv)
    CK(cudaMemcpyAsync(b->deg, out_degree, nv * sizeof(uint32_t), dptr ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       s),
       "copy out_degree");
  PrState h = {};
  h.max_iters = max_iters;
  h.chunk_end = kGraphChunk;
  h.threshold = (double)threshold;
  h.done = (max_iters == 0) ? 1u : 0u;
  const bool      use_unions = !b->unions.empty();
  const SweepArgs a = ragged_args(b, damping);
  if (!use_unions) {
    *b->h_st = h;
    CK(cudaMemcpyAsync(b->st, b->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
    // every graph starts running: the tile list is all tiles
    b->h_act.resize(G + 1);
    for (uint64_t g = 0; g <= G; ++g) b->h_act[g] = g < G ? b->h_graphs[g].tile0 : b->num_tiles;
    CK(cudaMemcpyAsync(b->rs.act_off, b->h_act.data(), (G + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s),
       "copy tile list");
    CK(launch_ragged_init(a, b->rs, b->num_graphs, nv, damping, h.done, b->sms, s), "ragged init");
    CK(launch_ragged_list(a, b->rs, b->sms, s), "ragged tile list");
  }
  CK(cudaEventRecord(b->ev0, s), "cudaEventRecord");
  // The graphs solved alone run on their own stream, after the degree copy,
  // while the batch's sweep loop runs: each writes only its slice of the rank
  // array, which no batch kernel touches. They start once the first round of
  // the batch loop is queued.
  std::vector<nwgpu_pr_stats> solo_st(b->solos.size());
  bool                        solos_run = b->solos.empty();
  auto                        run_solos = [&]() -> int {
    solos_run = true;
    const size_t nstreams = b->solo_streams.size();
    auto         stream_of = [&](size_t i) { return b->solo_streams[i % nstreams]; };
    for (cudaStream_t t : b->solo_streams) CK(cudaStreamWaitEvent(t, b->ev0, 0), "solo stream");
    auto graph_fail = [&](int rc, uint32_t g) {
      char msg[400];
      nwgpu_last_error(msg, sizeof(msg));
      return fail(rc, "graph %u: %s", g, msg);
    };
    // With the CUDA-graph loop, every solo solve is queued back to back and the
    // stream is synchronized once; the rest (if any) take the full call.
    std::vector<char> queued(b->solos.size(), 0);
    if (opt.launch == NWGPU_LAUNCH_GRAPH) {
      for (size_t i = 0; i < b->solos.size(); ++i) {
        const RaggedSolo& S = b->solos[i];
        bool              q = false;
        int rc = pr_solve_queue(S.h, b->deg + S.v0, b->rank + S.v0, damping, threshold, max_iters, stream_of(i), &q);
        if (rc) return graph_fail(rc, S.g);
        queued[i] = q ? 1 : 0;
      }
      for (cudaStream_t t : b->solo_streams) CK(cudaStreamSynchronize(t), "solo graphs");
      for (size_t i = 0; i < b->solos.size(); ++i) {
        if (!queued[i]) continue;
        const RaggedSolo& S = b->solos[i];
        solo_st[i] = nwgpu_pr_stats{};
        int rc = pr_solve_finish(S.h, b->rank + S.v0, damping, threshold, max_iters, stream_of(i), &solo_st[i]);
        if (rc) return graph_fail(rc, S.g);
      }
    }
    for (size_t i = 0; i < b->solos.size(); ++i) {
      if (queued[i]) continue;
      const RaggedSolo& S = b->solos[i];
      nwgpu_pr_options  so = {};
      so.size = sizeof(so);
      so.mode = NWGPU_MODE_PARITY;
      so.launch = opt.launch;
      so.device_ptrs = 1;
      so.stream = (void*)stream_of(i);
      solo_st[i] = nwgpu_pr_stats{};
      int rc = nwgpu_pr_run(S.h, b->deg + S.v0, b->rank + S.v0, damping, threshold, max_iters, &so, &solo_st[i]);
      if (rc) return graph_fail(rc, S.g);
    }
    for (size_t i = 0; i < nstreams; ++i) {
      CK(cudaEventRecord(b->solo_done[i], b->solo_streams[i]), "solo stream");
      CK(cudaStreamWaitEvent(s, b->solo_done[i], 0), "solo stream");
    }
    return NWGPU_OK;
  };
  auto drained = [&](int rc) {  // nothing of this call left in flight on an error
    cudaStreamSynchronize(s);
    for (cudaStream_t t : b->solo_streams) cudaStreamSynchronize(t);
    return rc;
  };
  PrState fin{};
  if (use_unions) {
    // Each union's whole solve goes on a stream of its own (round robin with the solo graphs'): the per-graph
    // tables start, then the CUDA-graph loop (or, in stream mode, a few sweeps at a time until it stops).
    const size_t ns = b->solo_streams.size();
    auto         ustream = [&](size_t j) { return b->solo_streams[(b->solos.size() + j) % ns]; };
    for (cudaStream_t t : b->solo_streams) CK(cudaStreamWaitEvent(t, b->ev0, 0), "union stream");
    for (size_t j = 0; j < b->unions.size(); ++j) {
      RaggedUnion& U = b->unions[j];
      nwgpu_graph* uh = U.h;
      cudaStream_t t = ustream(j);
      int          rc = ensure_solve_buffers(uh);
      if (rc) return drained(rc);
      *uh->h_st = h;
      CK(cudaMemcpyAsync(uh->st, uh->h_st, sizeof(PrState), cudaMemcpyHostToDevice, t), "copy state");
      CK(launch_union_start(b->graphs, U.parts, uh->g.inv, U.row_graph, b->deg, damping, h.done, b->base, b->rs,
                            uh->deg, uh->rank, uh->contrib[0], b->sms, t),
         "union start");
      SweepArgs sw = make_sweep_args(uh, damping, 0.f, kTeleportUniform, 0u);
      sw.abort_word = b->d_abort;
      sw.graph_base = b->base;
      sw.row_graph = U.row_graph;
      sw.graph_done = b->rs.done;
      sw.row_res = U.row_res;
      U.args = make_binned_args(uh, uh->plan, sw, kModeRagged);
      if (opt.launch == NWGPU_LAUNCH_GRAPH &&
          (!U.exec || U.damping != damping || U.threshold != (double)threshold)) {
        if (U.exec) cudaGraphExecDestroy(U.exec);
        if (U.cg) cudaGraphDestroy(U.cg);
        U.exec = nullptr;
        U.cg = nullptr;
        CK(cudaGraphCreate(&U.cg, 0), "cudaGraphCreate");
        CK(build_union_graph(U.cg, U.args, binned_grid(uh, uh->plan, kModeRagged), uh->plan.finish_grid, U.parts,
                             uh->g.perm, U.row_res, b->rs, uh->st, (double)threshold, b->d_abort, b->sms, &U.exec),
           "union graph");
        U.damping = damping;
        U.threshold = (double)threshold;
      }
    }
    // Queue every running union's next round, then read their states back: one CUDA-graph launch (up to
    // kGraphChunk sweeps) or, in stream mode, up to 8 sweeps.
    auto queue_round = [&]() -> int {
      for (size_t j = 0; j < b->unions.size(); ++j) {
        RaggedUnion& U = b->unions[j];
        nwgpu_graph* uh = U.h;
        cudaStream_t t = ustream(j);
        if (uh->h_st->done) continue;
        if (opt.launch == NWGPU_LAUNCH_GRAPH) {
          CK(cudaGraphLaunch(U.exec, t), "cudaGraphLaunch");
        } else {
          const uint64_t left = max_iters - uh->h_st->iter, k = left < 8 ? left : 8;
          for (uint64_t i = 0; i < k; ++i) {
            CK(launch_binned_sweep(U.args, true, kModeRagged, binned_grid(uh, uh->plan, kModeRagged),
                                   uh->plan.finish_grid, t),
               "union sweep");
            CK(launch_union_converge(U.parts, uh->g.perm, U.row_res, b->rs, uh->st, (double)threshold, b->d_abort,
                                     b->sms, t),
               "union convergence");
          }
        }
        CK(cudaMemcpyAsync(uh->h_st, uh->st, sizeof(PrState), cudaMemcpyDeviceToHost, t), "copy state");
      }
      return NWGPU_OK;
    };
    const uint64_t max_rounds = (opt.launch == NWGPU_LAUNCH_GRAPH ? max_iters / kGraphChunk : max_iters / 8) + 2;
    for (uint64_t round = 0;; ++round) {
      if (round == max_rounds)
        return drained(fail(NWGPU_ERR_CUDA, "union sweep loop did not finish after %llu rounds", (unsigned long long)round));
      int rc = queue_round();
      if (rc) return drained(rc);
      if (!solos_run) {
        if ((rc = run_solos())) return drained(rc);
      }
      for (cudaStream_t t : b->solo_streams) CK(cudaStreamSynchronize(t), "union sweep loop");
      bool all = true;
      for (RaggedUnion& U : b->unions) all = all && (U.h->h_st->done || U.h->h_st->iter >= max_iters);
      if (all) break;
    }
    for (size_t j = 0; j < b->unions.size(); ++j) {
      RaggedUnion&   U = b->unions[j];
      const PrState& f = *U.h->h_st;
      fin.iter = f.iter > fin.iter ? f.iter : fin.iter;
      fin.fault |= f.fault;
      fin.aborted |= f.aborted;
      CK(launch_union_output(b->graphs, U.parts, U.h->g.perm, U.h->rank, b->rank, b->sms, ustream(j)), "union ranks");
    }
    for (size_t i = 0; i < b->solo_streams.size(); ++i) {
      CK(cudaEventRecord(b->solo_done[i], b->solo_streams[i]), "union stream");
      CK(cudaStreamWaitEvent(s, b->solo_done[i], 0), "union stream");
    }
  } else {
    if (opt.launch == NWGPU_LAUNCH_GRAPH) {
      if (!b->cg_exec || b->cg_damping != damping) {
        int rc = build_ragged_graph(b, a);
        if (rc) return rc;
      }
      cudaGraphExec_t exec = b->cg_exec;
      const uint64_t max_launches = max_iters / kGraphChunk + 2;
      for (uint64_t launches = 0; !b->h_st->done; ++launches) {
        if (launches == max_launches)
          return drained(
              fail(NWGPU_ERR_CUDA, "sweep loop did not finish after %llu graph launches", (unsigned long long)launches));
        CK(cudaGraphLaunch(exec, s), "cudaGraphLaunch");
        CK(cudaMemcpyAsync(b->h_st, b->st, sizeof(PrState), cudaMemcpyDeviceToHost, s), "copy state");
        if (!solos_run) {
          int rc = run_solos();
          if (rc) return drained(rc);
        }
        CK(cudaStreamSynchronize(s), "sweep loop");
      }
    } else {
      uint64_t launched = 0;
      while (!b->h_st->done && launched < max_iters) {
        const uint64_t batch = (max_iters - launched) < kGraphChunk ? (max_iters - launched) : kGraphChunk;
        for (uint64_t k = 0; k < batch; ++k)
          CK(launch_ragged_sweep(a, b->sweep_grid, b->finish_grid, b->num_graphs, b->rs, b->conv_grid, s), "ragged sweep");
        launched += batch;
        CK(cudaMemcpyAsync(b->h_st, b->st, sizeof(PrState), cudaMemcpyDeviceToHost, s), "copy state");
        if (!solos_run) {
          int rc = run_solos();
          if (rc) return drained(rc);
        }
        CK(cudaStreamSynchronize(s), "sweep loop");
      }
    }
    if (!solos_run) {  // the batch loop ran no round (max_iters 0)
      int rc = run_solos();
      if (rc) return drained(rc);
    }
    fin = *b->h_st;
  }

  if (fin.fault) return drained(fail(NWGPU_ERR_CUDA, "a bounded device wait gave up (fault word %u)", fin.fault));
  CK(cudaEventRecord(b->ev1, s), "cudaEventRecord");  // after the solo graphs too (s waits for them)
  if (nv)
    CK(cudaMemcpyAsync(ranks, b->rank, nv * sizeof(float), dptr ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s),
       "copy ranks");
  std::vector<uint32_t> iters(G);
  std::vector<uint32_t> conv(G);
  CK(cudaMemcpyAsync(iters.data(), b->rs.iters, G * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy graph state");
  CK(cudaMemcpyAsync(conv.data(), b->rs.conv, G * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy graph state");
  if (stats && stats->graph_errors)
    CK(cudaMemcpyAsync(stats->graph_errors, b->rs.err, G * sizeof(double), cudaMemcpyDeviceToHost, s), "copy graph errors");
  CK(cudaStreamSynchronize(s), "copy ranks");
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    double   swept = 0.0;
    uint64_t nconv = 0, sweeps = fin.iter;
    for (size_t i = 0; i < b->solos.size(); ++i) {  // the solo graphs' own counts
      const RaggedSolo& S = b->solos[i];
      iters[S.g] = (uint32_t)solo_st[i].iterations;
      conv[S.g] = solo_st[i].converged ? 1u : 0u;
      swept += (double)S.nnz * (double)solo_st[i].iterations;
      if (stats->graph_errors) stats->graph_errors[S.g] = solo_st[i].final_error;
      if (solo_st[i].iterations > sweeps) sweeps = solo_st[i].iterations;
    }
    for (uint64_t g = 0; g < G; ++g) {
      swept += (double)b->h_graphs[g].nnz * (double)iters[g];  // 0 entries for the solo graphs here
      nconv += conv[g] ? 1u : 0u;
      if (stats->graph_iterations) stats->graph_iterations[g] = iters[g];
      if (stats->graph_converged) stats->graph_converged[g] = conv[g] ? 1 : 0;
    }
    stats->sweeps = sweeps;
    stats->converged_graphs = nconv;
    stats->device_ms = ms;
    stats->entries_swept = swept;
    stats->gteps = ms > 0 ? swept / (ms * 1e6) : 0.0;
  }
  if (fin.aborted) return fail(NWGPU_ERR_ABORTED, "solve aborted after %llu sweeps", (unsigned long long)fin.iter);
  return NWGPU_OK;
}

}  // extern "C"
