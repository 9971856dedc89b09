// C ABI: weighted PageRank and the implicit adjoint of its fixed point
// (nwgpu_wpr_run, nwgpu_pr_vjp in include/nwgpu.h). No counterpart in the
// reference, whose page_rank is unweighted (page_rank.hpp:129-133); the
// update, the stopping rule and the FP64 residual are its own, with weighted,
// out-normalised contributions and a teleport vector. The adjoint solves
//   l = c + d P^T l   (P_ij = w(j->i) / s_j)
// with the same degree-binned sweep over the out-row CSR, so no forward
// iterates are stored; the gradients are one pass over the entries
// (pr_weighted.cu).
//
// The adjoint is solved by restarted GMRES (Saad & Schultz 1986) with
// classical Gram-Schmidt applied twice, an FP32 Krylov basis and FP64
// reductions; one operator application A v = v - d P^T v is one adjoint
// sweep. The plain fixed-point iteration converges at rate d on every mode
// of P^T with eigenvalue 1 (one per connected component) and -1 (one per
// bipartite component); GMRES removes each such cluster with one polynomial
// factor and needs about as many sweeps as the forward solve.
// NWGPU_VJP_SOLVER=jacobi selects the fixed-point iteration instead.
#include <chrono>

#include "handle.h"

using namespace nwgpu;

namespace nwgpu {

void WprBuffers::release(cudaStream_t s) {
  void* ptrs[] = {t.row_ptr, t.col, t.w, t.fwd, t.s, t.erow, vbase, vaux, r_int, stage, stage2, res, gw, basis, w, vneg,
                  part, dout, f, q};
  for (void* p : ptrs) pool_free(p, s);
  tplan.release(s);
  *this = WprBuffers();
}

int ensure_wpr(nwgpu_graph* g) {
  WprBuffers& b = g->wpr;
  if (b.ready) return NWGPU_OK;
  const uint64_t n = g->n, nnz = g->nnz;
  CK(build_transpose(g->g.row_ptr, g->g.col, g->g.w, n, nnz, g->sms, &b.t, g->stream), "out-row CSR");
  g->device_bytes += (4 * (nnz + kPad) + 2 * (n + kPad) + 1) * sizeof(uint32_t);
  int rc = build_bin_plan(g, b.t.row_ptr, n, true, &b.tplan);
  if (rc) return rc;
  CK(dalloc(g, &b.vbase, n), "cudaMalloc(wpr base)");
  CK(dalloc(g, &b.vaux, n), "cudaMalloc(wpr aux)");
  CK(dalloc(g, &b.r_int, n), "cudaMalloc(wpr ranks)");
  CK(dalloc(g, &b.stage, n), "cudaMalloc(wpr staging)");
  CK(dalloc(g, &b.stage2, n), "cudaMalloc(wpr staging)");
  CK(dalloc(g, &b.f, n), "cudaMalloc(dL/dw factors)");
  CK(dalloc(g, &b.q, n), "cudaMalloc(dL/dw offsets)");
  const uint64_t parts = (uint64_t)binned_sweep_grid(g->sms, true) + (uint64_t)b.tplan.finish_grid;
  CK(dalloc(g, &b.res, parts), "cudaMalloc(wpr residuals)");
  CK(cudaStreamSynchronize(g->stream), "wpr buffers");
  b.ready = true;
  return NWGPU_OK;
}

namespace {

// Arguments shared by both calls; returns the stream or sets an error.
int check_common(nwgpu_graph* g, const void* out, float damping, const nwgpu_pr_options& opt) {
  if (!g) return fail(NWGPU_ERR_INVALID_ARG, "graph is NULL");
  if (g->n && !out) return fail(NWGPU_ERR_INVALID_ARG, "output is NULL");
  if (!(damping >= 0.0f && damping <= 1.0f)) return fail(NWGPU_ERR_INVALID_ARG, "damping %g outside [0, 1]", (double)damping);
  if (opt.mode != NWGPU_MODE_PARITY) return fail(NWGPU_ERR_UNSUPPORTED, "mode %u is not supported", opt.mode);
  if (opt.launch > NWGPU_LAUNCH_STREAM) return fail(NWGPU_ERR_INVALID_ARG, "launch %u unknown", opt.launch);
  if (!g->g.w) return fail(NWGPU_ERR_UNSUPPORTED, "the graph has no edge weights (pass them to nwgpu_graph_create)");
  if (!g->relabelled || !g->plan.ok)
    return fail(NWGPU_ERR_UNSUPPORTED, "weighted PageRank runs on the degree-binned sweep: create the graph relabelled");
  return NWGPU_OK;
}

int start_state(nwgpu_graph* g, uint64_t max_iters, float threshold, cudaStream_t s) {
  PrState h = {};
  h.max_iters = max_iters;
  h.chunk_end = kGraphChunk;
  h.threshold = (double)threshold;
  h.done = (max_iters == 0) ? 1u : 0u;
  *g->h_st = h;
  *(volatile unsigned int*)g->h_abort = 0u;
  CK(cudaMemcpyAsync(g->st, g->h_st, sizeof(PrState), cudaMemcpyHostToDevice, s), "copy state");
  return NWGPU_OK;
}

void init_stats(nwgpu_pr_stats* stats, double bytes) {
  if (!stats) return;
  double*  eb = stats->errors;
  uint64_t ec = stats->errors_cap;
  memset(stats, 0, sizeof(*stats));
  stats->errors = eb;
  stats->errors_cap = ec;
  stats->bytes_per_iter = bytes;
}

int finish_stats(nwgpu_graph* g, const PrState& fin, float ms, nwgpu_pr_stats* stats, cudaStream_t s) {
  if (!stats) return NWGPU_OK;
  stats->iterations = fin.iter;
  stats->final_error = fin.last_error;
  stats->converged = (int32_t)fin.converged;
  stats->device_ms = ms;
  stats->ms_per_iter = fin.iter ? ms / (double)fin.iter : 0.0;
  stats->gteps = ms > 0 ? (double)g->nnz * (double)fin.iter / (ms * 1e6) : 0.0;
  if (stats->errors && stats->errors_cap) {
    uint64_t m = fin.iter < stats->errors_cap ? fin.iter : stats->errors_cap;
    if (m > g->err_cap) m = g->err_cap;
    if (m) {
      CK(cudaMemcpyAsync(stats->errors, g->err_hist, m * sizeof(double), cudaMemcpyDeviceToHost, s), "copy errors");
      CK(cudaStreamSynchronize(s), "copy errors");
    }
  }
  return NWGPU_OK;
}

// An n-vector argument on the device: the caller's pointer, or a copy of the
// host vector in `stage`.
int device_vector(const float* v, float* stage, uint64_t n, bool device_ptrs, cudaStream_t s, const float** out) {
  if (!v || device_ptrs) {
    *out = v;
    return NWGPU_OK;
  }
  CK(cudaMemcpyAsync(stage, v, n * sizeof(float), cudaMemcpyHostToDevice, s), "copy vector");
  *out = stage;
  return NWGPU_OK;
}

constexpr int kGmresRestart = 30;
static_assert(kGmresRestart <= kGmresMaxBasis, "more basis vectors than the update kernel takes");

int ensure_gmres(nwgpu_graph* g) {
  WprBuffers& b = g->wpr;
  if (b.basis) return NWGPU_OK;
  const uint64_t n = g->n;
  b.ld = (n + kPad + 3) & ~3ull;
  const VecGrid vg = vec_grid(n, g->sms);
  CK(dalloc(g, &b.basis, b.ld * (kGmresRestart + 1)), "cudaMalloc(Krylov basis)");
  CK(dalloc(g, &b.w, n), "cudaMalloc(gmres work)");
  CK(dalloc(g, &b.vneg, n), "cudaMalloc(gmres -d/s)");
  CK(dalloc(g, &b.part, (uint64_t)vg.blocks * (kGmresRestart + 1)), "cudaMalloc(gmres partials)");
  CK(dalloc(g, &b.dout, (uint64_t)kGmresRestart + 2), "cudaMalloc(gmres dots)");
  return NWGPU_OK;
}

// out = A v = v - d P^T v: one adjoint sweep over the out-row CSR with
// vbase = v and vaux = -d/s, reading v as the contribution vector.
int apply_adjoint_op(nwgpu_graph* g, const SweepArgs& proto, const float* v, float* out, cudaStream_t s) {
  WprBuffers& b = g->wpr;
  SweepArgs   a = proto;
  a.vbase = v;
  a.vaux = b.vneg;
  a.contrib0 = const_cast<float*>(v);
  a.contrib1 = out;
  a.rank = out;
  CK(launch_op_state(g->st, s), "operator state");
  const BinnedArgs ba = make_binned_args(g, b.tplan, a, kModeAdjoint);
  CK(launch_binned_sweep(ba, b.tplan.hot, kModeAdjoint, binned_grid(g, b.tplan, kModeAdjoint), b.tplan.finish_grid, s),
     "adjoint operator");
  return NWGPU_OK;
}

int read_doubles(const double* d, double* h, int count, cudaStream_t s) {
  CK(cudaMemcpyAsync(h, d, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, s), "copy reduction");
  CK(cudaStreamSynchronize(s), "reduction");
  return NWGPU_OK;
}

// Restarted GMRES for A x = c (c = vbase, internal order), x in/out (x0 on
// entry). Stops when the L1 norm of the true residual c - A x, evaluated in
// FP64 at the start of each cycle, is below thr, or after max_ops operator
// applications. *ops = operator applications, *res_l1 = last true residual.
int gmres_adjoint(nwgpu_graph* g, const SweepArgs& proto, const float* c, float* x, double thr, uint64_t max_ops,
                  cudaStream_t s, uint64_t* ops, double* res_l1, bool* converged) {
  WprBuffers&    b = g->wpr;
  const uint64_t n = g->n;
  const VecGrid  vg = vec_grid(n, g->sms);
  const int      m = kGmresRestart;
  auto           V = [&](int i) { return b.basis + (uint64_t)i * b.ld; };
  double         H[kGmresRestart + 1][kGmresRestart], cs[kGmresRestart], sn[kGmresRestart], gv[kGmresRestart + 1];
  double         h[kGmresRestart + 2];
  float          coef[kGmresMaxBasis];
  *ops = 0;
  *converged = false;
  int rc;
  for (;;) {
    // r = c - A x, its L1 norm (the fixed-point iteration's L1 change) and 2-norm
    if ((rc = apply_adjoint_op(g, proto, x, b.w, s))) return rc;
    ++*ops;
    CK(launch_vec_axpby(1.f, c, 0.f, V(0), n, vg, b.part, nullptr, s), "residual");
    CK(launch_vec_axpby(-1.f, b.w, 1.f, V(0), n, vg, b.part, b.dout, s), "residual");
    CK(launch_vec_dots(V(0), b.ld, 1, V(0), n, vg, b.part, b.dout + 1, s), "residual norm");
    if ((rc = read_doubles(b.dout, h, 2, s))) return rc;
    *res_l1 = h[0];
    if (h[0] < thr) {
      *converged = true;
      return NWGPU_OK;
    }
    if (*ops >= max_ops) return NWGPU_OK;
    const double beta = sqrt(h[1]);
    if (!(beta > 0.0)) return NWGPU_OK;
    const double l1_per_l2 = h[0] / beta;  // how the L1 norm scales with the 2-norm this cycle
    CK(launch_vec_axpby((float)(1.0 / beta), V(0), 0.f, V(0), n, vg, b.part, nullptr, s), "normalise");
    for (int i = 0; i <= m; ++i) gv[i] = 0.0;
    gv[0] = beta;
    int k = 0;  // basis vectors used this cycle
    for (int j = 0; j < m; ++j) {
      if ((rc = apply_adjoint_op(g, proto, V(j), b.w, s))) return rc;
      ++*ops;
      // classical Gram-Schmidt, twice: h1 = V^T w; w' = w - V h1 with h2 = V^T w'
      // and |w'|^2 in the same pass; the new vector (w' - V h2) / |w' - V h2|,
      // whose norm is sqrt(|w'|^2 - |h2|^2)
      double hj[kGmresRestart + 1] = {0.0};
      CK(launch_vec_dots(V(0), b.ld, j + 1, b.w, n, vg, b.part, b.dout, s), "Gram-Schmidt dots");
      if ((rc = read_doubles(b.dout, h, j + 1, s))) return rc;
      for (int i = 0; i <= j; ++i) {
        hj[i] = h[i];
        coef[i] = (float)h[i];
      }
      CK(launch_vec_update(b.w, b.w, V(0), b.ld, j + 1, coef, 1.f, n, vg, b.part, b.dout, s), "Gram-Schmidt update");
      if ((rc = read_doubles(b.dout, h, j + 2, s))) return rc;
      double h2sq = 0.0;
      for (int i = 0; i <= j; ++i) {
        hj[i] += h[i];
        coef[i] = (float)h[i];
        h2sq += h[i] * h[i];
      }
      const double nrm2 = h[j + 1] - h2sq;
      hj[j + 1] = nrm2 > 0.0 ? sqrt(nrm2) : 0.0;
      // apply the previous rotations, then a new one that zeroes hj[j + 1]
      for (int i = 0; i < j; ++i) {
        const double t = cs[i] * hj[i] + sn[i] * hj[i + 1];
        hj[i + 1] = -sn[i] * hj[i] + cs[i] * hj[i + 1];
        hj[i] = t;
      }
      const double hn = hj[j + 1];
      const double r = sqrt(hj[j] * hj[j] + hn * hn);
      cs[j] = r > 0.0 ? hj[j] / r : 1.0;
      sn[j] = r > 0.0 ? hn / r : 0.0;
      hj[j] = r;
      gv[j + 1] = -sn[j] * gv[j];
      gv[j] = cs[j] * gv[j];
      for (int i = 0; i <= j; ++i) H[i][j] = hj[i];
      k = j + 1;
      const bool breakdown = !(hn > 1e-30 * beta);
      if (!breakdown)
        CK(launch_vec_update(b.w, V(j + 1), V(0), b.ld, j + 1, coef, (float)(1.0 / hn), n, vg, b.part, nullptr, s),
           "new basis vector");
      // estimated L1 residual: the 2-norm estimate |g_{j+1}| scaled like this cycle's start
      if (breakdown || fabs(gv[j + 1]) * l1_per_l2 < 0.5 * thr || *ops >= max_ops) break;
    }
    // x += V y, H y = g (upper triangular)
    double y[kGmresRestart];
    for (int i = k - 1; i >= 0; --i) {
      double t = gv[i];
      for (int l = i + 1; l < k; ++l) t -= H[i][l] * y[l];
      y[i] = H[i][i] != 0.0 ? t / H[i][i] : 0.0;
    }
    for (int i = 0; i < k; ++i) coef[i] = (float)-y[i];
    CK(launch_vec_update(x, x, V(0), b.ld, k, coef, 1.f, n, vg, b.part, nullptr, s), "update solution");
  }
}

}  // namespace
}  // namespace nwgpu

extern "C" int nwgpu_wpr_run(nwgpu_graph* g, const float* teleport, float* ranks, float damping, float threshold,
                             uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats) {
  clear_error();
  const nwgpu_pr_options opt = read_options(options);
  int                    rc = check_common(g, ranks, damping, opt);
  if (rc) return rc;
  const uint64_t n = g->n;
  // weights per entry on top of the plain sweep's bytes, plus the base term per row
  init_stats(stats, 8.0 * (double)g->nnz + 4.0 * (double)(n + 1) + 24.0 * (double)n);
  if (n == 0) return NWGPU_OK;
  cudaStream_t s = opt.stream ? (cudaStream_t)opt.stream : g->stream;
  if ((rc = ensure_solve_buffers(g)) || (rc = ensure_wpr(g))) return rc;
  WprBuffers&  b = g->wpr;
  const float* t = nullptr;
  if ((rc = device_vector(teleport, b.stage, n, opt.device_ptrs != 0, s, &t))) return rc;
  CK(launch_wpr_prepare(t, g->g.inv, b.t.s, n, damping, b.vbase, g->rank, g->contrib[0], g->sms, s), "wpr prepare");
  if ((rc = start_state(g, max_iters, threshold, s))) return rc;
  SweepArgs a = make_sweep_args(g, damping, 0.f, kTeleportUniform, 0u);
  a.w = g->g.w;
  a.vbase = b.vbase;
  a.vaux = b.t.s;
  CK(cudaEventRecord(g->ev0, s), "cudaEventRecord");
  PrState fin{};
  if ((rc = run_sweeps(g, a, opt.launch, max_iters, s, &fin, &g->plan, kModeWeighted))) return rc;
  CK(cudaEventRecord(g->ev1, s), "cudaEventRecord");
  float* dst = opt.device_ptrs ? ranks : b.stage;
  CK(launch_gather_f32(g->rank, g->g.perm, dst, n, g->sms, s), "permute ranks");
  if (!opt.device_ptrs) CK(cudaMemcpyAsync(ranks, dst, n * sizeof(float), cudaMemcpyDeviceToHost, s), "copy ranks");
  CK(cudaStreamSynchronize(s), "copy ranks");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, g->ev0, g->ev1);
  if ((rc = finish_stats(g, fin, ms, stats, s))) return rc;
  if (fin.aborted) return fail(NWGPU_ERR_ABORTED, "solve aborted after %llu sweeps", (unsigned long long)fin.iter);
  return NWGPU_OK;
}

extern "C" int nwgpu_pr_vjp(nwgpu_graph* g, const float* ranks, const float* dL_dr, float* dL_dw, float* dL_dt, float damping,
                            float threshold, uint64_t max_iters, const nwgpu_pr_options* options, nwgpu_pr_stats* stats) {
  clear_error();
  const nwgpu_pr_options opt = read_options(options);
  int                    rc = check_common(g, ranks, damping, opt);
  if (rc) return rc;
  const uint64_t n = g->n, nnz = g->nnz;
  if (n && !dL_dr) return fail(NWGPU_ERR_INVALID_ARG, "dL_dr is NULL");
  init_stats(stats, 8.0 * (double)nnz + 4.0 * (double)(n + 1) + 24.0 * (double)n);
  if (n == 0) return NWGPU_OK;
  cudaStream_t s = opt.stream ? (cudaStream_t)opt.stream : g->stream;
  if ((rc = ensure_solve_buffers(g)) || (rc = ensure_wpr(g))) return rc;
  WprBuffers& b = g->wpr;
  if (!b.tplan.ok)
    return fail(NWGPU_ERR_UNSUPPORTED,
                "the adjoint sweep needs the out-rows in the relabelled (non-increasing length) order; "
                "this holds for symmetric graphs");
  const float *r = nullptr, *c = nullptr;
  if ((rc = device_vector(ranks, b.stage, n, opt.device_ptrs != 0, s, &r))) return rc;
  if ((rc = device_vector(dL_dr, b.stage2, n, opt.device_ptrs != 0, s, &c))) return rc;
  CK(launch_vjp_prepare(r, c, g->g.inv, b.t.s, n, damping, b.r_int, b.vbase, b.vaux, g->rank, g->contrib[0], g->sms, s),
     "vjp prepare");
  SweepArgs a = make_sweep_args(g, damping, 0.f, kTeleportUniform, 0u);
  a.row_ptr = b.t.row_ptr;
  a.col = b.t.col;
  a.w = b.t.w;
  a.vbase = b.vbase;
  a.vaux = b.vaux;
  a.res_part = b.res;
  const char* solver = getenv("NWGPU_VJP_SOLVER");
  const bool  jacobi = solver && !strcmp(solver, "jacobi");
  PrState     fin{};
  if (jacobi) {
    if ((rc = start_state(g, max_iters, threshold, s))) return rc;
    CK(cudaEventRecord(g->ev0, s), "cudaEventRecord");
    if ((rc = run_sweeps(g, a, opt.launch, max_iters, s, &fin, &b.tplan, kModeAdjoint))) return rc;
  } else {
    if ((rc = ensure_gmres(g))) return rc;
    CK(launch_neg_dinv(b.t.s, n, damping, b.vneg, g->sms, s), "-d/s");
    CK(cudaEventRecord(g->ev0, s), "cudaEventRecord");
    uint64_t ops = 0;
    double   res = 0.0;
    bool     conv = false;
    if ((rc = gmres_adjoint(g, a, b.vbase, g->rank, (double)threshold, max_iters, s, &ops, &res, &conv))) return rc;
    fin.iter = ops;
    fin.last_error = res;
    fin.converged = conv ? 1u : 0u;
  }
  // gradients from the adjoint l (in g->rank)
  if (dL_dw) {
    if (!opt.device_ptrs && !b.gw) CK(dalloc(g, &b.gw, nnz), "cudaMalloc(dL/dw staging)");
    float* dst = opt.device_ptrs ? dL_dw : b.gw;
    CK(launch_vjp_grad_w(b.t, g->g.col, g->g.emap, b.r_int, g->rank, b.vbase, n, nnz, damping, b.f, b.q, dst, g->sms, s),
       "dL/dw");
    if (!opt.device_ptrs) CK(cudaMemcpyAsync(dL_dw, dst, nnz * sizeof(float), cudaMemcpyDeviceToHost, s), "copy dL/dw");
  }
  if (dL_dt) {
    float* dst = opt.device_ptrs ? dL_dt : b.stage;
    CK(launch_vjp_grad_t(g->rank, g->g.perm, n, damping, dst, g->sms, s), "dL/dt");
    if (!opt.device_ptrs) CK(cudaMemcpyAsync(dL_dt, dst, n * sizeof(float), cudaMemcpyDeviceToHost, s), "copy dL/dt");
  }
  CK(cudaEventRecord(g->ev1, s), "cudaEventRecord");
  CK(cudaStreamSynchronize(s), "vjp");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, g->ev0, g->ev1);
  if ((rc = finish_stats(g, fin, ms, stats, s))) return rc;
  if (fin.aborted) return fail(NWGPU_ERR_ABORTED, "solve aborted after %llu sweeps", (unsigned long long)fin.iter);
  return NWGPU_OK;
}

namespace nwgpu {
__global__ void spmv_fill_kernel(float* __restrict__ p, uint64_t n, float v) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}
}  // namespace nwgpu

// y = A x over the graph's rows: one sweep of the weighted binned kernel with
// damping 1, base terms 0 and out-weight sums 1, so each row's update
// fmaf(1, z, 0) is its weighted sum z = sum_k w_k x[col_k] exactly.
extern "C" int nwgpu_spmv(nwgpu_graph* g, const float* x, float* y, const nwgpu_pr_options* options) {
  clear_error();
  const nwgpu_pr_options opt = read_options(options);
  int                    rc = check_common(g, y, 1.0f, opt);
  if (rc) return rc;
  const uint64_t n = g->n;
  if (n && !x) return fail(NWGPU_ERR_INVALID_ARG, "x is NULL");
  if (n == 0) return NWGPU_OK;
  cudaStream_t s = opt.stream ? (cudaStream_t)opt.stream : g->stream;
  if ((rc = ensure_solve_buffers(g))) return rc;
  if (!g->unit) {
    CK(dalloc(g, &g->unit, n), "cudaMalloc(spmv ones)");
    CK(dalloc(g, &g->zero, n), "cudaMalloc(spmv zeros)");
    spmv_fill_kernel<<<g->sms * 4, 256, 0, g->stream>>>(g->unit, n, 1.0f);
    CK(cudaGetLastError(), "spmv ones");
    CK(cudaStreamSynchronize(g->stream), "spmv buffers");
  }
  // x in internal order as the sweep's contributions
  const float* xd = x;
  if (!opt.device_ptrs) {
    CK(cudaMemcpyAsync(g->stage_u32, x, n * sizeof(float), cudaMemcpyHostToDevice, s), "copy x");
    xd = reinterpret_cast<const float*>(g->stage_u32);
  }
  CK(launch_gather_f32(xd, g->g.inv, g->contrib[0], n, g->sms, s), "permute x");
  if ((rc = start_state(g, 1, -1.0f, s))) return rc;
  SweepArgs a = make_sweep_args(g, 1.0f, 0.f, kTeleportUniform, 0u);
  a.w = g->g.w;
  a.vbase = g->zero;
  a.vaux = g->unit;
  PrState fin{};
  if ((rc = run_sweeps(g, a, NWGPU_LAUNCH_STREAM, 1, s, &fin, &g->plan, kModeWeighted))) return rc;
  float* dst = opt.device_ptrs ? y : reinterpret_cast<float*>(g->stage_u32);
  CK(launch_gather_f32(g->rank, g->g.perm, dst, n, g->sms, s), "permute y");
  if (!opt.device_ptrs) CK(cudaMemcpyAsync(y, dst, n * sizeof(float), cudaMemcpyDeviceToHost, s), "copy y");
  CK(cudaStreamSynchronize(s), "spmv");
  return NWGPU_OK;
}
