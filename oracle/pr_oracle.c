/*
 * CPU oracle for the PageRank hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * this library, and only as the checker. The product (nwgraph_b200 +
 * libnwgpu.so) never calls it and has no CPU fallback.
 *
 * Parity pin: orc_pr_jacobi_f32 and orc_pr_gauss_seidel_f32 are checked
 * bit-for-bit against NWGraph's page_rank_v10 / page_rank (v11, 1 thread)
 * compiled from the reference headers (oracle/_ref/libnwref.so), and
 * orc_pr_v1_f64 against the karate golden vector of test/page_rank_test.cpp:72-75
 * (fixtures in tests/golden/, generated by tests/golden/make_golden.py).
 * The extensions (personalized teleport, edge weights, implicit adjoint) have
 * no counterpart in the reference; they are pinned by FP64 central finite
 * differences and by internal consistency (tests/test_oracle.py).
 *
 * CSR convention (adjacency<1> of the reference, adjacency.hpp:86-195):
 * row i lists the in-neighbours j of i, i.e. entry k of row i is edge j->i;
 * deg[j] is the out-degree of j (bench/gapbs/common.hpp:110-121).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/*
 * Host threads for the FP64 oracles (orc_pr_f64, orc_pr_vjp_f64): every row
 * is still summed by one thread in CSR order, so their vectors do not depend
 * on the thread count; only the L1 change of a sweep is summed per thread and
 * then in thread order. ORACLE_THREADS overrides the online core count.
 */
static int orc_threads(void) {
  const char* e = getenv("ORACLE_THREADS");
  long        t = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
  if (t < 1) t = 1;
  if (t > 64) t = 64;
  return (int)t;
}

typedef void (*orc_rows_fn)(void* ctx, uint64_t lo, uint64_t hi, int part);

typedef struct {
  orc_rows_fn fn;
  void*       ctx;
  uint64_t    lo, hi;
  int         part;
} orc_task;

static void* orc_task_run(void* a) {
  orc_task* t = (orc_task*)a;
  t->fn(t->ctx, t->lo, t->hi, t->part);
  return NULL;
}

/* Runs fn over rows [0, n) in `parts` ranges of about equal rows + entries
 * (row_ptr, may be NULL for rows alone), one thread each; part p gets the
 * p-th range. */
static void orc_parallel_rows(const uint32_t* row_ptr, uint64_t n, int parts, orc_rows_fn fn, void* ctx) {
  orc_task  task[64];
  pthread_t th[64];
  int       started[64] = {0};
  uint64_t  total = n + (row_ptr ? row_ptr[n] : 0), lo = 0;
  for (int p = 0; p < parts; ++p) {
    uint64_t want = total * (uint64_t)(p + 1) / (uint64_t)parts, hi = lo;
    if (p == parts - 1) {
      hi = n;
    } else {
      uint64_t a = lo, b = n; /* smallest hi with hi + row_ptr[hi] >= want */
      while (a < b) {
        uint64_t m = (a + b) / 2;
        if (m + (row_ptr ? row_ptr[m] : 0) < want) a = m + 1; else b = m;
      }
      hi = a;
    }
    task[p] = (orc_task){fn, ctx, lo, hi, p};
    lo = hi;
  }
  for (int p = 1; p < parts; ++p) started[p] = pthread_create(&th[p], NULL, orc_task_run, &task[p]) == 0;
  orc_task_run(&task[0]);
  for (int p = 1; p < parts; ++p) {
    if (started[p]) pthread_join(th[p], NULL);
    else orc_task_run(&task[p]);
  }
}

/* Constants exactly as page_rank.hpp:92-94: computed in double, stored as float. */
static void pr_constants_f32(uint64_t n, float damping, float* init, float* base) {
  *init = (float)(1.0 / (double)n);
  *base = (float)((1.0 - (double)damping) / (double)n);
}

/*
 * Restates nw::graph::page_rank_v10 (experimental/algorithms/page_rank.hpp:377-432):
 * Jacobi. Per sweep: contrib[i] = rank[i] / deg[i] (:401-405), then per row in
 * row order z = sum of contrib over the row in CSR order (:413-415),
 * rank = base + d*z (:417, contracted to one FMA as GCC does for the
 * reference's gnu++20 build), error += |new - old| in double (:418); stop
 * after the sweep when error < threshold (:427). Returns sweeps run.
 * errors[] (may be NULL) receives each sweep's L1 error.
 */
int64_t orc_pr_jacobi_f32(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const uint32_t* deg, float* rank,
                          float damping, float threshold, uint64_t max_iters, double* errors) {
  float init, base;
  pr_constants_f32(n, damping, &init, &base);
  float* contrib = (float*)malloc((n ? n : 1) * sizeof(float));
  if (!contrib) return -1;
  for (uint64_t i = 0; i < n; ++i) rank[i] = init;
  uint64_t it = 0;
  for (; it < max_iters; ++it) {
    for (uint64_t i = 0; i < n; ++i) contrib[i] = rank[i] / (float)deg[i];
    double err = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
      float z = 0.0f;
      for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) z += contrib[col[k]];
      float old = rank[i];
      rank[i] = fmaf(damping, z, base);
      err += (double)fabsf(rank[i] - old);
    }
    if (errors) errors[it] = err;
    if (err < (double)threshold) {
      ++it;
      break;
    }
  }
  free(contrib);
  return (int64_t)it;
}

/*
 * Personalised variant of the restatement above (an extension with no
 * reference counterpart): teleport one-hot at `seed`, so base_i = (1 - d)
 * for i == seed (computed in double, stored as float) and 0 elsewhere, and
 * r(0) = e_seed. Everything else is page_rank_v10's sweep.
 */
int64_t orc_ppr_jacobi_f32(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const uint32_t* deg,
                           uint32_t seed, float* rank, float damping, float threshold, uint64_t max_iters,
                           double* errors) {
  const float base = (float)(1.0 - (double)damping);
  float*      contrib = (float*)malloc((n ? n : 1) * sizeof(float));
  if (!contrib) return -1;
  for (uint64_t i = 0; i < n; ++i) rank[i] = (i == seed) ? 1.0f : 0.0f;
  uint64_t it = 0;
  for (; it < max_iters; ++it) {
    for (uint64_t i = 0; i < n; ++i) contrib[i] = rank[i] / (float)deg[i];
    double err = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
      float z = 0.0f;
      for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) z += contrib[col[k]];
      float old = rank[i];
      rank[i] = fmaf(damping, z, (i == seed) ? base : 0.0f);
      err += (double)fabsf(rank[i] - old);
    }
    if (errors) errors[it] = err;
    if (err < (double)threshold) {
      ++it;
      break;
    }
  }
  free(contrib);
  return (int64_t)it;
}

/*
 * Restates nw::graph::page_rank v11 (algorithms/page_rank.hpp:89-148) run on
 * one thread: Gauss-Seidel, contrib initialised once (:114-118) and rewritten
 * in place right after each row's update (:135), so later rows of the same
 * sweep read the new value.
 */
int64_t orc_pr_gauss_seidel_f32(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const uint32_t* deg,
                                float* rank, float damping, float threshold, uint64_t max_iters, double* errors) {
  float init, base;
  pr_constants_f32(n, damping, &init, &base);
  float* contrib = (float*)malloc((n ? n : 1) * sizeof(float));
  if (!contrib) return -1;
  for (uint64_t i = 0; i < n; ++i) rank[i] = init;
  for (uint64_t i = 0; i < n; ++i) contrib[i] = rank[i] / (float)deg[i];
  uint64_t it = 0;
  for (; it < max_iters; ++it) {
    double err = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
      float z = 0.0f;
      for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) z += contrib[col[k]];
      float old = rank[i];
      rank[i] = fmaf(damping, z, base);
      err += (double)fabsf(rank[i] - old);
      contrib[i] = rank[i] / (float)deg[i];
    }
    if (errors) errors[it] = err;
    if (err < (double)threshold) {
      ++it;
      break;
    }
  }
  free(contrib);
  return (int64_t)it;
}

/*
 * Restates page_rank_v1 (experimental/algorithms/page_rank.hpp:82-119) with
 * Real = double, the form test/page_rank_test.cpp:93 calls: serial Jacobi,
 * init/base from page_rank.size() (:88-89), contrib = rank/deg (:99-102).
 */
int64_t orc_pr_v1_f64(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const uint32_t* deg, double* rank,
                      double damping, double threshold, uint64_t max_iters) {
  const double init = 1.0 / (double)n;
  const double base = (1.0 - damping) / (double)n;
  double*      contrib = (double*)malloc((n ? n : 1) * sizeof(double));
  if (!contrib) return -1;
  for (uint64_t i = 0; i < n; ++i) rank[i] = init;
  uint64_t it = 0;
  for (; it < max_iters; ++it) {
    double err = 0.0;
    for (uint64_t i = 0; i < n; ++i) contrib[i] = rank[i] / (double)deg[i];
    for (uint64_t i = 0; i < n; ++i) {
      double z = 0.0;
      for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) z += contrib[col[k]];
      double old = rank[i];
      rank[i] = fma(damping, z, base);
      err += fabs(rank[i] - old);
    }
    if (err < threshold) {
      ++it;
      break;
    }
  }
  free(contrib);
  return (int64_t)it;
}

/*
 * Out-weight sums s[j] = sum of w over the out-edges of j, gathered from the
 * in-row CSR (entry k of row i is edge col[k] -> i). With w == NULL this is the
 * out-degree.
 */
void orc_out_weight(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const float* w, double* s) {
  for (uint64_t j = 0; j < n; ++j) s[j] = 0.0;
  uint64_t nnz = row_ptr[n];
  for (uint64_t k = 0; k < nnz; ++k) s[col[k]] += w ? (double)w[k] : 1.0;
}

/*
 * General FP64 Jacobi power iteration with the reference's leak semantics
 * (no dangling redistribution, page_rank.hpp:94,133):
 *   r_i <- (1-d) t_i + d * sum_{k in row i} wn_k r_{col[k]}
 * where wn_k = w_k / s_{col[k]} (weighted, out-normalised) or 1/deg (w == NULL),
 * and t = teleport (NULL means the uniform 1/n of plain PageRank).
 * r starts at r0 (NULL: t, or 1/n for plain). Runs until the L1 change of a
 * sweep is < tol or max_iters sweeps. Returns sweeps run; *final_err = last L1.
 * This is the FP64 oracle O3 (plain) and O4 (PPR / weighted).
 */
typedef struct {
  const uint32_t *row_ptr, *col;
  const float*    w;
  const double *  teleport, *c, *r;
  double*         nr;
  double          damping, inv_n;
  double          err[64];
} orc_pr_sweep;

static void orc_pr_rows(void* p, uint64_t lo, uint64_t hi, int part) {
  orc_pr_sweep* a = (orc_pr_sweep*)p;
  double        err = 0.0;
  for (uint64_t i = lo; i < hi; ++i) {
    double z = 0.0;
    for (uint32_t k = a->row_ptr[i]; k < a->row_ptr[i + 1]; ++k) z += (a->w ? (double)a->w[k] : 1.0) * a->c[a->col[k]];
    double t = a->teleport ? a->teleport[i] : a->inv_n;
    a->nr[i] = (1.0 - a->damping) * t + a->damping * z;
    err += fabs(a->nr[i] - a->r[i]);
  }
  a->err[part] = err;
}

int64_t orc_pr_f64(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const float* w, const double* teleport,
                   const double* r0, double damping, double tol, uint64_t max_iters, double* r, double* final_err) {
  double* s = (double*)malloc((n ? n : 1) * sizeof(double));
  double* c = (double*)malloc((n ? n : 1) * sizeof(double));
  double* nr = (double*)malloc((n ? n : 1) * sizeof(double));
  if (!s || !c || !nr) return -1;
  orc_out_weight(row_ptr, col, n, w, s);
  for (uint64_t i = 0; i < n; ++i) r[i] = r0 ? r0[i] : (teleport ? teleport[i] : 1.0 / (double)n);
  uint64_t it = 0;
  double   err = INFINITY;
  const int    parts = n >= 65536 ? orc_threads() : 1;
  orc_pr_sweep sw = {row_ptr, col, w, teleport, c, r, nr, damping, 1.0 / (double)n, {0}};
  for (; it < max_iters; ++it) {
    for (uint64_t j = 0; j < n; ++j) c[j] = r[j] / s[j];
    orc_parallel_rows(row_ptr, n, parts, orc_pr_rows, &sw);
    err = 0.0;
    for (int p = 0; p < parts; ++p) err += sw.err[p];
    memcpy(r, nr, n * sizeof(double));
    if (err < tol) {
      ++it;
      break;
    }
  }
  if (final_err) *final_err = err;
  free(s);
  free(c);
  free(nr);
  return (int64_t)it;
}

/*
 * Implicit adjoint of the converged fixed point r = (1-d) t + d P r,
 * P_{i j} = wn(j->i). For L = sum_v cvec_v r_v:
 *   lambda = cvec + d P^T lambda, i.e. lambda_j = c_j + d sum_{i: j->i} wn(j->i) lambda_i
 *   dL/dt = (1-d) lambda
 *   dL/dw(j->i) = d r_j / s_j * (lambda_i - sum_{i'} wn(j->i') lambda_{i'})
 * (the last term is the derivative through the out-normalisation; w == NULL
 * means unit weights). The transpose is applied as a scatter over the in-row
 * CSR. Iterates lambda to L1 change < tol. Writes lambda, dL/dt (n) and
 * dL/dw (nnz, may be NULL). Returns sweeps run.
 */
typedef struct {
  const uint64_t* tptr;  /* n + 1: out-row j's entries are [tptr[j], tptr[j+1]) */
  const uint32_t* trow;  /* the in-row (destination) i of each entry, ascending k within j */
  const double*   twn;   /* its normalised weight wn(j->i) */
  const double *  lambda, *cvec;
  double*         out;   /* per j: cvec_j + d * sum (step), or the plain sum (damping < 0) */
  double          damping;
  double          err[64];
} orc_adj_sweep;

static void orc_adj_rows(void* p, uint64_t lo, uint64_t hi, int part) {
  orc_adj_sweep* a = (orc_adj_sweep*)p;
  double         err = 0.0;
  for (uint64_t j = lo; j < hi; ++j) {
    double z = 0.0;
    for (uint64_t e = a->tptr[j]; e < a->tptr[j + 1]; ++e) z += a->twn[e] * a->lambda[a->trow[e]];
    if (a->damping < 0.0) {
      a->out[j] = z;
    } else {
      double v = a->cvec[j] + a->damping * z;
      err += fabs(v - a->lambda[j]);
      a->out[j] = v;
    }
  }
  a->err[part] = err;
}

int64_t orc_pr_vjp_f64(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const float* w, const double* r,
                       const double* cvec, double damping, double tol, uint64_t max_iters, double* lambda, double* d_t,
                       double* d_w) {
  uint64_t  nnz = row_ptr[n];
  double*   s = (double*)malloc((n ? n : 1) * sizeof(double));
  double*   nl = (double*)malloc((n ? n : 1) * sizeof(double));
  double*   q = (double*)malloc((n ? n : 1) * sizeof(double));
  uint64_t* tptr = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  uint32_t* trow = (uint32_t*)malloc((nnz ? nnz : 1) * sizeof(uint32_t));
  double*   twn = (double*)malloc((nnz ? nnz : 1) * sizeof(double));
  if (!s || !nl || !q || !tptr || !trow || !twn) return -1;
  orc_out_weight(row_ptr, col, n, w, s);
  /* The out-row CSR, each out-row's entries in ascending in-row order: the
   * order in which a serial scatter over the in-row CSR adds them, so the
   * gathered sums equal that scatter's bit for bit. */
  for (uint64_t k = 0; k < nnz; ++k) ++tptr[col[k] + 1];
  for (uint64_t j = 0; j < n; ++j) tptr[j + 1] += tptr[j];
  {
    uint64_t* fill = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
    if (!fill) return -1;
    memcpy(fill, tptr, n * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i)
      for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
        uint32_t j = col[k];
        uint64_t e = fill[j]++;
        trow[e] = (uint32_t)i;
        twn[e] = (w ? (double)w[k] : 1.0) / s[j];
      }
    free(fill);
  }
  for (uint64_t j = 0; j < n; ++j) lambda[j] = cvec[j];
  const int     parts = n >= 65536 ? orc_threads() : 1;
  orc_adj_sweep sw = {tptr, trow, twn, lambda, cvec, nl, damping, {0}};
  uint64_t      it = 0;
  for (; it < max_iters; ++it) {
    orc_parallel_rows(NULL, n, parts, orc_adj_rows, &sw);
    double err = 0.0;
    for (int p = 0; p < parts; ++p) err += sw.err[p];
    memcpy(lambda, nl, n * sizeof(double));
    if (err < tol) {
      ++it;
      break;
    }
  }
  for (uint64_t j = 0; j < n; ++j) d_t[j] = (1.0 - damping) * lambda[j];
  if (d_w) {
    /* q_j = sum_{i: j->i} wn(j->i) lambda_i */
    orc_adj_sweep qs = {tptr, trow, twn, lambda, cvec, q, -1.0, {0}};
    orc_parallel_rows(NULL, n, parts, orc_adj_rows, &qs);
    for (uint64_t i = 0; i < n; ++i)
      for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
        uint32_t j = col[k];
        d_w[k] = damping * r[j] / s[j] * (lambda[i] - q[j]);
      }
  }
  free(s);
  free(nl);
  free(q);
  free(tptr);
  free(trow);
  free(twn);
  return (int64_t)it;
}

/*
 * Restates nw::graph::page_rank_v13 (experimental/algorithms/page_rank.hpp:
 * 552-625), the residual-push PageRank, on one thread: ranks start at 0 and
 * every residual at (float)(1 - d) (:562-568). Per iteration: for every
 * vertex, delta = 0, and if residual > threshold the residual moves into the
 * rank and, for out-degree > 0, delta = residual * d / deg in FP32 (:576-589);
 * then every row sums the positive deltas of its entries in CSR order, and
 * its residual becomes that sum if > 0, else 0 (:593-605). It stops after the
 * first iteration in which no vertex with out-degree > 0 pushed (:610-612).
 * Returns the iterations run; changed[] (may be NULL) receives how many
 * vertices pushed in each.
 */
int64_t orc_pr_residual_f32(const uint32_t* row_ptr, const uint32_t* col, uint64_t n, const uint32_t* deg, float* rank,
                            float damping, float threshold, uint64_t max_iters, double* changed) {
  float* delta = (float*)malloc((n ? n : 1) * sizeof(float));
  float* residual = (float*)malloc((n ? n : 1) * sizeof(float));
  if (!delta || !residual) {
    free(delta);
    free(residual);
    return -1;
  }
  for (uint64_t i = 0; i < n; ++i) {
    rank[i] = 0.0f;
    delta[i] = 0.0f;
    residual[i] = (float)(1.0 - (double)damping);
  }
  uint64_t it = 0;
  for (; it < max_iters; ++it) {
    uint64_t count = 0;
    for (uint64_t s = 0; s < n; ++s) {
      delta[s] = 0.0f;
      if (residual[s] > threshold) {
        const float old = residual[s];
        rank[s] += old;
        residual[s] = 0.0f;
        if (deg[s] > 0) {
          delta[s] = old * damping / (float)deg[s];
          ++count;
        }
      }
    }
    for (uint64_t i = 0; i < n; ++i) {
      float sum = 0.0f;
      for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
        if (delta[col[k]] > 0) sum += delta[col[k]];
      residual[i] = sum > 0 ? sum : 0.0f;
    }
    if (changed) changed[it] = (double)count;
    if (count == 0) {
      ++it;
      break;
    }
  }
  free(delta);
  free(residual);
  return (int64_t)it;
}
