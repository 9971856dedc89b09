// Weighted PageRank and its implicit adjoint: the per-solve set-up kernels and
// the gradient pass. The sweeps themselves are the binned kernel's
// kModeWeighted / kModeAdjoint instances (pr_binned.cu).
//
// With edge j -> i of weight w (entry k of in-row i, col[k] = j), s_j the
// out-weight sum of j and teleport t (a distribution over the vertices):
//   forward  r_i = (1-d) t_i + d sum_k w_k r_j / s_j
//   adjoint  l_j = c_j + d sum_{k: col[k] = j} (w_k / s_j) l_i   for L = sum_v c_v r_v
//   dL/dt_v  = (1-d) l_v
//   dL/dw_k  = d r_j / s_j (l_i - q_j),  q_j = sum_{k': col[k'] = j} (w_k' / s_j) l_row(k') = (l_j - c_j) / d
// The forward is page_rank's update (include/nwgraph/algorithms/page_rank.hpp:133)
// with weighted, out-normalised contributions and a teleport vector; the
// adjoint solves the transposed system with the same sweep over the out-row
// CSR, so no forward iterates are kept.
#include "common.cuh"
#include "engine.h"

namespace nwgpu {

// Internal-order vectors of a weighted solve. t is in input order (NULL:
// uniform 1/n). vbase = (1-d) t, rank = r0 = t, contrib = r0 / s.
__global__ void wpr_prepare_kernel(const float* __restrict__ t, const uint32_t* __restrict__ inv, const float* __restrict__ s,
                                   uint64_t n, float one_minus_d, float uniform, float* __restrict__ vbase,
                                   float* __restrict__ rank, float* __restrict__ contrib) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float ti = t ? t[inv[i]] : uniform;
    vbase[i] = one_minus_d * ti;
    rank[i] = ti;
    contrib[i] = ti / s[i];
  }
}

// Internal-order vectors of an adjoint solve from the input-order forward
// ranks r and cotangent c: r_int, vbase = c, vaux = d / s (0 where s = 0:
// such a vertex has no out-entries, so its sum is empty), l0 = c.
__global__ void vjp_prepare_kernel(const float* __restrict__ r, const float* __restrict__ c, const uint32_t* __restrict__ inv,
                                   const float* __restrict__ s, uint64_t n, float damping, float* __restrict__ r_int,
                                   float* __restrict__ vbase, float* __restrict__ vaux, float* __restrict__ lam,
                                   float* __restrict__ contrib) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t v = inv[i];
    const float    ci = c[v];
    r_int[i] = r[v];
    vbase[i] = ci;
    vaux[i] = s[i] > 0.f ? damping / s[i] : 0.f;
    lam[i] = ci;
    contrib[i] = ci;
  }
}

// dL/dw over the out-row CSR: entry e of out-row j is forward entry fwd[e]
// (input entry emap[fwd[e]]) with destination i = tcol[e]. The row's factor
// d r_j / s_j and q_j are computed once per entry from per-vertex vectors.
__global__ void vjp_grad_w_kernel(const uint32_t* __restrict__ trow, const uint32_t* __restrict__ tcol,
                                  const uint32_t* __restrict__ fwd, const uint32_t* __restrict__ emap,
                                  const float* __restrict__ s, const float* __restrict__ r_int,
                                  const float* __restrict__ lam, const float* __restrict__ c_int, uint64_t n, uint64_t nnz,
                                  float damping, float* __restrict__ d_w) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
    uint64_t lo = 0, hi = n;  // out-row j: trow[j] <= e < trow[j + 1]
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) >> 1;
      if (trow[mid] <= e)
        lo = mid;
      else
        hi = mid;
    }
    const uint32_t j = (uint32_t)lo;
    float          g = 0.f;
    if (damping > 0.f) {
      const float q = (lam[j] - c_int[j]) / damping;
      g = damping * r_int[j] / s[j] * (lam[tcol[e]] - q);
    }
    const uint32_t k = fwd[e];
    d_w[emap ? emap[k] : k] = g;
  }
}

// dL/dt in input order: (1-d) l[perm[v]].
__global__ void vjp_grad_t_kernel(const float* __restrict__ lam, const uint32_t* __restrict__ perm, uint64_t n,
                                  float one_minus_d, float* __restrict__ d_t) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) d_t[v] = one_minus_d * lam[perm[v]];
}

cudaError_t launch_wpr_prepare(const float* t, const uint32_t* inv, const float* s, uint64_t n, float damping,
                               float* vbase, float* rank, float* contrib, int sms, cudaStream_t st) {
  if (!n) return cudaSuccess;
  const float uniform = (float)(1.0 / (double)n);
  wpr_prepare_kernel<<<sms * 8, 256, 0, st>>>(t, inv, s, n, (float)(1.0 - (double)damping), uniform, vbase, rank, contrib);
  return cudaGetLastError();
}

cudaError_t launch_vjp_prepare(const float* r, const float* c, const uint32_t* inv, const float* s, uint64_t n,
                               float damping, float* r_int, float* vbase, float* vaux, float* lam, float* contrib, int sms,
                               cudaStream_t st) {
  if (!n) return cudaSuccess;
  vjp_prepare_kernel<<<sms * 8, 256, 0, st>>>(r, c, inv, s, n, damping, r_int, vbase, vaux, lam, contrib);
  return cudaGetLastError();
}

cudaError_t launch_vjp_grad_w(const Transposed& t, const uint32_t* emap, const float* r_int, const float* lam,
                              const float* c_int, uint64_t n, uint64_t nnz, float damping, float* d_w, int sms,
                              cudaStream_t st) {
  if (!nnz) return cudaSuccess;
  vjp_grad_w_kernel<<<sms * 8, 256, 0, st>>>(t.row_ptr, t.col, t.fwd, emap, t.s, r_int, lam, c_int, n, nnz, damping, d_w);
  return cudaGetLastError();
}

cudaError_t launch_vjp_grad_t(const float* lam, const uint32_t* perm, uint64_t n, float damping, float* d_t, int sms,
                              cudaStream_t st) {
  if (!n) return cudaSuccess;
  vjp_grad_t_kernel<<<sms * 8, 256, 0, st>>>(lam, perm, n, (float)(1.0 - (double)damping), d_t);
  return cudaGetLastError();
}

}  // namespace nwgpu
