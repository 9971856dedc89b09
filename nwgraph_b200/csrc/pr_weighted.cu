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

// Per-vertex factors of dL/dw: f_j = d r_j / s_j, q_j = (l_j - c_j) / d
// (= sum over j's out-entries of (w / s_j) l_dest at the adjoint's fixed point).
__global__ void vjp_fq_kernel(const float* __restrict__ r_int, const float* __restrict__ s, const float* __restrict__ lam,
                              const float* __restrict__ c_int, uint64_t n, float damping, float* __restrict__ f,
                              float* __restrict__ q) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
    const bool live = damping > 0.f && s[j] > 0.f;
    f[j] = live ? damping * r_int[j] / s[j] : 0.f;
    q[j] = live ? (lam[j] - c_int[j]) / damping : 0.f;
  }
}

// dL/dw_k = f_j (l_i - q_j) for forward entry k of row i, col[k] = j; written
// to the input entry emap[k].
__global__ void vjp_grad_w_kernel(const uint32_t* __restrict__ erow, const uint32_t* __restrict__ col,
                                  const uint32_t* __restrict__ emap, const float* __restrict__ f,
                                  const float* __restrict__ q, const float* __restrict__ lam, uint64_t nnz,
                                  float* __restrict__ d_w) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
    const uint32_t j = __ldcs(col + k);
    const float    g = f[j] * (lam[__ldcs(erow + k)] - q[j]);
    d_w[emap ? __ldcs(emap + k) : k] = g;
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

cudaError_t launch_vjp_grad_w(const Transposed& t, const uint32_t* col, const uint32_t* emap, const float* r_int,
                              const float* lam, const float* c_int, uint64_t n, uint64_t nnz, float damping, float* f,
                              float* q, float* d_w, int sms, cudaStream_t st) {
  if (n) {
    vjp_fq_kernel<<<sms * 8, 256, 0, st>>>(r_int, t.s, lam, c_int, n, damping, f, q);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (!nnz) return cudaSuccess;
  vjp_grad_w_kernel<<<sms * 8, 256, 0, st>>>(t.erow, col, emap, f, q, lam, nnz, d_w);
  return cudaGetLastError();
}

cudaError_t launch_vjp_grad_t(const float* lam, const uint32_t* perm, uint64_t n, float damping, float* d_t, int sms,
                              cudaStream_t st) {
  if (!n) return cudaSuccess;
  vjp_grad_t_kernel<<<sms * 8, 256, 0, st>>>(lam, perm, n, (float)(1.0 - (double)damping), d_t);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Vector kernels of the GMRES adjoint solve (api_wpr.cu). Every reduction
// runs in FP64 in a fixed order: per-block partials over contiguous ranges,
// then one warp per output over the blocks.
// ---------------------------------------------------------------------------
constexpr int kVecThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* s_red) {
  v = warp_sum_lane0(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kVecThreads / 32; ++w) t += s_red[w];
  __syncthreads();
  return t;  // valid in thread 0
}

// out[i] = sum_b part[b * nv + i], lane-strided over the blocks, fixed tree.
__global__ void vec_reduce_kernel(const double* __restrict__ part, int nblocks, int nv, double* __restrict__ out) {
  const int i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= nv) return;
  double acc = 0.0;
  for (int b = lane; b < nblocks; b += 32) acc += part[(uint64_t)b * nv + i];
  acc = warp_sum_lane0(acc);
  if (lane == 0) out[i] = acc;
}

struct VecCoeffs {
  float c[kGmresMaxBasis];
};

// One pass over the nv (<= NV) basis vectors of V (stride ld) and x:
//   UPDATE: y[k] = scale * (x[k] - sum_i coef[i] V_i[k])   (else y = x, unwritten)
//   DOTS:   part[b * (nv + 1) + i] = block b's sum of V_i[k] y[k], i < nv,
//           and part[b * (nv + 1) + nv] = block b's sum of y[k]^2.
// x and y may alias (each thread owns its elements). Per-thread FP32
// partials over at most chunk / 256 elements, FP64 from the warp reduction
// on, fixed order.
template <int NV, bool UPDATE, bool DOTS>
__global__ void __launch_bounds__(kVecThreads) vec_gs_kernel(const float* x, float* y, const float* __restrict__ V,
                                                             uint64_t ld, int nv, const VecCoeffs a, float scale,
                                                             uint64_t n, uint64_t chunk, double* __restrict__ part) {
  __shared__ double s_red[kVecThreads / 32][NV + 1];
  const uint64_t    k0 = (uint64_t)blockIdx.x * chunk, k1 = min(n, k0 + chunk);
  float             acc[NV + 1];
#pragma unroll
  for (int i = 0; i <= NV; ++i) acc[i] = 0.f;
  for (uint64_t k = k0 + threadIdx.x; k < k1; k += kVecThreads) {
    float vv[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) vv[i] = (i < nv) ? V[(uint64_t)i * ld + k] : 0.f;
    float v = x[k];
    if constexpr (UPDATE) {
#pragma unroll
      for (int i = 0; i < NV; ++i) v = fmaf(-a.c[i], vv[i], v);
      v *= scale;
      y[k] = v;
    }
    if constexpr (DOTS) {
#pragma unroll
      for (int i = 0; i < NV; ++i) acc[i] = fmaf(vv[i], v, acc[i]);
      acc[NV] = fmaf(v, v, acc[NV]);
    }
  }
  if constexpr (DOTS) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i <= NV; ++i) {
      const double t = warp_sum_lane0((double)acc[i]);
      if (lane == 0) s_red[warp][i] = t;
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= nv; i += kVecThreads) {
      const int src = (i == nv) ? NV : i;  // the norm sits after the NV dot slots
      double    t = 0.0;
      for (int w = 0; w < kVecThreads / 32; ++w) t += s_red[w][src];
      part[(uint64_t)blockIdx.x * (nv + 1) + i] = t;
    }
  }
}

template <bool UPDATE, bool DOTS>
static cudaError_t launch_gs(const float* x, float* y, const float* V, uint64_t ld, int nv, const VecCoeffs& a, float scale,
                             uint64_t n, const VecGrid& vg, double* part, cudaStream_t st) {
  if (nv <= 8)
    vec_gs_kernel<8, UPDATE, DOTS><<<vg.blocks, kVecThreads, 0, st>>>(x, y, V, ld, nv, a, scale, n, vg.chunk, part);
  else if (nv <= 16)
    vec_gs_kernel<16, UPDATE, DOTS><<<vg.blocks, kVecThreads, 0, st>>>(x, y, V, ld, nv, a, scale, n, vg.chunk, part);
  else if (nv <= 24)
    vec_gs_kernel<24, UPDATE, DOTS><<<vg.blocks, kVecThreads, 0, st>>>(x, y, V, ld, nv, a, scale, n, vg.chunk, part);
  else
    vec_gs_kernel<32, UPDATE, DOTS><<<vg.blocks, kVecThreads, 0, st>>>(x, y, V, ld, nv, a, scale, n, vg.chunk, part);
  return cudaGetLastError();
}

// y[k] = alpha * x[k] + beta * y[k]; with part: block b's sum of |y[k]|
// (beta = 0: y is written without being read).
__global__ void __launch_bounds__(kVecThreads) vec_axpby_kernel(float alpha, const float* __restrict__ x, float beta,
                                                                float* __restrict__ y, uint64_t n, uint64_t chunk,
                                                                double* __restrict__ part) {
  __shared__ double s_red[kVecThreads / 32];
  const uint64_t k0 = (uint64_t)blockIdx.x * chunk, k1 = min(n, k0 + chunk);
  double         acc = 0.0;
  for (uint64_t k = k0 + threadIdx.x; k < k1; k += kVecThreads) {
    const float v = beta == 0.f ? alpha * x[k] : fmaf(alpha, x[k], beta * y[k]);
    y[k] = v;
    acc += fabs((double)v);
  }
  if (part) {
    const double t = block_sum(acc, s_red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

// vaux = -d / s (0 where s = 0): with vbase = v, one adjoint sweep then
// computes v - d P^T v.
__global__ void neg_dinv_kernel(const float* __restrict__ s, uint64_t n, float damping, float* __restrict__ vaux) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    vaux[i] = s[i] > 0.f ? -damping / s[i] : 0.f;
}

VecGrid vec_grid(uint64_t n, int sms) {
  VecGrid g;
  g.blocks = sms * 4;
  g.chunk = (n + (uint64_t)g.blocks - 1) / (uint64_t)g.blocks;
  g.chunk = (g.chunk + 3) & ~3ull;
  if (!g.chunk) g.chunk = 4;
  g.blocks = (int)((n + g.chunk - 1) / g.chunk);
  if (g.blocks < 1) g.blocks = 1;
  return g;
}

// out[0..nv) = V_i . x, out[nv] = x . x
cudaError_t launch_vec_dots(const float* V, uint64_t ld, int nv, const float* x, uint64_t n, const VecGrid& vg,
                            double* part, double* out, cudaStream_t st) {
  if (nv < 1 || nv > kGmresMaxBasis) return cudaErrorInvalidValue;
  VecCoeffs   a = {};
  cudaError_t e = launch_gs<false, true>(x, nullptr, V, ld, nv, a, 1.f, n, vg, part, st);
  if (e != cudaSuccess) return e;
  vec_reduce_kernel<<<(nv + 1 + 7) / 8, 256, 0, st>>>(part, vg.blocks, nv + 1, out);
  return cudaGetLastError();
}

// y = scale * (x - sum_i coef[i] V_i); with out: out[0..nv) = V_i . y, out[nv] = y . y
cudaError_t launch_vec_update(const float* x, float* y, const float* V, uint64_t ld, int nv, const float* coef, float scale,
                              uint64_t n, const VecGrid& vg, double* part, double* out, cudaStream_t st) {
  if (nv < 1 || nv > kGmresMaxBasis) return cudaErrorInvalidValue;
  VecCoeffs a = {};
  for (int i = 0; i < nv; ++i) a.c[i] = coef[i];
  if (!out) return launch_gs<true, false>(x, y, V, ld, nv, a, scale, n, vg, part, st);
  cudaError_t e = launch_gs<true, true>(x, y, V, ld, nv, a, scale, n, vg, part, st);
  if (e != cudaSuccess) return e;
  vec_reduce_kernel<<<(nv + 1 + 7) / 8, 256, 0, st>>>(part, vg.blocks, nv + 1, out);
  return cudaGetLastError();
}

cudaError_t launch_vec_axpby(float alpha, const float* x, float beta, float* y, uint64_t n, const VecGrid& vg,
                             double* part, double* l1_out, cudaStream_t st) {
  vec_axpby_kernel<<<vg.blocks, kVecThreads, 0, st>>>(alpha, x, beta, y, n, vg.chunk, l1_out ? part : nullptr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !l1_out) return e;
  vec_reduce_kernel<<<1, 256, 0, st>>>(part, vg.blocks, 1, l1_out);
  return cudaGetLastError();
}

// Solve state for one operator application: one sweep from parity 0.
__global__ void op_state_kernel(PrState* st) {
  PrState h = {};
  h.max_iters = 1ull;
  h.chunk_end = kGraphChunk;
  h.threshold = -1.0;  // never "converged": the sweep is an operator application
  *st = h;
}

cudaError_t launch_op_state(PrState* st, cudaStream_t s) {
  op_state_kernel<<<1, 1, 0, s>>>(st);
  return cudaGetLastError();
}

cudaError_t launch_neg_dinv(const float* s, uint64_t n, float damping, float* vaux, int sms, cudaStream_t st) {
  if (!n) return cudaSuccess;
  neg_dinv_kernel<<<sms * 8, 256, 0, st>>>(s, n, damping, vaux);
  return cudaGetLastError();
}

}  // namespace nwgpu
