// The time-integration variants of the stored-matrix linear system
// (Fem::Ls::CLinearSystem_SaveDiaM_Newmark and ..._NewmarkBeta,
// src/femls/linearsystem_fieldsave.cpp:367-880) on the device:
//
//  * dfm_mat_zero_rows - CMat_BlkCrs::SetBoundaryCondition_Row
//    (src/matvec/mat_blkcrs.cpp:910-951): the rows of fixed DOFs of the
//    stored matrix B zeroed (every block of the row, its diagonal included).
//  * dfm_newmark_residual - MakeResidual (:446-520 first order, :706-794
//    second order): the predictor t = u + dt (1 - gamma) v, or
//    t = u + dt v + dt^2 (1/2 - beta) a, then r = force - B t, r = 0 at fixed
//    DOFs, |r|.
//  * dfm_newmark_update - UpdateValueOfField (:522-566, :796-877): x holds the
//    solved velocity (first order) or acceleration (second order); fixed DOFs
//    take the old one into x, free DOFs advance u (and v), then v := x
//    (first order) or a := x (second order).
//
// Products and sums follow the reference's expressions term by term without
// contraction (__dmul_rn / __dadd_rn), so the updates are bit-identical to
// it; the residual's matrix-vector product sums in the device SpMV's order.
#include <algorithm>
#include <cmath>

#include "dfm_internal.h"

namespace dfm {

constexpr int kNmThreads = 256;

static int nm_grid(size_t n) {
  return (int)std::max<size_t>(1, std::min<size_t>((n + kNmThreads - 1) / kNmThreads, (size_t)kMaxBlocks));
}

#define NM_LOOP(k, n) \
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (n); k += (size_t)gridDim.x * blockDim.x)

// one thread per (block row, DOF): zero that row of the diagonal block and of
// every off-diagonal block of the block row
__global__ void k_zero_rows(unsigned N, unsigned b, const unsigned* __restrict__ rowptr, const int* __restrict__ flags,
                            double* __restrict__ diag, double* __restrict__ off) {
  NM_LOOP(t, (size_t)N * b) {
    if (!flags[t]) continue;
    const size_t i = t / b, d = t % b, bb = (size_t)b * b;
    for (unsigned c = 0; c < b; c++) diag[i * bb + d * b + c] = 0.0;
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++)
      for (unsigned c = 0; c < b; c++) off[(size_t)s * bb + d * b + c] = 0.0;
  }
}

// t = u + v*c1 (first order, c1 = dt*(1-gamma)); t = (u + v*dt) + a*c2
// (second order, c2 = dt*dt*(0.5-beta)) - AddValueFromNodeSegment adds val*alpha
__global__ void k_nm_predict(size_t n, int scheme, double c1, double c2, const double* __restrict__ u,
                             const double* __restrict__ v, const double* __restrict__ a, double* __restrict__ t) {
  NM_LOOP(k, n) {
    double s = __dadd_rn(u[k], __dmul_rn(v[k], c1));
    if (scheme == 2) s = __dadd_rn(s, __dmul_rn(a[k], c2));
    t[k] = s;
  }
}

// r = 0 at fixed DOFs (CBCFlag::SetZeroToBCDof); partials of (r, r)
__global__ void __launch_bounds__(kNmThreads)
k_nm_mask_norm(size_t n, const int* __restrict__ flags, double* __restrict__ r, double* part) {
  double acc = 0.0;
  NM_LOOP(k, n) {
    double rv = r[k];
    if (flags[k]) {
      rv = 0.0;
      r[k] = 0.0;
    }
    acc += rv * rv;
  }
  block_partial<kNmThreads>(acc, part);
}

__global__ void k_nm_sum(const double* part, int np, double* out) {
  const double s = reduce_partials(part, np);
  if (threadIdx.x == 0) *out = s;
}

// first order: free DOFs u += dt*(1-gamma)*v0 + dt*gamma*x; fixed x = v0; v = x
__global__ void k_nm_update1(size_t n, double dt, double gamma, const int* __restrict__ flags,
                             double* __restrict__ x, double* __restrict__ u, double* __restrict__ v) {
  const double c0 = __dmul_rn(dt, __dsub_rn(1.0, gamma)), c1 = __dmul_rn(dt, gamma);
  NM_LOOP(k, n) {
    const double v0 = v[k];
    double xv = x[k];
    if (flags[k] == 0) {
      u[k] = __dadd_rn(u[k], __dadd_rn(__dmul_rn(c0, v0), __dmul_rn(c1, xv)));
    } else {
      xv = v0;
      x[k] = xv;
    }
    v[k] = xv;
  }
}

// second order: free DOFs u += dt*v0 + dt*dt*(0.5-beta)*a0 + dt*dt*beta*x,
// v += dt*(1-gamma)*a0 + gamma*dt*x; fixed x = a0; a = x
__global__ void k_nm_update2(size_t n, double dt, double gamma, double beta, const int* __restrict__ flags,
                             double* __restrict__ x, double* __restrict__ u, double* __restrict__ v,
                             double* __restrict__ a) {
  const double dt2 = __dmul_rn(dt, dt);
  const double cu_a = __dmul_rn(dt2, __dsub_rn(0.5, beta)), cu_x = __dmul_rn(dt2, beta);
  const double cv_a = __dmul_rn(dt, __dsub_rn(1.0, gamma)), cv_x = __dmul_rn(gamma, dt);
  NM_LOOP(k, n) {
    const double a0 = a[k];
    double xv = x[k];
    if (flags[k] == 0) {
      const double v0 = v[k];
      const double du = __dadd_rn(__dadd_rn(__dmul_rn(dt, v0), __dmul_rn(cu_a, a0)), __dmul_rn(cu_x, xv));
      u[k] = __dadd_rn(u[k], du);
      v[k] = __dadd_rn(v0, __dadd_rn(__dmul_rn(cv_a, a0), __dmul_rn(cv_x, xv)));
    } else {
      xv = a0;
      x[k] = xv;
    }
    a[k] = xv;
  }
}

}  // namespace dfm

using namespace dfm;

extern "C" {

int dfm_mat_zero_rows(dfm_mat B, const int* flags) {
  if (!B || B->vt != DFM_REAL || (B->N && !flags)) return DFM_ERR_INVALID;
  if (B->N == 0) return DFM_OK;
  const size_t n = (size_t)B->N * B->b;
  k_zero_rows<<<nm_grid(n), kNmThreads, 0, B->ctx->stream>>>(B->N, B->b, B->d_rowptr, flags, B->d_diag, B->d_off);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

int dfm_newmark_residual(dfm_mat B, int scheme, double dt, double gamma, double beta, const double* force,
                         const double* u, const double* v, const double* a, const int* flags, double* t, double* r,
                         double* norm) {
  if (!B || B->vt != DFM_REAL || (scheme != 1 && scheme != 2)) return DFM_ERR_INVALID;
  const size_t n = (size_t)B->N * B->b;
  if (n && (!force || !u || !v || !flags || !t || !r || (scheme == 2 && !a))) return DFM_ERR_INVALID;
  if (t == r || t == u || t == v || t == a || r == u || r == v || r == a) return DFM_ERR_INVALID;
  dfm_ctx c = B->ctx;
  if (n) {
    // the reference's coefficients, as it forms them (host IEEE doubles)
    const double c1 = scheme == 1 ? dt * (1.0 - gamma) : dt;
    const double c2 = scheme == 2 ? (dt * dt) * (0.5 - beta) : 0.0;
    k_nm_predict<<<nm_grid(n), kNmThreads, 0, c->stream>>>(n, scheme, c1, c2, u, v, a, t);
    DFM_CUDA_TRY(cudaGetLastError());
    if (r != force) DFM_CUDA_TRY(cudaMemcpyAsync(r, force, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    int rc = dfm_spmv(B, -1.0, t, 1.0, r);
    if (rc) return rc;
  }
  const int g = nm_grid(std::max<size_t>(n, 1));
  double* part = c->part(6);
  double* res = c->part(7);
  if (n) k_nm_mask_norm<<<g, kNmThreads, 0, c->stream>>>(n, flags, r, part);
  else DFM_CUDA_TRY(cudaMemsetAsync(part, 0, sizeof(double), c->stream));
  k_nm_sum<<<1, 32, 0, c->stream>>>(part, n ? g : 1, res);
  DFM_CUDA_TRY(cudaGetLastError());
  double h = 0.0;
  DFM_CUDA_TRY(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (norm) *norm = std::sqrt(h);
  return DFM_OK;
}

int dfm_newmark_update(dfm_ctx ctx, size_t n, int scheme, double dt, double gamma, double beta, const int* flags,
                       double* x, double* u, double* v, double* a) {
  if (!ctx || (scheme != 1 && scheme != 2)) return DFM_ERR_INVALID;
  if (n && (!flags || !x || !u || !v || (scheme == 2 && !a))) return DFM_ERR_INVALID;
  if (n == 0) return DFM_OK;
  if (scheme == 1)
    k_nm_update1<<<nm_grid(n), kNmThreads, 0, ctx->stream>>>(n, dt, gamma, flags, x, u, v);
  else
    k_nm_update2<<<nm_grid(n), kNmThreads, 0, ctx->stream>>>(n, dt, gamma, beta, flags, x, u, v, a);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

}  // extern "C"
