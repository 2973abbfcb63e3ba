// ILU(0)-preconditioned CG on the device, LsSol::Solve_PCG
// (src/ls/solver_ls_iter.cpp:100-172), with the reference's stop test
// (recursive residual, |r|^2/|r0|^2 < tol^2) and iteration convention.
//
// One iteration = 5 kernels, all scalars in device memory (KrylovScalars):
//   K1 q = A p, partial (p, q)                     [SpMV + fused dot]
//   K2 alpha = (r,z)/(p,q); r -= alpha q; x += alpha p; partial (r, r);
//      pre-fill the sweep outputs with the sentinel
//   K3 y = L^-1 r   (first: stop if |r|^2/|r0|^2 < tol^2)
//   K4 z = U^-1 y, partial (r, z)
//   K5 beta = (r,z)_new/(r,z); p = beta p + z; it++
// Every reduction is a fixed-order sum of per-block partials, so a solve is
// bit-reproducible run to run.  A CUDA graph of kIterPerGraph iterations is
// replayed until the device sets `done` (converged, maxit, breakdown).
#include <algorithm>
#include <cmath>

#include "dfm_internal.h"

namespace dfm {

constexpr int kIterPerGraph = 16;
constexpr int kVecThreads = 256;

static int vec_grid(dfm_mat A) { return spmv_grid(A); }

__global__ void __launch_bounds__(kVecThreads)
k_pcg_start(size_t n, const double* __restrict__ r, double* __restrict__ x, double* y, double* z, double* part_rr) {
  double acc = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const double rv = r[k];
    acc += rv * rv;
    x[k] = 0.0;
    y[k] = Sent<double>::value();
    z[k] = Sent<double>::value();
  }
  block_partial<kVecThreads>(acc, part_rr);
}

__global__ void __launch_bounds__(kVecThreads)
k_pcg_start2(size_t n, KrylovScalars* sc, const double* part_rr, int np_rr, const double* __restrict__ z,
             double* __restrict__ p) {
  const double rr0 = reduce_partials(part_rr, np_rr);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->it = 0;
    if (rr0 < 1.0e-30) {  // reference: conv_ratio = 0, iteration = 0, return true
      sc->conv = 0.0;
      sc->conv_it = 0;
      sc->done = 100 + DFM_OK;
    } else {
      sc->inv0 = 1.0 / rr0;
      sc->done = 0;
    }
  }
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    p[k] = z[k];
}

__global__ void __launch_bounds__(kVecThreads)
k_pcg_update_xr(size_t n, KrylovScalars* sc, const double* part_pq, int np_pq, const double* part_rz, int np_rz,
                double* part_rr_prev_and_new, int np_rr, double* __restrict__ q_then_z, const double* __restrict__ p,
                double* __restrict__ r, double* __restrict__ x, double* __restrict__ y) {
  if (block_flag(&sc->done)) return;
  if (sc->it >= sc->maxit) {  // reference: loop ends, conv from the last (r, r)
    const double rr = reduce_partials(part_rr_prev_and_new, np_rr);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      sc->conv = sqrt(rr * sc->inv0);
      sc->conv_it = sc->it;
      sc->done = 100 + DFM_NOT_CONVERGED;
    }
    return;
  }
  const double rz = reduce_partials(part_rz, np_rz);
  const double pq = reduce_partials(part_pq, np_pq);
  const double alpha = rz / pq;
  if (!isfinite(alpha)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      sc->conv_it = sc->it;
      sc->conv = NAN;
      sc->done = 100 + DFM_BREAKDOWN;
    }
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->rz = rz;
    sc->alpha = alpha;
  }
  double acc = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const double qv = q_then_z[k];
    const double rv = r[k] - alpha * qv;
    r[k] = rv;
    x[k] += alpha * p[k];
    acc += rv * rv;
    y[k] = Sent<double>::value();
    q_then_z[k] = Sent<double>::value();
  }
  block_partial<kVecThreads>(acc, part_rr_prev_and_new);
}

__global__ void __launch_bounds__(kVecThreads)
k_pcg_update_p(size_t n, KrylovScalars* sc, const double* part_rz, int np_rz, const double* __restrict__ z,
               double* __restrict__ p) {
  if (block_flag(&sc->done)) return;
  const double rz_new = reduce_partials(part_rz, np_rz);
  const double beta = rz_new / sc->rz;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    p[k] = p[k] * beta + z[k];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->beta = beta;
    sc->it = sc->it + 1;
  }
}

// Solve workspace kept on the ILU object: vectors, and the captured graph of
// kIterPerGraph iterations for the (A, M) pair it was built with.
struct PcgPlan {
  dfm_mat A = nullptr;
  double *r = nullptr, *x = nullptr, *p = nullptr, *z = nullptr, *y = nullptr;
  size_t n = 0;
  cudaGraphExec_t exec = nullptr;
  bool graph_failed = false;
};

static PcgPlan* plan_of(dfm_ilu M);

static int enqueue_iteration(dfm_mat A, dfm_ilu M, PcgPlan* P, KrylovScalars* sc) {
  dfm_ctx c = A->ctx;
  const int gv = vec_grid(A);
  const int gs = sweep_grid(M, M->sweep);
  int rc = spmv_launch(A, 1.0, P->p, 0.0, P->z, c->part(0), gv, sc, A->lanes);
  if (rc) return rc;
  k_pcg_update_xr<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(0), gv, c->part(1), gs, c->part(2), gv, P->z,
                                                    P->p, P->r, P->x, P->y);
  DFM_CUDA_TRY(cudaGetLastError());
  rc = ilu_fwd_launch(M, P->r, P->y, sc, M->sweep);
  if (rc) return rc;
  rc = ilu_bwd_launch(M, P->y, P->z, P->r, c->part(1), sc, M->sweep);
  if (rc) return rc;
  k_pcg_update_p<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(1), gs, P->z, P->p);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

int pcg_solve(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit, unsigned* iters,
              double* conv) {
  dfm_ctx c = A->ctx;
  cudaStream_t s = c->stream;
  int rc = spmv_autotune(A);
  if (rc) return rc;
  rc = ilu_autotune(M);
  if (rc) return rc;
  PcgPlan* P = plan_of(M);
  const size_t n = (size_t)A->N * A->xw();
  if (P->n != n) return DFM_ERR_INVALID;
  KrylovScalars* sc = c->d_scal;
  {
    KrylovScalars h = {};
    h.maxit = maxit;
    h.tol2 = tol * tol;
    DFM_CUDA_TRY(cudaMemcpyAsync(sc, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  }
  DFM_CUDA_TRY(cudaMemcpyAsync(P->r, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  const int gv = vec_grid(A);
  const int gs = sweep_grid(M, M->sweep);
  // x = 0; (r, r); z = M^-1 r; p = z; (r, z)
  k_pcg_start<<<gv, kVecThreads, 0, s>>>(n, P->r, P->x, P->y, P->z, c->part(2));
  DFM_CUDA_TRY(cudaGetLastError());
  if ((rc = ilu_fwd_launch(M, P->r, P->y, nullptr, M->sweep))) return rc;
  if ((rc = ilu_bwd_launch(M, P->y, P->z, P->r, c->part(1), nullptr, M->sweep))) return rc;
  k_pcg_start2<<<gv, kVecThreads, 0, s>>>(n, sc, c->part(2), gv, P->z, P->p);
  DFM_CUDA_TRY(cudaGetLastError());

  // capture kIterPerGraph iterations once per plan
  if (!P->exec && !P->graph_failed) {
    cudaGraph_t g = nullptr;
    bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    int erc = DFM_OK;
    if (ok) {
      for (int k = 0; k < kIterPerGraph && erc == DFM_OK; k++) erc = enqueue_iteration(A, M, P, sc);
      ok = (cudaStreamEndCapture(s, &g) == cudaSuccess) && erc == DFM_OK;
    }
    if (ok) ok = cudaGraphInstantiate(&P->exec, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
      P->exec = nullptr;
      P->graph_failed = true;
      cudaGetLastError();  // clear a capture error; fall back to direct launches
    }
  }
  for (;;) {
    if (P->exec) {
      DFM_CUDA_TRY(cudaGraphLaunch(P->exec, s));
    } else {
      for (int k = 0; k < kIterPerGraph; k++)
        if ((rc = enqueue_iteration(A, M, P, sc))) return rc;
    }
    DFM_CUDA_TRY(cudaMemcpyAsync(c->h_scal, sc, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, s));
    DFM_CUDA_TRY(cudaStreamSynchronize(s));
    if (c->h_scal->done) break;
    const int code = take_code(c);
    if (code) return code;
  }
  DFM_CUDA_TRY(cudaMemcpyAsync(x, P->x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  DFM_CUDA_TRY(cudaMemcpyAsync(r, P->r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  {
    const int code = take_code(c);
    if (code) return code;
  }
  const KrylovScalars* h = c->h_scal;
  if (iters) *iters = h->conv_it;
  if (conv) *conv = h->conv;
  return h->done - 100;
}

// -------------------------------------------------------------- plan cache
struct PlanRegistry {
  dfm_ilu M;
  PcgPlan plan;
};
static std::vector<PlanRegistry*>& registry() {
  static std::vector<PlanRegistry*> r;
  return r;
}

static PcgPlan* plan_of(dfm_ilu M) {
  for (auto* e : registry())
    if (e->M == M) return &e->plan;
  auto* e = new PlanRegistry();
  e->M = M;
  PcgPlan& P = e->plan;
  P.A = M->A;
  P.n = (size_t)M->N * M->xw();
  const size_t bytes = std::max<size_t>(P.n, 1) * sizeof(double);
  cudaMalloc(&P.r, bytes);
  cudaMalloc(&P.x, bytes);
  cudaMalloc(&P.p, bytes);
  cudaMalloc(&P.z, bytes);
  cudaMalloc(&P.y, bytes);
  registry().push_back(e);
  return &P;
}

void pcg_release(dfm_ilu M) {
  auto& r = registry();
  for (size_t k = 0; k < r.size(); k++) {
    if (r[k]->M != M) continue;
    PcgPlan& P = r[k]->plan;
    if (P.exec) cudaGraphExecDestroy(P.exec);
    cudaFree(P.r); cudaFree(P.x); cudaFree(P.p); cudaFree(P.z); cudaFree(P.y);
    delete r[k];
    r.erase(r.begin() + k);
    return;
  }
}

}  // namespace dfm
