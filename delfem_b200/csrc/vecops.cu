// Vector operations of MatVec::CVector_Blk on device arrays, as
// LsSol::CLinearSystem exposes them to the solvers through its integer
// handles (DOT / COPY / SCAL / AXPY, src/ls/linearsystem.cpp:298-415, over
// src/matvec/vector_blk.cpp:37-112).  A caller that drives its own Krylov
// loop through the reference's solver interface (the C++ adapter
// dfm_delfem::CLinearSystemGPU) runs each step here.
//
// The dot product is deterministic: a fixed grid of blocks writes one partial
// each (fixed order inside a block), one warp sums the partials in order.
// Elementwise operations are streaming, one double per thread per step, and
// bit-identical to the reference's loops.
#include <algorithm>

#include "dfm_internal.h"

namespace dfm {

constexpr int kVecOpThreads = 256;

static int vecop_grid(size_t n) {
  const size_t g = (n + kVecOpThreads - 1) / kVecOpThreads;
  return (int)std::max<size_t>(1, std::min<size_t>(g, (size_t)kMaxBlocks));
}

#define VEC_LOOP(k, n) \
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (n); k += (size_t)gridDim.x * blockDim.x)

__global__ void __launch_bounds__(kVecOpThreads)
k_vec_dot(size_t n, const double* __restrict__ x, const double* __restrict__ y, double* part) {
  double acc = 0.0;
  VEC_LOOP(k, n) acc += x[k] * y[k];
  block_partial<kVecOpThreads>(acc, part);
}

__global__ void k_vec_dot_final(const double* part, int np, double* out) {
  const double s = reduce_partials(part, np);
  if (threadIdx.x == 0) *out = s;
}

// y += alpha x   (CVector_Blk::AXPY: the product rounded, then the sum - no
// fused multiply-add, as the reference computes it)
__global__ void __launch_bounds__(kVecOpThreads)
k_vec_axpy(size_t n, double alpha, const double* __restrict__ x, double* __restrict__ y) {
  VEC_LOOP(k, n) y[k] = __dadd_rn(y[k], __dmul_rn(alpha, x[k]));
}

// x *= alpha   (CVector_Blk::operator*=: a product, so NaN * 0 stays NaN)
__global__ void __launch_bounds__(kVecOpThreads) k_vec_scal(size_t n, double alpha, double* __restrict__ x) {
  VEC_LOOP(k, n) x[k] = __dmul_rn(x[k], alpha);
}

// y[i] := x[idx[i]] block by block (b doubles per block): a vector into or
// out of a block ordering (COrdering_Blk::OrderingVector_OldToNew / _NewToOld)
__global__ void __launch_bounds__(kVecOpThreads)
k_vec_gather(size_t nblk, unsigned b, const unsigned* __restrict__ idx, const double* __restrict__ x,
             double* __restrict__ y) {
  VEC_LOOP(k, nblk * b) y[k] = x[(size_t)idx[k / b] * b + k % b];
}

}  // namespace dfm

using namespace dfm;

extern "C" {

int dfm_vec_dot(dfm_ctx ctx, size_t n, const double* x, const double* y, double* out) {
  if (!ctx || !out || (n && (!x || !y))) return DFM_ERR_INVALID;
  if (n == 0) {
    *out = 0.0;
    return DFM_OK;
  }
  const int g = vecop_grid(n);
  double* part = ctx->part(6);
  double* res = ctx->part(7);
  k_vec_dot<<<g, kVecOpThreads, 0, ctx->stream>>>(n, x, y, part);
  k_vec_dot_final<<<1, 32, 0, ctx->stream>>>(part, g, res);
  DFM_CUDA_TRY(cudaGetLastError());
  double h = 0.0;
  DFM_CUDA_TRY(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = h;
  return DFM_OK;
}

int dfm_vec_axpy(dfm_ctx ctx, size_t n, double alpha, const double* x, double* y) {
  if (!ctx || (n && (!x || !y))) return DFM_ERR_INVALID;
  if (n == 0) return DFM_OK;
  k_vec_axpy<<<vecop_grid(n), kVecOpThreads, 0, ctx->stream>>>(n, alpha, x, y);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

int dfm_vec_scal(dfm_ctx ctx, size_t n, double alpha, double* x) {
  if (!ctx || (n && !x)) return DFM_ERR_INVALID;
  if (n == 0) return DFM_OK;
  k_vec_scal<<<vecop_grid(n), kVecOpThreads, 0, ctx->stream>>>(n, alpha, x);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

int dfm_vec_gather(dfm_ctx ctx, size_t nblk, unsigned b, const unsigned* idx, const double* x, double* y) {
  if (!ctx || b < 1 || (nblk && (!idx || !x || !y)) || (const double*)y == x) return DFM_ERR_INVALID;
  if (nblk == 0) return DFM_OK;
  k_vec_gather<<<vecop_grid(nblk * b), kVecOpThreads, 0, ctx->stream>>>(nblk, b, idx, x, y);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

int dfm_vec_copy(dfm_ctx ctx, size_t n, const double* x, double* y) {
  if (!ctx || (n && (!x || !y))) return DFM_ERR_INVALID;
  if (n == 0 || x == y) return DFM_OK;
  DFM_CUDA_TRY(cudaMemcpyAsync(y, x, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  return DFM_OK;
}

}  // extern "C"
