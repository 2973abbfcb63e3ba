// Block-CRS SpMV, y = beta*y + alpha*A x, for the reference's storage
// (CMatDia_BlkCrs::MatVec, src/matvec/matdia_blkcrs.cpp:921-1094; complex:
// CZMatDia_BlkCrs::MatVec, src/matvec/zmatdia_blkcrs.cpp:737-801).
//
// A group of LPR lanes owns one block row at a time.  Lane j takes the row's
// off-diagonal blocks j, j+LPR, ... and the lane whose turn falls on index
// nnz takes the diagonal block, so a row's contiguous b*b*8-byte blocks are
// read by consecutive lanes (coalesced, streamed with evict-first hints) while
// x is gathered through L1/L2.  Partial products are summed inside the group
// with shuffles; lane 0 writes the b outputs.  Optional fused dots: w.y
// (w = x unless given) and y.y, reduced per block into deterministic
// partial arrays.
#include <algorithm>

#include "dfm_internal.h"

namespace dfm {

template <int B, int LPR, typename TV, typename TX, int NDOT>
__global__ void __launch_bounds__(256)
k_spmv(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
       const TV* __restrict__ diag, const TV* __restrict__ off, double alpha,
       const TX* __restrict__ x, double beta, TX* __restrict__ y, double* __restrict__ part,
       const int* done, const TX* __restrict__ w, double* __restrict__ part2) {
  if (done && block_flag(done)) return;
  constexpr int BB = B * B;
  const int lane = threadIdx.x % LPR;
  const unsigned g0 = (blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const unsigned ng = gridDim.x * blockDim.x / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  double dacc = 0.0, dacc2 = 0.0;
  for (unsigned i = g0; i < N; i += ng) {
    const unsigned s0 = __ldg(rowptr + i), s1 = __ldg(rowptr + i + 1);
    double acc[B];
#pragma unroll
    for (int r = 0; r < B; r++) acc[r] = 0.0;
    for (unsigned s = s0 + lane; s <= s1; s += LPR) {
      const TV* m;
      unsigned col;
      if (s < s1) {
        m = off + (size_t)s * BB;
        col = __ldcs(colind + s);
      } else {
        m = diag + (size_t)i * BB;
        col = i;
      }
      TV mv[BB];
#pragma unroll
      for (int e = 0; e < BB; e++) mv[e] = __ldcs(m + e);
      TX xv[B];
#pragma unroll
      for (int c = 0; c < B; c++) xv[c] = __ldg(x + (size_t)col * B + c);
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int c = 0; c < B; c++) acc[r] += (double)mv[r * B + c] * (double)xv[c];
    }
#pragma unroll
    for (int r = 0; r < B; r++)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
    if (lane == 0) {
#pragma unroll
      for (int r = 0; r < B; r++) {
        double v = alpha * acc[r];
        if (beta != 0.0) v += beta * (double)y[(size_t)i * B + r];
        const TX out = (TX)v;
        y[(size_t)i * B + r] = out;
        if (NDOT >= 1) dacc += (double)w[(size_t)i * B + r] * (double)out;
        if (NDOT >= 2) dacc2 += (double)out * (double)out;
      }
    }
  }
  if (NDOT >= 1) block_partial<256>(dacc, part);
  if (NDOT >= 2) block_partial<256>(dacc2, part2);
}

// Complex b = 1: values and vectors interleaved (re, im).
template <int LPR, bool DOT>
__global__ void __launch_bounds__(256)
k_zspmv(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
        const double2* __restrict__ diag, const double2* __restrict__ off, double alpha,
        const double2* __restrict__ x, double beta, double2* __restrict__ y, double* __restrict__ part,
        const int* done) {
  if (done && block_flag(done)) return;
  const int lane = threadIdx.x % LPR;
  const unsigned g0 = (blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const unsigned ng = gridDim.x * blockDim.x / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  double dre = 0.0, dim = 0.0;
  for (unsigned i = g0; i < N; i += ng) {
    const unsigned s0 = __ldg(rowptr + i), s1 = __ldg(rowptr + i + 1);
    double re = 0.0, im = 0.0;
    for (unsigned s = s0 + lane; s <= s1; s += LPR) {
      double2 m;
      unsigned col;
      if (s < s1) { m = __ldcs(off + s); col = __ldcs(colind + s); }
      else { m = diag[i]; col = i; }
      const double2 xv = __ldg(x + col);
      re += m.x * xv.x - m.y * xv.y;
      im += m.x * xv.y + m.y * xv.x;
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      re += __shfl_xor_sync(gmask, re, o);
      im += __shfl_xor_sync(gmask, im, o);
    }
    if (lane == 0) {
      double2 v = make_double2(alpha * re, alpha * im);
      if (beta != 0.0) { const double2 yo = y[i]; v.x += beta * yo.x; v.y += beta * yo.y; }
      y[i] = v;
      if (DOT) {  // unconjugated x^T y (CZVector_Blk operator*, src/matvec/zvector_blk.cpp:39-59)
        const double2 xi = x[i];
        dre += xi.x * v.x - xi.y * v.y;
        dim += xi.x * v.y + xi.y * v.x;
      }
    }
  }
  if (DOT) {
    block_partial<256>(dre, part);
    block_partial<256>(dim, part + kMaxBlocks);
  }
}

int spmv_grid(dfm_mat A) {
  // grid-stride: 8 blocks of 256 threads per SM keep enough loads in flight
  const int want = A->ctx->nsm * 8;
  return std::max(1, std::min(want, kMaxBlocks));
}

template <int B, int LPR>
static void launch_real(dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x, double beta,
                        double* y, double* part, const int* done, const double* w, double* part2) {
  if (!w) w = x;
  if (part && part2)
    k_spmv<B, LPR, double, double, 2><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, A->d_diag, A->d_off,
                                                           alpha, x, beta, y, part, done, w, part2);
  else if (part)
    k_spmv<B, LPR, double, double, 1><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, A->d_diag, A->d_off,
                                                           alpha, x, beta, y, part, done, w, nullptr);
  else
    k_spmv<B, LPR, double, double, 0><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, A->d_diag, A->d_off,
                                                           alpha, x, beta, y, nullptr, done, nullptr, nullptr);
}

template <int B>
static void launch_real_lpr(int lanes, dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x,
                            double beta, double* y, double* part, const int* done, const double* w,
                            double* part2) {
  switch (lanes) {
    case 4: launch_real<B, 4>(A, grid, s, alpha, x, beta, y, part, done, w, part2); break;
    case 8: launch_real<B, 8>(A, grid, s, alpha, x, beta, y, part, done, w, part2); break;
    case 16: launch_real<B, 16>(A, grid, s, alpha, x, beta, y, part, done, w, part2); break;
    default: launch_real<B, 32>(A, grid, s, alpha, x, beta, y, part, done, w, part2); break;
  }
}

template <int LPR>
static void launch_cplx(dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x, double beta,
                        double* y, double* part, const int* done) {
  auto* d = reinterpret_cast<const double2*>(A->d_diag);
  auto* o = reinterpret_cast<const double2*>(A->d_off);
  auto* xx = reinterpret_cast<const double2*>(x);
  auto* yy = reinterpret_cast<double2*>(y);
  if (part)
    k_zspmv<LPR, true><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, d, o, alpha, xx, beta, yy, part, done);
  else
    k_zspmv<LPR, false><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, d, o, alpha, xx, beta, yy, nullptr,
                                             done);
}

int spmv_launch(dfm_mat A, double alpha, const double* x, double beta, double* y, double* dot_part,
                int grid, KrylovScalars* sc, int lanes, const double* dot_w, double* dot_part2) {
  if (A->vt == DFM_COMPLEX && (dot_w || dot_part2)) return DFM_ERR_UNSUPPORTED;
  if (A->N == 0) return DFM_OK;
  cudaStream_t s = A->ctx->stream;
  if (grid <= 0) grid = spmv_grid(A);
  if (lanes <= 0) lanes = A->lanes > 0 ? A->lanes : (A->b == 3 ? 16 : 8);
  const int* done = sc ? &sc->done : nullptr;
  if (A->vt == DFM_COMPLEX) {
    switch (lanes) {
      case 4: launch_cplx<4>(A, grid, s, alpha, x, beta, y, dot_part, done); break;
      case 8: launch_cplx<8>(A, grid, s, alpha, x, beta, y, dot_part, done); break;
      case 16: launch_cplx<16>(A, grid, s, alpha, x, beta, y, dot_part, done); break;
      default: launch_cplx<32>(A, grid, s, alpha, x, beta, y, dot_part, done); break;
    }
  } else if (A->b == 1) {
    launch_real_lpr<1>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, dot_w, dot_part2);
  } else if (A->b == 2) {
    launch_real_lpr<2>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, dot_w, dot_part2);
  } else {
    launch_real_lpr<3>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, dot_w, dot_part2);
  }
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

// Autotuner: times every lanes-per-row choice on this matrix (CUDA events on
// the context stream, best of 3 after a warm-up) and keeps the fastest.
int spmv_autotune(dfm_mat A) {
  if (A->lanes > 0) return DFM_OK;
  if (A->N == 0) { A->lanes = 8; return DFM_OK; }
  cudaStream_t s = A->ctx->stream;
  const size_t n = (size_t)A->N * A->xw();
  double *x = nullptr, *y = nullptr;
  DFM_CUDA_TRY(cudaMallocAsync(&x, n * sizeof(double), s));
  DFM_CUDA_TRY(cudaMallocAsync(&y, n * sizeof(double), s));
  DFM_CUDA_TRY(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int cand[4] = {4, 8, 16, 32};
  float best = 1e30f;
  int best_l = 8;
  for (int c = 0; c < 4; c++) {
    int rc = spmv_launch(A, 1.0, x, 0.0, y, nullptr, 0, nullptr, cand[c]);
    if (rc) return rc;
    float tmin = 1e30f;
    for (int rep = 0; rep < 3; rep++) {
      cudaEventRecord(e0, s);
      spmv_launch(A, 1.0, x, 0.0, y, nullptr, 0, nullptr, cand[c]);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      tmin = std::min(tmin, ms);
    }
    if (tmin < best) { best = tmin; best_l = cand[c]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(x, s);
  cudaFreeAsync(y, s);
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  A->lanes = best_l;
  return DFM_OK;
}

}  // namespace dfm
