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
       const int* done, const TX* __restrict__ w, double* __restrict__ part2, const TX* __restrict__ y0) {
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
        if (y0) v += (double)y0[(size_t)i * B + r];
        else if (beta != 0.0) v += beta * (double)y[(size_t)i * B + r];
        const TX out = (TX)v;
        y[(size_t)i * B + r] = out;
        if (NDOT == 1 || NDOT == 2) dacc += (double)w[(size_t)i * B + r] * (double)out;
        if (NDOT == 2) dacc2 += (double)out * (double)out;
        if (NDOT == 3) dacc += (double)out * (double)out;
      }
    }
  }
  if (NDOT >= 1) block_partial<256>(dacc, part);
  if (NDOT == 2) block_partial<256>(dacc2, part2);
}

// Complex b = 1: values and vectors interleaved (re, im).  NDOT: 0 none,
// 1 unconjugated x^T y (re / im partials), 3 |y|^2 (one partial).  TV is the
// value type (double2, or float2 for the mixed-precision solve).
template <int LPR, int NDOT, typename TV>
__global__ void __launch_bounds__(256)
k_zspmv(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
        const TV* __restrict__ diag, const TV* __restrict__ off, double alpha,
        const double2* __restrict__ x, double beta, double2* __restrict__ y, double* __restrict__ part,
        const int* done, const double2* __restrict__ y0) {
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
      TV mv;
      unsigned col;
      if (s < s1) { mv = __ldcs(off + s); col = __ldcs(colind + s); }
      else { mv = diag[i]; col = i; }
      const double2 m = make_double2((double)mv.x, (double)mv.y);
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
      if (y0) { const double2 a = y0[i]; v.x += a.x; v.y += a.y; }
      else if (beta != 0.0) { const double2 yo = y[i]; v.x += beta * yo.x; v.y += beta * yo.y; }
      y[i] = v;
      if (NDOT == 1) {  // unconjugated x^T y (CZVector_Blk operator*, src/matvec/zvector_blk.cpp:39-59)
        const double2 xi = x[i];
        dre += xi.x * v.x - xi.y * v.y;
        dim += xi.x * v.y + xi.y * v.x;
      }
      if (NDOT == 3) dre += v.x * v.x + v.y * v.y;
    }
  }
  if (NDOT >= 1) block_partial<256>(dre, part);
  if (NDOT == 1) block_partial<256>(dim, part + kMaxBlocks);
}

int spmv_grid(dfm_mat A) {
  // grid-stride: 8 blocks of 256 threads per SM keep enough loads in flight
  const int want = A->ctx->nsm * 8;
  return std::max(1, std::min(want, kMaxBlocks));
}

template <int B, int LPR, typename TV>
static void launch_real_tv(dfm_mat A, const TV* diag, const TV* off, int grid, cudaStream_t s, double alpha,
                           const double* x, double beta, double* y, double* part, const int* done,
                           const SpmvOpts& o) {
  const double* w = o.dot_w ? o.dot_w : x;
  if (part && o.yy)
    k_spmv<B, LPR, TV, double, 3><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                       part, done, nullptr, nullptr, o.y0);
  else if (part && o.dot_part2)
    k_spmv<B, LPR, TV, double, 2><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                       part, done, w, o.dot_part2, o.y0);
  else if (part)
    k_spmv<B, LPR, TV, double, 1><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                       part, done, w, nullptr, o.y0);
  else
    k_spmv<B, LPR, TV, double, 0><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                       nullptr, done, nullptr, nullptr, o.y0);
}

template <int B, int LPR>
static void launch_real(dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x, double beta,
                        double* y, double* part, const int* done, const SpmvOpts& o) {
  if (o.f32)
    launch_real_tv<B, LPR, float>(A, A->d_diag32, A->d_off32, grid, s, alpha, x, beta, y, part, done, o);
  else
    launch_real_tv<B, LPR, double>(A, A->d_diag, A->d_off, grid, s, alpha, x, beta, y, part, done, o);
}

template <int B>
static void launch_real_lpr(int lanes, dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x,
                            double beta, double* y, double* part, const int* done, const SpmvOpts& o) {
  switch (lanes) {
    case 4: launch_real<B, 4>(A, grid, s, alpha, x, beta, y, part, done, o); break;
    case 8: launch_real<B, 8>(A, grid, s, alpha, x, beta, y, part, done, o); break;
    case 16: launch_real<B, 16>(A, grid, s, alpha, x, beta, y, part, done, o); break;
    default: launch_real<B, 32>(A, grid, s, alpha, x, beta, y, part, done, o); break;
  }
}

template <int LPR, typename TV>
static void launch_cplx_tv(dfm_mat A, const TV* d, const TV* o, int grid, cudaStream_t s, double alpha,
                           const double* x, double beta, double* y, double* part, const int* done,
                           const SpmvOpts& op) {
  auto* xx = reinterpret_cast<const double2*>(x);
  auto* yy = reinterpret_cast<double2*>(y);
  auto* y0 = reinterpret_cast<const double2*>(op.y0);
  if (part && op.yy)
    k_zspmv<LPR, 3, TV><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, d, o, alpha, xx, beta, yy, part, done,
                                             y0);
  else if (part)
    k_zspmv<LPR, 1, TV><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, d, o, alpha, xx, beta, yy, part, done,
                                             y0);
  else
    k_zspmv<LPR, 0, TV><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, d, o, alpha, xx, beta, yy, nullptr,
                                             done, y0);
}

template <int LPR>
static void launch_cplx(dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x, double beta,
                        double* y, double* part, const int* done, const SpmvOpts& op) {
  if (op.f32)
    launch_cplx_tv<LPR, float2>(A, reinterpret_cast<const float2*>(A->d_diag32),
                                reinterpret_cast<const float2*>(A->d_off32), grid, s, alpha, x, beta, y, part, done,
                                op);
  else
    launch_cplx_tv<LPR, double2>(A, reinterpret_cast<const double2*>(A->d_diag),
                                 reinterpret_cast<const double2*>(A->d_off), grid, s, alpha, x, beta, y, part, done,
                                 op);
}

int spmv_launch(dfm_mat A, double alpha, const double* x, double beta, double* y, double* dot_part,
                int grid, KrylovScalars* sc, int lanes, const SpmvOpts& o) {
  if (A->vt == DFM_COMPLEX && (o.dot_w || o.dot_part2)) return DFM_ERR_UNSUPPORTED;
  if (o.f32 && !A->d_off32) return DFM_ERR_INVALID;
  if (A->N == 0) return DFM_OK;
  cudaStream_t s = A->ctx->stream;
  if (grid <= 0) grid = spmv_grid(A);
  if (lanes <= 0) lanes = A->lanes > 0 ? A->lanes : (A->b == 3 ? 16 : 8);
  const int* done = sc ? &sc->done : nullptr;
  if (A->vt == DFM_COMPLEX) {
    switch (lanes) {
      case 4: launch_cplx<4>(A, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      case 8: launch_cplx<8>(A, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      case 16: launch_cplx<16>(A, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      default: launch_cplx<32>(A, grid, s, alpha, x, beta, y, dot_part, done, o); break;
    }
  } else if (A->b == 1) {
    launch_real_lpr<1>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, o);
  } else if (A->b == 2) {
    launch_real_lpr<2>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, o);
  } else {
    launch_real_lpr<3>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, o);
  }
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

__global__ void k_to_f32(size_t n, const double* __restrict__ in, float* __restrict__ out) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    out[k] = (float)in[k];
}

int to_f32(dfm_ctx c, const double* in, float* out, size_t n) {
  if (n == 0) return DFM_OK;
  const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)c->nsm * 8);
  k_to_f32<<<grid, 256, 0, c->stream>>>(n, in, out);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

// FP32 copy of the values (allocated on first use, refreshed on every call).
int mat_make_f32(dfm_mat A) {
  const size_t nd = (size_t)A->N * A->vw(), no = (size_t)A->ncrs * A->vw();
  if (!A->d_diag32) {
    DFM_CUDA_TRY(cudaMalloc(&A->d_diag32, std::max<size_t>(nd, 1) * sizeof(float)));
    DFM_CUDA_TRY(cudaMalloc(&A->d_off32, std::max<size_t>(no, 1) * sizeof(float)));
  }
  int rc = to_f32(A->ctx, A->d_diag, A->d_diag32, nd);
  if (!rc) rc = to_f32(A->ctx, A->d_off, A->d_off32, no);
  return rc;
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
