// Rectangular block-CRS matrices (MatVec::CMat_BlkCrs, include/delfem/matvec/
// mat_blkcrs.h:44-190): the couplings between two segments of a linear
// system (CLinearSystem::m_Matrix_NonDia) - nrow x ncol blocks of brow x bcol
// values, every block in the CRS list (no separate diagonal), row-major
// blocks, ascending columns per row.  y = beta y + alpha R x is
// CMat_BlkCrs::MatVec (src/matvec/mat_blkcrs.cpp:955-1175).
//
// A group of LPR lanes takes a block row; lane j multiplies the row's blocks
// j, j + LPR, ... (values and columns read once, streamed past L1), x is
// gathered through L1/L2; the group reduces by shuffles and one lane writes
// the row's brow entries of y.  HBM-bound like the square SpMV.
#include <algorithm>
#include <new>

#include "dfm_internal.h"

struct dfm_rmat_s {
  dfm_ctx ctx = nullptr;
  unsigned nrow = 0, ncol = 0, brow = 1, bcol = 1, nnz = 0;
  unsigned* d_rowptr = nullptr;
  unsigned* d_colind = nullptr;
  double* d_val = nullptr;
};

namespace dfm {

constexpr int kRmThreads = 256;

template <int BR, int BC, int LPR>
__global__ void __launch_bounds__(kRmThreads)
k_rmat_spmv(unsigned nrow, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
            const double* __restrict__ val, double alpha, const double* __restrict__ x, double beta,
            double* __restrict__ y) {
  constexpr int BB = BR * BC;
  const unsigned lane = threadIdx.x % LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  const unsigned groups = (gridDim.x * blockDim.x) / LPR;
  // every lane of a group takes the same rows, so the group's shuffles see all its lanes
  for (unsigned i = (blockIdx.x * blockDim.x + threadIdx.x) / LPR; i < nrow; i += groups) {
    double acc[BR];
#pragma unroll
    for (int r = 0; r < BR; r++) acc[r] = 0.0;
    const unsigned s1 = rowptr[i + 1];
    for (unsigned s = rowptr[i] + lane; s < s1; s += LPR) {
      const size_t j = __ldcs(colind + s);
      const double* m = val + (size_t)s * BB;
      double xv[BC];
#pragma unroll
      for (int c = 0; c < BC; c++) xv[c] = x[j * BC + c];
#pragma unroll
      for (int r = 0; r < BR; r++)
#pragma unroll
        for (int c = 0; c < BC; c++) acc[r] += __ldcs(m + r * BC + c) * xv[c];
    }
#pragma unroll
    for (int r = 0; r < BR; r++)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
    if (lane == 0) {
#pragma unroll
      for (int r = 0; r < BR; r++) {
        const size_t k = (size_t)i * BR + r;
        y[k] = beta == 0.0 ? alpha * acc[r] : beta * y[k] + alpha * acc[r];
      }
    }
  }
}

template <int BR, int BC>
static cudaError_t rmat_launch_bc(dfm_rmat R, double alpha, const double* x, double beta, double* y) {
  const int grid = (int)std::max<size_t>(1, std::min<size_t>(((size_t)R->nrow * 8 + kRmThreads - 1) / kRmThreads,
                                                              (size_t)R->ctx->nsm * 8));
  k_rmat_spmv<BR, BC, 8><<<grid, kRmThreads, 0, R->ctx->stream>>>(R->nrow, R->d_rowptr, R->d_colind, R->d_val,
                                                                    alpha, x, beta, y);
  return cudaGetLastError();
}

template <int BR>
static cudaError_t rmat_launch_br(dfm_rmat R, double alpha, const double* x, double beta, double* y) {
  switch (R->bcol) {
    case 1: return rmat_launch_bc<BR, 1>(R, alpha, x, beta, y);
    case 2: return rmat_launch_bc<BR, 2>(R, alpha, x, beta, y);
    default: return rmat_launch_bc<BR, 3>(R, alpha, x, beta, y);
  }
}

}  // namespace dfm

using namespace dfm;

extern "C" {

int dfm_rmat_create(dfm_ctx ctx, unsigned nrow, unsigned ncol, unsigned brow, unsigned bcol, const unsigned* rowptr,
                    const unsigned* colind, dfm_rmat* out) {
  if (!ctx || !out || brow < 1 || brow > 3 || bcol < 1 || bcol > 3 || !rowptr) return DFM_ERR_INVALID;
  *out = nullptr;
  if (rowptr[0] != 0) return DFM_ERR_INVALID;
  for (unsigned i = 0; i < nrow; i++) {
    if (rowptr[i + 1] < rowptr[i]) return DFM_ERR_INVALID;
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
      if (!colind || colind[s] >= ncol) return DFM_ERR_INVALID;
      if (s > rowptr[i] && colind[s] <= colind[s - 1]) return DFM_ERR_INVALID;  // ascending, no repeats
    }
  }
  dfm_rmat R = new (std::nothrow) dfm_rmat_s();
  if (!R) return DFM_ERR_NOMEM;
  R->ctx = ctx;
  ctx_retain(ctx);
  R->nrow = nrow;
  R->ncol = ncol;
  R->brow = brow;
  R->bcol = bcol;
  R->nnz = rowptr[nrow];
  cudaSetDevice(ctx->device);
  const size_t nval = std::max<size_t>((size_t)R->nnz * brow * bcol, 1);
  int rc = dalloc(&R->d_rowptr, (size_t)nrow + 1);
  if (!rc) rc = dalloc(&R->d_colind, std::max<unsigned>(R->nnz, 1));
  if (!rc) rc = dalloc(&R->d_val, nval);
  if (!rc) rc = copy_in(R->d_rowptr, rowptr, sizeof(unsigned) * (nrow + 1), DFM_HOST, ctx->stream);
  if (!rc && R->nnz) rc = copy_in(R->d_colind, colind, sizeof(unsigned) * R->nnz, DFM_HOST, ctx->stream);
  if (!rc && cudaMemsetAsync(R->d_val, 0, sizeof(double) * nval, ctx->stream) != cudaSuccess) rc = DFM_ERR_CUDA;
  if (rc) {
    dfm_rmat_destroy(R);
    return rc;
  }
  *out = R;
  return DFM_OK;
}

int dfm_rmat_destroy(dfm_rmat R) {
  if (!R) return DFM_OK;
  dfm_ctx ctx = R->ctx;
  cudaStreamSynchronize(R->ctx->stream);
  cudaFree(R->d_rowptr);
  cudaFree(R->d_colind);
  cudaFree(R->d_val);
  delete R;
  ctx_release(ctx);
  return DFM_OK;
}

int dfm_rmat_set_values(dfm_rmat R, const double* val, int where) {
  if (!R || (R->nnz && !val)) return DFM_ERR_INVALID;
  return copy_in(R->d_val, val, sizeof(double) * R->nnz * R->brow * R->bcol, where, R->ctx->stream);
}

int dfm_rmat_spmv(dfm_rmat R, double alpha, const double* x, double beta, double* y) {
  if (!R || (R->nrow && !y) || (R->nnz && !x) || (const double*)y == x) return DFM_ERR_INVALID;
  if (R->nrow == 0) return DFM_OK;
  cudaError_t e;
  switch (R->brow) {
    case 1: e = rmat_launch_br<1>(R, alpha, x, beta, y); break;
    case 2: e = rmat_launch_br<2>(R, alpha, x, beta, y); break;
    default: e = rmat_launch_br<3>(R, alpha, x, beta, y); break;
  }
  DFM_CUDA_TRY(e);
  return DFM_OK;
}

}  // extern "C"
