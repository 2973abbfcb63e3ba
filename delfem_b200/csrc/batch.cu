// Batched ILU(0)-PCG: many independent systems, of uneven sizes, solved
// together.  The instances are stored as one block-diagonal block-CRS matrix
// (instance k owns the block rows [row_off[k], row_off[k+1]) and no entry
// crosses an instance boundary), so the existing matrix, ILU(0) factor and
// level sets serve the whole batch unchanged: the factor of a block-diagonal
// pattern is the per-instance factors, and the level sets of different
// instances interleave, so every sweep advances all instances at once.
//
// Each instance runs its own LsSol::Solve_PCG (src/ls/solver_ls_iter.cpp:
// 100-172): its own alpha, beta, (r, z), stop test and iteration count.  Every
// phase is ONE launch over all instances:
//   per-instance offsets  a chunk table cuts each instance's rows into chunks
//                         (the tile; its size is autotuned); a warp owns a
//                         chunk at a time and writes one partial per chunk
//   per-instance scalars  a warp per instance reduces its chunks' partials in
//                         fixed order (deterministic) and updates the scalars
//   convergence masks     rows of an instance that has stopped are skipped by
//                         the update kernels; its x and r stay frozen
// The ILU sweeps run over the whole batch (the persistent sync-free or level
// schedules).  One iteration = 10 launches, captured as a CUDA graph of
// kBatchIterPerGraph iterations and replayed until every instance has stopped.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "dfm_internal.h"

struct InstScal {
  double rz, inv0, rr, conv, alpha, beta;
  unsigned it, conv_it;
  int status;  // 0 running, else dfm_status + 100
  int pad;
};

struct dfm_batch_s {
  dfm_ctx ctx = nullptr;
  dfm_mat A = nullptr;
  dfm_ilu M = nullptr;
  unsigned ninst = 0;
  std::vector<unsigned> h_row_off;
  // chunk table (rebuilt when the tile size changes)
  int chunk_rows = 0;
  unsigned nch = 0;
  unsigned* d_ch_inst = nullptr;
  unsigned* d_ch_row = nullptr;    // nch + 1 row bounds
  unsigned* d_inst_ch = nullptr;   // ninst + 1 chunk bounds
  double* d_part = nullptr;        // nch partials
  InstScal* d_scal = nullptr;
  InstScal* h_scal = nullptr;      // pinned
  unsigned* d_ndone = nullptr;     // instances stopped
  unsigned* h_ndone = nullptr;     // pinned
  double *r = nullptr, *x = nullptr, *p = nullptr, *z = nullptr, *y = nullptr, *q = nullptr;
  cudaGraphExec_t exec = nullptr;
  int key_sweep = -1, key_lanes = -1, key_chunk = -1;
  unsigned key_gen = ~0u;
  unsigned long long key_wait = 0;
  int lanes = 0;  // SpMV lanes per row for the batch kernels (autotuned)
};

namespace dfm {

constexpr int kBatchIterPerGraph = 8;
constexpr int kBatchThreads = 256;

struct BatchCtl {
  unsigned maxit;
  double tol2;
};
constexpr size_t kCtlOffset = 64;  // BatchCtl's place in the d_ndone allocation

DFM_DEVINL double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

#define WARP_LOOP(c, n)                                                                            \
  for (unsigned c = (blockIdx.x * blockDim.x + threadIdx.x) / 32; c < (n);                         \
       c += gridDim.x * blockDim.x / 32)

// q = A p over the chunks of running instances; partial (p, q) per chunk.
template <int B, int LPR>
__global__ void __launch_bounds__(kBatchThreads)
k_b_spmv(unsigned nch, const unsigned* __restrict__ ch_inst, const unsigned* __restrict__ ch_row,
         const InstScal* __restrict__ sc, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
         const double* __restrict__ diag, const double* __restrict__ off, const double* __restrict__ p,
         double* __restrict__ q, double* __restrict__ part) {
  constexpr int BB = B * B;
  const int lane = threadIdx.x & 31, sub = lane % LPR, grp = lane / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << (grp * LPR));
  WARP_LOOP(c, nch) {
    if (sc[ch_inst[c]].status) {
      if (lane == 0) part[c] = 0.0;
      continue;
    }
    const unsigned r0 = ch_row[c], r1 = ch_row[c + 1];
    double dot = 0.0;
    for (unsigned i = r0 + grp; i < r1; i += 32 / LPR) {
      const unsigned s0 = __ldg(rowptr + i), s1 = __ldg(rowptr + i + 1);
      double acc[B];
#pragma unroll
      for (int r = 0; r < B; r++) acc[r] = 0.0;
      for (unsigned s = s0 + sub; s <= s1; s += LPR) {
        const double* m = (s < s1) ? off + (size_t)s * BB : diag + (size_t)i * BB;
        const unsigned col = (s < s1) ? __ldg(colind + s) : i;
#pragma unroll
        for (int r = 0; r < B; r++)
#pragma unroll
          for (int cc = 0; cc < B; cc++) acc[r] += __ldcs(m + r * B + cc) * __ldg(p + (size_t)col * B + cc);
      }
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
      if (sub == 0)
#pragma unroll
        for (int r = 0; r < B; r++) {
          q[(size_t)i * B + r] = acc[r];
          dot += p[(size_t)i * B + r] * acc[r];
        }
    }
    dot = warp_sum(dot);
    if (lane == 0) part[c] = dot;
  }
}

// Per-instance reduction of the chunk partials (one warp per instance, fixed order).
DFM_DEVINL double inst_sum(const double* part, unsigned c0, unsigned c1, int lane) {
  double v = 0.0;
  for (unsigned c = c0 + lane; c < c1; c += 32) v += part[c];
  return warp_sum(v);
}

// after q = A p: alpha = (r, z) / (p, q); max_iter and breakdown
__global__ void __launch_bounds__(kBatchThreads)
k_b_alpha(unsigned ninst, const unsigned* __restrict__ inst_ch, const double* __restrict__ part, InstScal* sc,
          const BatchCtl* __restrict__ ctl, unsigned* ndone) {
  const int lane = threadIdx.x & 31;
  WARP_LOOP(k, ninst) {
    const double pq = inst_sum(part, inst_ch[k], inst_ch[k + 1], lane);
    if (lane != 0) continue;
    InstScal& s = sc[k];
    if (s.status) continue;
    if (s.it >= ctl->maxit) {
      s.conv = sqrt(s.rr * s.inv0);
      s.conv_it = s.it;
      s.status = 100 + DFM_NOT_CONVERGED;
      atomicAdd(ndone, 1u);
      continue;
    }
    const double a = s.rz / pq;
    if (!isfinite(a)) {
      s.conv = NAN;
      s.conv_it = s.it;
      s.status = 100 + DFM_BREAKDOWN;
      atomicAdd(ndone, 1u);
      continue;
    }
    s.alpha = a;
  }
}

// x += alpha p; r -= alpha q; partial (r, r); sweep outputs to the sentinel (all rows)
template <int B>
__global__ void __launch_bounds__(kBatchThreads)
k_b_update_xr(unsigned nch, const unsigned* __restrict__ ch_inst, const unsigned* __restrict__ ch_row,
              const InstScal* __restrict__ sc, const double* __restrict__ p, const double* __restrict__ q,
              double* __restrict__ r, double* __restrict__ x, double* y, double* z, double* __restrict__ part) {
  const int lane = threadIdx.x & 31;
  WARP_LOOP(c, nch) {
    const InstScal& s = sc[ch_inst[c]];
    const bool run = s.status == 0;
    const double a = s.alpha;
    const size_t k0 = (size_t)ch_row[c] * B, k1 = (size_t)ch_row[c + 1] * B;
    double acc = 0.0;
    for (size_t k = k0 + lane; k < k1; k += 32) {
      if (run) {
        const double rv = r[k] - a * q[k];
        r[k] = rv;
        x[k] += a * p[k];
        acc += rv * rv;
      }
      y[k] = Sent<double>::value();
      z[k] = Sent<double>::value();
    }
    acc = warp_sum(acc);
    if (lane == 0) part[c] = acc;
  }
}

// stop test |r|^2 / |r0|^2 < tol^2 (0-based iteration index, as Solve_PCG)
__global__ void __launch_bounds__(kBatchThreads)
k_b_check(unsigned ninst, const unsigned* __restrict__ inst_ch, const double* __restrict__ part, InstScal* sc,
          const BatchCtl* __restrict__ ctl, unsigned* ndone) {
  const int lane = threadIdx.x & 31;
  WARP_LOOP(k, ninst) {
    const double rr = inst_sum(part, inst_ch[k], inst_ch[k + 1], lane);
    if (lane != 0) continue;
    InstScal& s = sc[k];
    if (s.status) continue;
    s.rr = rr;
    if (rr * s.inv0 < ctl->tol2) {
      s.conv = sqrt(rr * s.inv0);
      s.conv_it = s.it;
      s.status = 100 + DFM_OK;
      atomicAdd(ndone, 1u);
    }
  }
}

// partial (r, z) per chunk of running instances
template <int B>
__global__ void __launch_bounds__(kBatchThreads)
k_b_dot_rz(unsigned nch, const unsigned* __restrict__ ch_inst, const unsigned* __restrict__ ch_row,
           const InstScal* __restrict__ sc, const double* __restrict__ r, const double* __restrict__ z,
           double* __restrict__ part) {
  const int lane = threadIdx.x & 31;
  WARP_LOOP(c, nch) {
    double acc = 0.0;
    if (sc[ch_inst[c]].status == 0) {
      const size_t k0 = (size_t)ch_row[c] * B, k1 = (size_t)ch_row[c + 1] * B;
      for (size_t k = k0 + lane; k < k1; k += 32) acc += r[k] * z[k];
    }
    acc = warp_sum(acc);
    if (lane == 0) part[c] = acc;
  }
}

// beta = (r, z)_new / (r, z); it++   (first = true: only record (r, z))
__global__ void __launch_bounds__(kBatchThreads)
k_b_beta(unsigned ninst, const unsigned* __restrict__ inst_ch, const double* __restrict__ part, InstScal* sc,
         bool first) {
  const int lane = threadIdx.x & 31;
  WARP_LOOP(k, ninst) {
    const double rz = inst_sum(part, inst_ch[k], inst_ch[k + 1], lane);
    if (lane != 0) continue;
    InstScal& s = sc[k];
    if (s.status) continue;
    if (first) {
      s.beta = 0.0;
    } else {
      s.beta = rz / s.rz;
      s.it = s.it + 1;
    }
    s.rz = rz;
  }
}

// p = z + beta p   (first: p = z)
template <int B>
__global__ void __launch_bounds__(kBatchThreads)
k_b_update_p(unsigned nch, const unsigned* __restrict__ ch_inst, const unsigned* __restrict__ ch_row,
             const InstScal* __restrict__ sc, const double* __restrict__ z, double* __restrict__ p, bool first) {
  const int lane = threadIdx.x & 31;
  WARP_LOOP(c, nch) {
    const InstScal& s = sc[ch_inst[c]];
    if (s.status) continue;
    const double b = s.beta;
    const size_t k0 = (size_t)ch_row[c] * B, k1 = (size_t)ch_row[c + 1] * B;
    for (size_t k = k0 + lane; k < k1; k += 32) p[k] = first ? z[k] : p[k] * b + z[k];
  }
}

// start: x = 0, partial (r, r), sentinels
template <int B>
__global__ void __launch_bounds__(kBatchThreads)
k_b_start(unsigned nch, const unsigned* __restrict__ ch_row, const double* __restrict__ r, double* __restrict__ x,
          double* y, double* z, double* __restrict__ part) {
  const int lane = threadIdx.x & 31;
  WARP_LOOP(c, nch) {
    const size_t k0 = (size_t)ch_row[c] * B, k1 = (size_t)ch_row[c + 1] * B;
    double acc = 0.0;
    for (size_t k = k0 + lane; k < k1; k += 32) {
      const double rv = r[k];
      acc += rv * rv;
      x[k] = 0.0;
      y[k] = Sent<double>::value();
      z[k] = Sent<double>::value();
    }
    acc = warp_sum(acc);
    if (lane == 0) part[c] = acc;
  }
}

// rr0 per instance: |r0|^2 < 1e-30 stops at once (conv 0, iteration 0)
__global__ void __launch_bounds__(kBatchThreads)
k_b_start2(unsigned ninst, const unsigned* __restrict__ inst_ch, const double* __restrict__ part, InstScal* sc,
           unsigned* ndone) {
  const int lane = threadIdx.x & 31;
  WARP_LOOP(k, ninst) {
    const double rr0 = inst_sum(part, inst_ch[k], inst_ch[k + 1], lane);
    if (lane != 0) continue;
    InstScal s = {};
    s.rr = rr0;
    if (rr0 < 1.0e-30) {
      s.status = 100 + DFM_OK;
      s.conv = 0.0;
      atomicAdd(ndone, 1u);
    } else {
      s.inv0 = 1.0 / rr0;
    }
    sc[k] = s;
  }
}

static int grid_for(dfm_batch B, unsigned nwarps) {
  const int per_block = kBatchThreads / 32;
  const unsigned want = (nwarps + per_block - 1) / per_block;
  return (int)std::max(1u, std::min<unsigned>(want, (unsigned)B->ctx->nsm * 8));
}

template <int BS, int LPR>
static void launch_b_spmv(dfm_batch B, cudaStream_t s, const double* p, double* q) {
  dfm_mat A = B->A;
  k_b_spmv<BS, LPR><<<grid_for(B, B->nch), kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row, B->d_scal,
                                                                  A->d_rowptr, A->d_colind, A->d_diag, A->d_off, p,
                                                                  q, B->d_part);
}

template <int BS>
static void launch_b_spmv_l(dfm_batch B, cudaStream_t s, int lanes, const double* p, double* q) {
  switch (lanes) {
    case 4: launch_b_spmv<BS, 4>(B, s, p, q); break;
    case 8: launch_b_spmv<BS, 8>(B, s, p, q); break;
    case 16: launch_b_spmv<BS, 16>(B, s, p, q); break;
    default: launch_b_spmv<BS, 32>(B, s, p, q); break;
  }
}

static void launch_spmv_any(dfm_batch B, cudaStream_t s, int lanes, const double* p, double* q) {
  switch (B->A->b) {
    case 1: launch_b_spmv_l<1>(B, s, lanes, p, q); break;
    case 2: launch_b_spmv_l<2>(B, s, lanes, p, q); break;
    default: launch_b_spmv_l<3>(B, s, lanes, p, q); break;
  }
}

template <int BS>
static int enqueue_start_b(dfm_batch B) {
  dfm_ctx c = B->ctx;
  cudaStream_t s = c->stream;
  const int gc = grid_for(B, B->nch), gi = grid_for(B, B->ninst);
  DFM_CUDA_TRY(cudaMemsetAsync(B->d_ndone, 0, sizeof(unsigned), s));
  k_b_start<BS><<<gc, kBatchThreads, 0, s>>>(B->nch, B->d_ch_row, B->r, B->x, B->y, B->z, B->d_part);
  k_b_start2<<<gi, kBatchThreads, 0, s>>>(B->ninst, B->d_inst_ch, B->d_part, B->d_scal, B->d_ndone);
  DFM_CUDA_TRY(cudaGetLastError());
  int rc = ilu_fwd_launch(B->M, B->r, B->y, nullptr, B->M->sweep);
  if (!rc) rc = ilu_bwd_launch(B->M, B->y, B->z, nullptr, nullptr, nullptr, B->M->sweep);
  if (rc) return rc;
  k_b_dot_rz<BS><<<gc, kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row, B->d_scal, B->r, B->z, B->d_part);
  k_b_beta<<<gi, kBatchThreads, 0, s>>>(B->ninst, B->d_inst_ch, B->d_part, B->d_scal, true);
  k_b_update_p<BS><<<gc, kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row, B->d_scal, B->z, B->p, true);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

template <int BS>
static int enqueue_iter_b(dfm_batch B, const BatchCtl* ctl) {
  dfm_ctx c = B->ctx;
  cudaStream_t s = c->stream;
  const int gc = grid_for(B, B->nch), gi = grid_for(B, B->ninst);
  launch_spmv_any(B, s, B->lanes, B->p, B->q);
  k_b_alpha<<<gi, kBatchThreads, 0, s>>>(B->ninst, B->d_inst_ch, B->d_part, B->d_scal, ctl, B->d_ndone);
  k_b_update_xr<BS><<<gc, kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row, B->d_scal, B->p, B->q, B->r,
                                                 B->x, B->y, B->z, B->d_part);
  k_b_check<<<gi, kBatchThreads, 0, s>>>(B->ninst, B->d_inst_ch, B->d_part, B->d_scal, ctl, B->d_ndone);
  DFM_CUDA_TRY(cudaGetLastError());
  int rc = ilu_fwd_launch(B->M, B->r, B->y, nullptr, B->M->sweep);
  if (!rc) rc = ilu_bwd_launch(B->M, B->y, B->z, nullptr, nullptr, nullptr, B->M->sweep);
  if (rc) return rc;
  k_b_dot_rz<BS><<<gc, kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row, B->d_scal, B->r, B->z, B->d_part);
  k_b_beta<<<gi, kBatchThreads, 0, s>>>(B->ninst, B->d_inst_ch, B->d_part, B->d_scal, false);
  k_b_update_p<BS><<<gc, kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row, B->d_scal, B->z, B->p, false);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

static int enqueue_start_any(dfm_batch B) {
  switch (B->A->b) {
    case 1: return enqueue_start_b<1>(B);
    case 2: return enqueue_start_b<2>(B);
    default: return enqueue_start_b<3>(B);
  }
}

static int enqueue_iter_any(dfm_batch B, const BatchCtl* ctl) {
  switch (B->A->b) {
    case 1: return enqueue_iter_b<1>(B, ctl);
    case 2: return enqueue_iter_b<2>(B, ctl);
    default: return enqueue_iter_b<3>(B, ctl);
  }
}

// Chunk table: each instance's rows cut into chunks of at most `rows` block rows.
static int build_chunks(dfm_batch B, int rows) {
  std::vector<unsigned> ch_inst, ch_row, inst_ch(B->ninst + 1, 0);
  for (unsigned k = 0; k < B->ninst; k++) {
    inst_ch[k] = (unsigned)ch_inst.size();
    for (unsigned r = B->h_row_off[k]; r < B->h_row_off[k + 1]; r += (unsigned)rows) {
      ch_inst.push_back(k);
      ch_row.push_back(r);
    }
  }
  inst_ch[B->ninst] = (unsigned)ch_inst.size();
  // row bound array: chunk c spans [ch_row[c], ch_row[c+1]); the end of an
  // instance's last chunk is the next instance's first row (or N)
  std::vector<unsigned> bounds(ch_row.size() + 1);
  // (instances are contiguous, so chunk c ends where chunk c + 1 starts)
  for (size_t c = 0; c < ch_row.size(); c++) bounds[c] = ch_row[c];
  bounds[ch_row.size()] = B->h_row_off[B->ninst];
  cudaFree(B->d_ch_inst);
  cudaFree(B->d_ch_row);
  cudaFree(B->d_inst_ch);
  cudaFree(B->d_part);
  B->d_ch_inst = B->d_ch_row = B->d_inst_ch = nullptr;
  B->d_part = nullptr;
  B->nch = (unsigned)ch_inst.size();
  const size_t nc = std::max<size_t>(B->nch, 1);
  DFM_CUDA_TRY(cudaMalloc(&B->d_ch_inst, nc * sizeof(unsigned)));
  DFM_CUDA_TRY(cudaMalloc(&B->d_ch_row, (nc + 1) * sizeof(unsigned)));
  DFM_CUDA_TRY(cudaMalloc(&B->d_inst_ch, (B->ninst + 1) * sizeof(unsigned)));
  DFM_CUDA_TRY(cudaMalloc(&B->d_part, nc * sizeof(double)));
  cudaStream_t s = B->ctx->stream;
  if (B->nch) {
    DFM_CUDA_TRY(cudaMemcpyAsync(B->d_ch_inst, ch_inst.data(), B->nch * sizeof(unsigned), cudaMemcpyHostToDevice, s));
    DFM_CUDA_TRY(cudaMemcpyAsync(B->d_ch_row, bounds.data(), (B->nch + 1) * sizeof(unsigned), cudaMemcpyHostToDevice,
                                 s));
  }
  DFM_CUDA_TRY(cudaMemcpyAsync(B->d_inst_ch, inst_ch.data(), (B->ninst + 1) * sizeof(unsigned),
                               cudaMemcpyHostToDevice, s));
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  B->chunk_rows = rows;
  return DFM_OK;
}

// Autotuner for the batch kernels: lanes per row of the chunked SpMV and the
// chunk (tile) size, timed together with the chunked (r, z) pass on this
// batch (CUDA events, best of 3 after a warm-up); the fastest pair is kept.
static int batch_autotune(dfm_batch B) {
  if (B->lanes > 0 && B->chunk_rows > 0) return DFM_OK;
  cudaStream_t s = B->ctx->stream;
  DFM_CUDA_TRY(cudaMemsetAsync(B->d_scal, 0, B->ninst * sizeof(InstScal), s));  // all running
  DFM_CUDA_TRY(cudaMemsetAsync(B->p, 0, (size_t)B->A->N * B->A->b * sizeof(double), s));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int lane_c[] = {4, 8, 16, 32};
  const int chunk_c[] = {32, 64, 128, 256, 512};
  float best = 1e30f;
  int bl = 8, bc = 64;
  for (int ch : chunk_c) {
    int rc = build_chunks(B, ch);
    if (rc) return rc;
    for (int ln : lane_c) {
      float tmin = 1e30f;
      for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0, s);
        launch_spmv_any(B, s, ln, B->p, B->q);
        switch (B->A->b) {
          case 1: k_b_dot_rz<1><<<grid_for(B, B->nch), kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row,
                                                                               B->d_scal, B->r, B->q, B->d_part);
            break;
          case 2: k_b_dot_rz<2><<<grid_for(B, B->nch), kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row,
                                                                               B->d_scal, B->r, B->q, B->d_part);
            break;
          default: k_b_dot_rz<3><<<grid_for(B, B->nch), kBatchThreads, 0, s>>>(B->nch, B->d_ch_inst, B->d_ch_row,
                                                                                B->d_scal, B->r, B->q, B->d_part);
            break;
        }
        cudaEventRecord(e1, s);
        DFM_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep) tmin = std::min(tmin, ms);
      }
      DFM_CUDA_TRY(cudaGetLastError());
      if (tmin < best) { best = tmin; bl = ln; bc = ch; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  B->lanes = bl;
  return build_chunks(B, bc);
}

}  // namespace dfm

using namespace dfm;

extern "C" {

int dfm_batch_create(dfm_ilu M, unsigned ninst, const unsigned* row_off, dfm_batch* out) {
  if (!M || !out || !row_off || ninst == 0) return DFM_ERR_INVALID;
  *out = nullptr;
  dfm_mat A = M->A;
  if (A->vt != DFM_REAL) return DFM_ERR_UNSUPPORTED;
  if (row_off[0] != 0 || row_off[ninst] != A->N) return DFM_ERR_INVALID;
  for (unsigned k = 0; k < ninst; k++) {
    if (row_off[k + 1] < row_off[k]) return DFM_ERR_INVALID;
    for (unsigned i = row_off[k]; i < row_off[k + 1]; i++)  // no entry may leave its instance
      for (unsigned s = A->h_rowptr[i]; s < A->h_rowptr[i + 1]; s++)
        if (A->h_colind[s] < row_off[k] || A->h_colind[s] >= row_off[k + 1]) return DFM_ERR_INVALID;
  }
  dfm_batch B = new (std::nothrow) dfm_batch_s();
  if (!B) return DFM_ERR_NOMEM;
  B->ctx = A->ctx;
  B->A = A;
  B->M = M;
  B->ninst = ninst;
  B->h_row_off.assign(row_off, row_off + ninst + 1);
  const size_t n = std::max<size_t>((size_t)A->N * A->b, 1) * sizeof(double);
  int rc = DFM_OK;
  for (double** v : {&B->r, &B->x, &B->p, &B->z, &B->y, &B->q})
    if (!rc && cudaMalloc(v, n) != cudaSuccess) rc = DFM_ERR_NOMEM;
  if (!rc && cudaMalloc(&B->d_scal, ninst * sizeof(InstScal)) != cudaSuccess) rc = DFM_ERR_NOMEM;
  // d_ndone: the stopped-instance counter at offset 0, the BatchCtl at kCtlOffset
  if (!rc && cudaMalloc(&B->d_ndone, kCtlOffset + sizeof(BatchCtl)) != cudaSuccess) rc = DFM_ERR_NOMEM;
  if (!rc && cudaMallocHost((void**)&B->h_scal, ninst * sizeof(InstScal)) != cudaSuccess) rc = DFM_ERR_NOMEM;
  if (!rc && cudaMallocHost((void**)&B->h_ndone, sizeof(unsigned)) != cudaSuccess) rc = DFM_ERR_NOMEM;
  if (rc) {
    cudaGetLastError();
    dfm_batch_destroy(B);
    return rc;
  }
  *out = B;
  return DFM_OK;
}

int dfm_batch_destroy(dfm_batch B) {
  if (!B) return DFM_OK;
  cudaStreamSynchronize(B->ctx->stream);
  if (B->exec) cudaGraphExecDestroy(B->exec);
  for (double* v : {B->r, B->x, B->p, B->z, B->y, B->q}) cudaFree(v);
  cudaFree(B->d_ch_inst);
  cudaFree(B->d_ch_row);
  cudaFree(B->d_inst_ch);
  cudaFree(B->d_part);
  cudaFree(B->d_scal);
  cudaFree(B->d_ndone);
  if (B->h_scal) cudaFreeHost(B->h_scal);
  if (B->h_ndone) cudaFreeHost(B->h_ndone);
  delete B;
  return DFM_OK;
}

int dfm_batch_set_tuning(dfm_batch B, int lanes, int chunk_rows) {
  if (!B || (lanes != 0 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) || chunk_rows < 0 ||
      chunk_rows > (1 << 20))
    return DFM_ERR_INVALID;
  B->lanes = lanes;
  if (lanes == 0 || chunk_rows == 0) {
    B->chunk_rows = 0;
    return DFM_OK;
  }
  return build_chunks(B, chunk_rows);
}

int dfm_batch_get_tuning(dfm_batch B, int* lanes, int* chunk_rows) {
  if (!B) return DFM_ERR_INVALID;
  if (lanes) *lanes = B->lanes;
  if (chunk_rows) *chunk_rows = B->chunk_rows;
  return DFM_OK;
}

int dfm_batch_solve_pcg(dfm_batch B, const double* b, int b_where, double* x, int x_where, double tol,
                        unsigned maxit, unsigned* iters, double* conv, int* status) {
  if (!B || !b || !x || !B->M->factored) return DFM_ERR_INVALID;
  dfm_ctx c = B->ctx;
  cudaStream_t s = c->stream;
  const size_t n = (size_t)B->A->N * B->A->b;
  int rc = ilu_autotune(B->M);
  if (!rc) rc = ilu_prepare(B->M, false);
  if (!rc) rc = batch_autotune(B);
  if (rc) return rc;
  BatchCtl* d_ctl = reinterpret_cast<BatchCtl*>(reinterpret_cast<char*>(B->d_ndone) + kCtlOffset);
  {
    BatchCtl h = {maxit, tol * tol};
    DFM_CUDA_TRY(cudaMemcpyAsync(d_ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  }
  DFM_CUDA_TRY(cudaMemcpyAsync(B->r, b, n * sizeof(double),
                               b_where == DFM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  if ((rc = enqueue_start_any(B))) return rc;
  const bool same = B->exec && B->key_sweep == B->M->sweep && B->key_lanes == B->lanes &&
                    B->key_chunk == B->chunk_rows && B->key_gen == B->M->plan_gen && B->key_wait == c->wait_ns;
  if (!same) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
    cudaGraph_t g = nullptr;
    bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    int erc = DFM_OK;
    if (ok) {
      for (int k = 0; k < kBatchIterPerGraph && !erc; k++) erc = enqueue_iter_any(B, d_ctl);
      ok = cudaStreamEndCapture(s, &g) == cudaSuccess && !erc;
    }
    if (ok) ok = cudaGraphInstantiate(&B->exec, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
      B->exec = nullptr;
      cudaGetLastError();
    }
    B->key_sweep = B->M->sweep;
    B->key_lanes = B->lanes;
    B->key_chunk = B->chunk_rows;
    B->key_gen = B->M->plan_gen;
    B->key_wait = c->wait_ns;
  }
  for (;;) {
    if (B->exec) {
      DFM_CUDA_TRY(cudaGraphLaunch(B->exec, s));
    } else {
      for (int k = 0; k < kBatchIterPerGraph; k++)
        if ((rc = enqueue_iter_any(B, d_ctl))) return rc;
    }
    DFM_CUDA_TRY(cudaMemcpyAsync(B->h_ndone, B->d_ndone, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    DFM_CUDA_TRY(cudaStreamSynchronize(s));
    const int code = take_code(c);
    if (code) return code;
    if (*B->h_ndone >= B->ninst) break;
  }
  DFM_CUDA_TRY(cudaMemcpyAsync(x, B->x, n * sizeof(double),
                               x_where == DFM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
  DFM_CUDA_TRY(cudaMemcpyAsync(B->h_scal, B->d_scal, B->ninst * sizeof(InstScal), cudaMemcpyDeviceToHost, s));
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  int worst = DFM_OK;
  for (unsigned k = 0; k < B->ninst; k++) {
    const InstScal& h = B->h_scal[k];
    const int st = h.status - 100;
    if (iters) iters[k] = h.conv_it;
    if (conv) conv[k] = h.conv;
    if (status) status[k] = st;
    if (st == DFM_BREAKDOWN) worst = DFM_BREAKDOWN;
    else if (st == DFM_NOT_CONVERGED && worst == DFM_OK) worst = DFM_NOT_CONVERGED;
  }
  return worst;
}

}  // extern "C"
