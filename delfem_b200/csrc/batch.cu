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
//
// A second schedule solves the batch in ONE persistent launch: every CTA
// takes instances from a queue (largest first) and runs an instance's whole
// PCG on its own - SpMV, level-by-level ILU sweeps over the instance's own
// level sets (a __syncthreads per level), block reductions in fixed order -
// so thousands of small solves proceed side by side with no grid-wide
// synchronisation.  The autotuner times both schedules (and the CTA size and
// lanes per row of the second) on the batch and keeps the faster.
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
  // persistent CTA-per-instance schedule
  int schedule = 0;           // 0 untuned, 1 graph of phases, 2 persistent CTA per instance
  int cta_threads = 0, cta_lanes = 0;
  unsigned* d_bord_f = nullptr;   // per-instance rows by forward level (instance k at row_off[k])
  unsigned* d_bord_b = nullptr;
  unsigned* d_blv_f = nullptr;    // concatenated per-instance level pointers (absolute positions)
  unsigned* d_blv_b = nullptr;
  unsigned* d_blvo_f = nullptr;   // ninst + 1 offsets into d_blv_f
  unsigned* d_blvo_b = nullptr;
  unsigned* d_queue = nullptr;    // instances, largest first
  unsigned* d_row_off = nullptr;  // ninst + 1
  unsigned* d_next = nullptr;     // queue head
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

// ------------------------------------------- persistent CTA-per-instance
struct CtaArgs {
  unsigned ninst;
  const unsigned* queue;
  unsigned* next;
  const unsigned* row_off;
  const unsigned *rowptr, *colind, *diaind;
  const double *diag, *off, *fdiag, *foff;
  const unsigned *ord_f, *ord_b, *lv_f, *lv_b, *lvo_f, *lvo_b;
  double *r, *x, *p, *z, *q;
  InstScal* sc;
  unsigned* ndone;
  const BatchCtl* ctl;
};

template <int NT>
DFM_DEVINL double cta_sum(double v, double* s_w) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();  // s_w free
  if (l == 0) s_w[w] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < NT / 32; k++) t += s_w[k];  // every thread, same fixed order
  return t;
}

// rows [ord[a], ...) of one level of one sweep; FWD: y_i = D^-1 (in_i - L y),
// BWD: z_i = in_i - (D^-1 U) z
template <int B, int LPR, bool FWD>
DFM_DEVINL void cta_sweep(const CtaArgs& A, unsigned k, const double* in, double* out) {
  constexpr int BB = B * B;
  const int lane = threadIdx.x % LPR;
  const unsigned g = threadIdx.x / LPR, ng = blockDim.x / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  const unsigned* ord = FWD ? A.ord_f : A.ord_b;
  const unsigned* lv = (FWD ? A.lv_f : A.lv_b) + (FWD ? A.lvo_f[k] : A.lvo_b[k]);
  const unsigned nlev = (FWD ? A.lvo_f[k + 1] - A.lvo_f[k] : A.lvo_b[k + 1] - A.lvo_b[k]) - 1;
  for (unsigned l = 0; l < nlev; l++) {
    const unsigned p0 = lv[l], p1 = lv[l + 1];
    for (unsigned pb = p0; pb < p1; pb += ng) {
      const unsigned pp = pb + g;
      const bool valid = pp < p1;  // uniform within a group
      unsigned i = 0, s0 = 0, s1 = 0;
      if (valid) {
        i = __ldg(ord + pp);
        if (FWD) { s0 = __ldg(A.rowptr + i); s1 = __ldg(A.diaind + i); }
        else { s0 = __ldg(A.diaind + i); s1 = __ldg(A.rowptr + i + 1); }
      }
      double acc[B];
#pragma unroll
      for (int r = 0; r < B; r++) acc[r] = 0.0;
      for (unsigned s = s0 + lane; s < s1; s += LPR) {
        const unsigned col = __ldg(A.colind + s);
        const double* m = A.foff + (size_t)s * BB;
#pragma unroll
        for (int r = 0; r < B; r++)
#pragma unroll
          for (int c = 0; c < B; c++) acc[r] += __ldg(m + r * B + c) * out[(size_t)col * B + c];
      }
      if (LPR > 1)
#pragma unroll
        for (int r = 0; r < B; r++)
#pragma unroll
          for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
      if (valid && lane == 0) {
        double t[B];
#pragma unroll
        for (int r = 0; r < B; r++) t[r] = in[(size_t)i * B + r] - acc[r];
        if (FWD) {
          const double* d = A.fdiag + (size_t)i * BB;
#pragma unroll
          for (int r = 0; r < B; r++) {
            double v = 0.0;
#pragma unroll
            for (int c = 0; c < B; c++) v += __ldg(d + r * B + c) * t[c];
            out[(size_t)i * B + r] = v;
          }
        } else {
#pragma unroll
          for (int r = 0; r < B; r++) out[(size_t)i * B + r] = t[r];
        }
      }
    }
    __syncthreads();  // level done
  }
}

template <int B, int LPR, int NT>
__global__ void __launch_bounds__(NT)
k_batch_cta(CtaArgs A) {
  constexpr int BB = B * B;
  __shared__ double s_w[NT / 32];
  __shared__ unsigned s_k;
  const int lane = threadIdx.x % LPR;
  const unsigned g = threadIdx.x / LPR, ng = NT / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  const unsigned maxit = A.ctl->maxit;
  const double tol2 = A.ctl->tol2;
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned t = atomicAdd(A.next, 1u);
      s_k = t < A.ninst ? A.queue[t] : 0xffffffffu;
    }
    __syncthreads();
    const unsigned k = s_k;
    __syncthreads();
    if (k == 0xffffffffu) break;
    const unsigned r0 = A.row_off[k], r1 = A.row_off[k + 1];
    const size_t e0 = (size_t)r0 * B, e1 = (size_t)r1 * B;
    double* r = A.r;
    double* x = A.x;
    double* p = A.p;
    double* z = A.z;
    double* q = A.q;  // holds y = L^-1 r during the preconditioner
    // x = 0, (r, r)
    double acc = 0.0;
    for (size_t e = e0 + threadIdx.x; e < e1; e += NT) {
      x[e] = 0.0;
      acc += r[e] * r[e];
    }
    const double rr0 = cta_sum<NT>(acc, s_w);
    InstScal res = {};
    if (rr0 < 1.0e-30) {
      res.status = 100 + DFM_OK;
    } else {
      const double inv0 = 1.0 / rr0;
      res.inv0 = inv0;
      __syncthreads();
      cta_sweep<B, LPR, true>(A, k, r, q);
      cta_sweep<B, LPR, false>(A, k, q, z);
      acc = 0.0;
      for (size_t e = e0 + threadIdx.x; e < e1; e += NT) {
        p[e] = z[e];
        acc += r[e] * z[e];
      }
      double rz = cta_sum<NT>(acc, s_w);
      double rr = rr0;
      unsigned it = 0;
      for (;; it++) {
        if (it >= maxit) {
          res.status = 100 + DFM_NOT_CONVERGED;
          res.conv = sqrt(rr * inv0);
          break;
        }
        // q = A p, (p, q)
        acc = 0.0;
        for (unsigned i = r0 + g; i < r1; i += ng) {
          const unsigned s0 = __ldg(A.rowptr + i), s1 = __ldg(A.rowptr + i + 1);
          double a[B];
#pragma unroll
          for (int rr_ = 0; rr_ < B; rr_++) a[rr_] = 0.0;
          for (unsigned s = s0 + lane; s <= s1; s += LPR) {
            const double* m = (s < s1) ? A.off + (size_t)s * BB : A.diag + (size_t)i * BB;
            const unsigned col = (s < s1) ? __ldg(A.colind + s) : i;
#pragma unroll
            for (int rr_ = 0; rr_ < B; rr_++)
#pragma unroll
              for (int c = 0; c < B; c++) a[rr_] += __ldg(m + rr_ * B + c) * p[(size_t)col * B + c];
          }
          if (LPR > 1)
#pragma unroll
            for (int rr_ = 0; rr_ < B; rr_++)
#pragma unroll
              for (int o = LPR / 2; o > 0; o >>= 1) a[rr_] += __shfl_xor_sync(gmask, a[rr_], o);
          if (lane == 0)
#pragma unroll
            for (int rr_ = 0; rr_ < B; rr_++) {
              q[(size_t)i * B + rr_] = a[rr_];
              acc += p[(size_t)i * B + rr_] * a[rr_];
            }
        }
        const double pq = cta_sum<NT>(acc, s_w);
        const double alpha = rz / pq;
        if (!isfinite(alpha)) {
          res.status = 100 + DFM_BREAKDOWN;
          res.conv = NAN;
          break;
        }
        acc = 0.0;
        for (size_t e = e0 + threadIdx.x; e < e1; e += NT) {
          x[e] += alpha * p[e];
          const double rv = r[e] - alpha * q[e];
          r[e] = rv;
          acc += rv * rv;
        }
        rr = cta_sum<NT>(acc, s_w);
        if (rr * inv0 < tol2) {
          res.status = 100 + DFM_OK;
          res.conv = sqrt(rr * inv0);
          break;
        }
        cta_sweep<B, LPR, true>(A, k, r, q);
        cta_sweep<B, LPR, false>(A, k, q, z);
        acc = 0.0;
        for (size_t e = e0 + threadIdx.x; e < e1; e += NT) acc += r[e] * z[e];
        const double rz_new = cta_sum<NT>(acc, s_w);
        const double beta = rz_new / rz;
        rz = rz_new;
        for (size_t e = e0 + threadIdx.x; e < e1; e += NT) p[e] = p[e] * beta + z[e];
        __syncthreads();
      }
      res.it = it;
      res.conv_it = it;
      res.rz = rz;
      res.rr = rr;
    }
    if (threadIdx.x == 0) {
      A.sc[k] = res;
      atomicAdd(A.ndone, 1u);
    }
    __syncthreads();
  }
}

// Per-instance level-ordered rows and level pointers from the global level
// sets (an instance's levels are its own: no entry leaves the instance).
static int build_cta_tables(dfm_batch B) {
  dfm_ilu M = B->M;
  const unsigned N = M->N;
  std::vector<unsigned> ord_f(N), ord_b(N), lv_f, lv_b, lvo_f(B->ninst + 1), lvo_b(B->ninst + 1);
  std::vector<unsigned> cnt;
  for (int f = 0; f < 2; f++) {
    const std::vector<unsigned>& lev = f ? M->lev_b : M->lev_f;
    std::vector<unsigned>& ord = f ? ord_b : ord_f;
    std::vector<unsigned>& lv = f ? lv_b : lv_f;
    std::vector<unsigned>& lvo = f ? lvo_b : lvo_f;
    for (unsigned k = 0; k < B->ninst; k++) {
      const unsigned r0 = B->h_row_off[k], r1 = B->h_row_off[k + 1];
      unsigned nl = 0;
      for (unsigned i = r0; i < r1; i++) nl = std::max(nl, lev[i] + 1);
      cnt.assign(nl + 1, 0);
      for (unsigned i = r0; i < r1; i++) cnt[lev[i] + 1]++;
      for (unsigned l = 0; l < nl; l++) cnt[l + 1] += cnt[l];
      lvo[k] = (unsigned)lv.size();
      for (unsigned l = 0; l <= nl; l++) lv.push_back(r0 + cnt[l]);
      for (unsigned i = r0; i < r1; i++) ord[r0 + cnt[lev[i]]++] = i;  // ascending row within a level
    }
    lvo[B->ninst] = (unsigned)lv.size();
  }
  std::vector<unsigned> queue(B->ninst);
  for (unsigned k = 0; k < B->ninst; k++) queue[k] = k;
  std::stable_sort(queue.begin(), queue.end(), [&](unsigned a, unsigned b) {
    return B->h_row_off[a + 1] - B->h_row_off[a] > B->h_row_off[b + 1] - B->h_row_off[b];
  });
  cudaStream_t s = B->ctx->stream;
  auto up = [&](unsigned** d, const std::vector<unsigned>& h) -> int {
    DFM_CUDA_TRY(cudaMalloc(d, std::max<size_t>(h.size(), 1) * sizeof(unsigned)));
    if (!h.empty())
      DFM_CUDA_TRY(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(unsigned), cudaMemcpyHostToDevice, s));
    return DFM_OK;
  };
  int rc = up(&B->d_bord_f, ord_f);
  if (!rc) rc = up(&B->d_bord_b, ord_b);
  if (!rc) rc = up(&B->d_blv_f, lv_f);
  if (!rc) rc = up(&B->d_blv_b, lv_b);
  if (!rc) rc = up(&B->d_blvo_f, lvo_f);
  if (!rc) rc = up(&B->d_blvo_b, lvo_b);
  if (!rc) rc = up(&B->d_queue, queue);
  if (!rc) DFM_CUDA_TRY(cudaMalloc(&B->d_next, sizeof(unsigned)));
  if (!rc) DFM_CUDA_TRY(cudaStreamSynchronize(s));
  return rc;
}

template <int BS, int LPR, int NT>
static cudaError_t launch_cta_t(dfm_batch B, const CtaArgs& a) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_cta<BS, LPR, NT>, NT, 0);
  const int grid = std::max(1, std::min<int>((int)B->ninst, B->ctx->nsm * std::max(per_sm, 1)));
  k_batch_cta<BS, LPR, NT><<<grid, NT, 0, B->ctx->stream>>>(a);
  return cudaGetLastError();
}

template <int BS, int NT>
static cudaError_t launch_cta_l(dfm_batch B, const CtaArgs& a, int lanes) {
  switch (lanes) {
    case 2: return launch_cta_t<BS, 2, NT>(B, a);
    case 4: return launch_cta_t<BS, 4, NT>(B, a);
    default: return launch_cta_t<BS, 8, NT>(B, a);
  }
}

template <int BS>
static cudaError_t launch_cta_n(dfm_batch B, const CtaArgs& a, int threads, int lanes) {
  switch (threads) {
    case 256: return launch_cta_l<BS, 256>(B, a, lanes);
    case 512: return launch_cta_l<BS, 512>(B, a, lanes);
    default: return launch_cta_l<BS, 1024>(B, a, lanes);
  }
}

// One persistent launch solves the whole batch (b already in B->r).
static int run_cta(dfm_batch B, const BatchCtl* d_ctl, int threads, int lanes) {
  if (!B->d_bord_f) {
    int rc = build_cta_tables(B);
    if (rc) return rc;
  }
  cudaStream_t s = B->ctx->stream;
  DFM_CUDA_TRY(cudaMemsetAsync(B->d_next, 0, sizeof(unsigned), s));
  DFM_CUDA_TRY(cudaMemsetAsync(B->d_ndone, 0, sizeof(unsigned), s));
  CtaArgs a;
  a.ninst = B->ninst;
  a.queue = B->d_queue;
  a.next = B->d_next;
  a.row_off = B->d_row_off;
  a.rowptr = B->A->d_rowptr;
  a.colind = B->A->d_colind;
  a.diaind = B->M->d_diaind;
  a.diag = B->A->d_diag;
  a.off = B->A->d_off;
  a.fdiag = B->M->d_fdiag;
  a.foff = B->M->d_foff;
  a.ord_f = B->d_bord_f;
  a.ord_b = B->d_bord_b;
  a.lv_f = B->d_blv_f;
  a.lv_b = B->d_blv_b;
  a.lvo_f = B->d_blvo_f;
  a.lvo_b = B->d_blvo_b;
  a.r = B->r;
  a.x = B->x;
  a.p = B->p;
  a.z = B->z;
  a.q = B->q;
  a.sc = B->d_scal;
  a.ndone = B->d_ndone;
  a.ctl = d_ctl;
  cudaError_t e;
  switch (B->A->b) {
    case 1: e = launch_cta_n<1>(B, a, threads, lanes); break;
    case 2: e = launch_cta_n<2>(B, a, threads, lanes); break;
    default: e = launch_cta_n<3>(B, a, threads, lanes); break;
  }
  DFM_CUDA_TRY(e);
  return DFM_OK;
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
  if (A->vt != DFM_REAL || M->fillpat) return DFM_ERR_UNSUPPORTED;  // batches use ILU(0)
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
  ctx_retain(B->ctx);
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
  if (!rc && cudaMalloc(&B->d_row_off, (ninst + 1) * sizeof(unsigned)) != cudaSuccess) rc = DFM_ERR_NOMEM;
  if (!rc && cudaMemcpy(B->d_row_off, row_off, (ninst + 1) * sizeof(unsigned), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = DFM_ERR_CUDA;
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
  for (unsigned* v : {B->d_bord_f, B->d_bord_b, B->d_blv_f, B->d_blv_b, B->d_blvo_f, B->d_blvo_b, B->d_queue,
                      B->d_next, B->d_row_off})
    cudaFree(v);
  if (B->h_scal) cudaFreeHost(B->h_scal);
  if (B->h_ndone) cudaFreeHost(B->h_ndone);
  dfm_ctx c = B->ctx;
  delete B;
  ctx_release(c);
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

// Runs the graph-of-phases schedule to the end (b already in B->r).
static int run_phases(dfm_batch B, const BatchCtl* d_ctl) {
  dfm_ctx c = B->ctx;
  cudaStream_t s = c->stream;
  int rc = enqueue_start_any(B);
  if (rc) return rc;
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
  return DFM_OK;
}

static int run_schedule(dfm_batch B, const BatchCtl* d_ctl, int schedule, int threads, int lanes) {
  if (schedule == 2) {
    int rc = run_cta(B, d_ctl, threads, lanes);
    if (rc) return rc;
    DFM_CUDA_TRY(cudaStreamSynchronize(B->ctx->stream));
    return take_code(B->ctx);
  }
  return run_phases(B, d_ctl);
}

static int set_ctl(dfm_batch B, BatchCtl* d_ctl, unsigned maxit, double tol) {
  BatchCtl h = {maxit, tol * tol};
  DFM_CUDA_TRY(cudaMemcpyAsync(d_ctl, &h, sizeof(h), cudaMemcpyHostToDevice, B->ctx->stream));
  return DFM_OK;
}

// Schedule autotuner: the graph of phases and the persistent CTA-per-instance
// kernel (CTA sizes 256 / 512 / 1024, 2 / 4 / 8 lanes per row) each run the
// batch for a few iterations from b; the fastest is kept.
static int schedule_autotune(dfm_batch B, BatchCtl* d_ctl, const double* b, int b_where, double tol) {
  if (B->schedule) return DFM_OK;
  cudaStream_t s = B->ctx->stream;
  const size_t n = (size_t)B->A->N * B->A->b;
  const unsigned trial_it = 12;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bs = 1, bt = 0, bl = 0;
  struct Cand { int sched, threads, lanes; };
  std::vector<Cand> cands = {{1, 0, 0}};
  for (int t : {256, 512, 1024})
    for (int l : {2, 4, 8}) cands.push_back({2, t, l});
  int rc = DFM_OK;
  for (const Cand& cd : cands) {
    if ((rc = set_ctl(B, d_ctl, trial_it, tol))) break;
    DFM_CUDA_TRY(cudaMemcpyAsync(B->r, b, n * sizeof(double),
                                 b_where == DFM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
    cudaEventRecord(e0, s);
    if ((rc = run_schedule(B, d_ctl, cd.sched, cd.threads, cd.lanes))) break;
    cudaEventRecord(e1, s);
    DFM_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) { best = ms; bs = cd.sched; bt = cd.threads; bl = cd.lanes; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  B->schedule = bs;
  B->cta_threads = bt;
  B->cta_lanes = bl;
  return DFM_OK;
}

int dfm_batch_set_schedule(dfm_batch B, int schedule, int cta_threads, int cta_lanes) {
  if (!B || schedule < 0 || schedule > 2) return DFM_ERR_INVALID;
  if (schedule == 2 && (cta_threads != 256 && cta_threads != 512 && cta_threads != 1024)) return DFM_ERR_INVALID;
  if (schedule == 2 && (cta_lanes != 2 && cta_lanes != 4 && cta_lanes != 8)) return DFM_ERR_INVALID;
  B->schedule = schedule;
  B->cta_threads = schedule == 2 ? cta_threads : 0;
  B->cta_lanes = schedule == 2 ? cta_lanes : 0;
  return DFM_OK;
}

int dfm_batch_get_schedule(dfm_batch B, int* schedule, int* cta_threads, int* cta_lanes) {
  if (!B) return DFM_ERR_INVALID;
  if (schedule) *schedule = B->schedule;
  if (cta_threads) *cta_threads = B->cta_threads;
  if (cta_lanes) *cta_lanes = B->cta_lanes;
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
  if ((rc = schedule_autotune(B, d_ctl, b, b_where, tol))) return rc;
  if ((rc = set_ctl(B, d_ctl, maxit, tol))) return rc;
  DFM_CUDA_TRY(cudaMemcpyAsync(B->r, b, n * sizeof(double),
                               b_where == DFM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  if ((rc = run_schedule(B, d_ctl, B->schedule, B->cta_threads, B->cta_lanes))) return rc;
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
