// ILU(0)-preconditioned Krylov solvers on the device, with the reference's
// stop tests and iteration conventions:
//   PCG        LsSol::Solve_PCG        src/ls/solver_ls_iter.cpp:100-172
//              (x = 0; stop on |r|^2/|r0|^2 < tol^2; *iters = 0-based index)
//   PBiCGSTAB  LsSol::Solve_PBiCGSTAB  src/ls/solver_ls_iter.cpp:291-408
//              (shadow residual r2 = r0; 1-based iterations; max_iter reached
//              is still `true` in the reference, DFM_NOT_CONVERGED here)
//   PCOCG      Fem::Ls::Solve_PCOCG    src/femls/zsolver_ls_iter.cpp:171-267
//              (complex symmetric, unconjugated products; 1-based iterations)
//   CG         LsSol::Solve_CG         src/ls/solver_ls_iter.cpp:31-97
//              (no preconditioner; x = 0; |r0|^2 < 1e-60 returns at once;
//              *iters = 0-based index; max_iter reached is `true` in the
//              reference with conv_ratio left at the tolerance)
//
// Every scalar lives in device memory (KrylovScalars); every reduction is a
// fixed-order sum of per-block partials (ctx part(k) arrays), so a solve is
// bit-reproducible run to run.  A CUDA graph of kIterPerGraph iterations is
// replayed until the device sets `done` (converged, max_iter, breakdown).
// Kernels after `done` return at once.  A scalar that one kernel derives and a
// later kernel needs is written by block 0 of the producer and read by the
// consumer kernel only, never within the kernel that writes it.
//
// Mixed precision (dfm_solve_pcg_mixed): the preconditioner runs with the FP32
// copies of L / D^-1 U (D^-1 and every vector, dot and scalar stay FP64), and
// the recurrences' SpMV with A's FP64 values or, when the context asks for it
// (mixed_op32), with FP32 copies, inside FP64 iterative refinement done as
// residual replacement: every kIterPerGraph-th iteration, and whenever the
// recursive residual meets the tolerance, r is replaced by the true b - A x
// computed with the FP64 values.  Only a true residual below the tolerance
// ends the solve.  Unlike restarting an inner solve per refinement step, this
// keeps the Krylov space across refinements.  An FP32 operator perturbs A by
// ~2^-24 |A|, so its search directions lose A-conjugacy on systems with
// cond(A) 2^-24 not << 1 (3-D elasticity: ~9x the iterations), hence the
// FP64 default.
//
// Partial slots: 0,1 SpMV dots; 2 (r, r); 3,4 preconditioned dots.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "dfm_internal.h"

namespace dfm {

constexpr int kIterPerGraph = 16;
constexpr int kVecThreads = 256;

static int vec_grid(dfm_mat A) { return spmv_grid(A); }

#define GRID_LOOP(k, n) \
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (n); k += (size_t)gridDim.x * blockDim.x)

DFM_DEVINL void finish(KrylovScalars* sc, int status, double conv) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->conv = conv;
    sc->conv_it = sc->it;
    sc->done = 100 + status;
  }
}

// ============================================================== PCG (real)
__global__ void __launch_bounds__(kVecThreads)
k_pcg_start(size_t n, const double* __restrict__ r, double* __restrict__ x, double* y, double* z, double* part_rr) {
  double acc = 0.0;
  GRID_LOOP(k, n) {
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
  GRID_LOOP(k, n) p[k] = z[k];
}

__global__ void __launch_bounds__(kVecThreads)
k_pcg_update_xr(size_t n, KrylovScalars* sc, const double* part_pq, int np_pq, const double* part_rz, int np_rz,
                double* part_rr, int np_rr, double* __restrict__ q_then_z, const double* __restrict__ p,
                double* __restrict__ r, double* __restrict__ x, double* __restrict__ y) {
  if (block_flag(&sc->done)) return;
  if (sc->it >= sc->maxit) {  // reference: loop ends, conv from the last (r, r)
    finish(sc, DFM_NOT_CONVERGED, sqrt(reduce_partials(part_rr, np_rr) * sc->inv0));
    return;
  }
  const double rz = reduce_partials(part_rz, np_rz);
  const double pq = reduce_partials(part_pq, np_pq);
  const double alpha = rz / pq;
  if (!isfinite(alpha)) {
    finish(sc, DFM_BREAKDOWN, NAN);
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->rz = rz;
    sc->alpha = alpha;
  }
  double acc = 0.0;
  GRID_LOOP(k, n) {
    const double qv = q_then_z[k];
    const double rv = r[k] - alpha * qv;
    r[k] = rv;
    x[k] += alpha * p[k];
    acc += rv * rv;
    y[k] = Sent<double>::value();
    q_then_z[k] = Sent<double>::value();
  }
  block_partial<kVecThreads>(acc, part_rr);
}

__global__ void __launch_bounds__(kVecThreads)
k_pcg_update_p(size_t n, KrylovScalars* sc, const double* part_rz, int np_rz, const double* __restrict__ z,
               double* __restrict__ p) {
  if (block_flag(&sc->done)) return;
  const double rz_new = reduce_partials(part_rz, np_rz);
  const double beta = rz_new / sc->rz;
  GRID_LOOP(k, n) p[k] = p[k] * beta + z[k];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->beta = beta;
    sc->it = sc->it + 1;
  }
}

// ======================================================= CG (real, no preconditioner)
// start: x = 0, partials of (r, r) into slot 2
__global__ void __launch_bounds__(kVecThreads)
k_cg_start(size_t n, const double* __restrict__ r, double* __restrict__ x, double* part_rr) {
  double acc = 0.0;
  GRID_LOOP(k, n) {
    const double rv = r[k];
    acc += rv * rv;
    x[k] = 0.0;
  }
  block_partial<kVecThreads>(acc, part_rr);
}

// |r0|^2 < 1e-60: the reference returns with num_iter = 0 and conv_ratio = |r0|
__global__ void __launch_bounds__(kVecThreads)
k_cg_start2(size_t n, KrylovScalars* sc, const double* part_rr, int np_rr, const double* __restrict__ r,
            double* __restrict__ p) {
  const double rr0 = reduce_partials(part_rr, np_rr);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->it = 0;
    if (rr0 < 1.0e-60) {
      sc->conv = sqrt(rr0);
      sc->conv_it = 0;
      sc->done = 100 + DFM_OK;
    } else {
      sc->inv0 = 1.0 / rr0;
      sc->rz = rr0;
      sc->done = 0;
    }
  }
  GRID_LOOP(k, n) p[k] = r[k];
}

// alpha = (r, r) / (p, Ap); x += alpha p; r -= alpha Ap; partials of the new (r, r).
// sc->rz holds (r, r); block 0 keeps it in sc->rho for k_cg_update_p, which
// writes the new one into sc->rz (no kernel writes a scalar it also reads).
__global__ void __launch_bounds__(kVecThreads)
k_cg_update_xr(size_t n, KrylovScalars* sc, const double* part_pq, int np_pq, const double* __restrict__ q,
               const double* __restrict__ p, double* __restrict__ r, double* __restrict__ x, double* part_rr) {
  if (block_flag(&sc->done)) return;
  if (sc->it >= sc->maxit) {
    finish(sc, DFM_NOT_CONVERGED, sqrt(sc->rz * sc->inv0));
    return;
  }
  const double rr = sc->rz;
  const double alpha = rr / reduce_partials(part_pq, np_pq);
  if (!isfinite(alpha)) {
    finish(sc, DFM_BREAKDOWN, NAN);
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->rho = rr;
    sc->alpha = alpha;
  }
  double acc = 0.0;
  GRID_LOOP(k, n) {
    x[k] += alpha * p[k];
    const double rv = r[k] - alpha * q[k];
    r[k] = rv;
    acc += rv * rv;
  }
  block_partial<kVecThreads>(acc, part_rr);
}

// stop test on the new (r, r); else beta = (r, r)_new / (r, r) and p = beta p + r
__global__ void __launch_bounds__(kVecThreads)
k_cg_update_p(size_t n, KrylovScalars* sc, const double* part_rr, int np_rr, const double* __restrict__ r,
              double* __restrict__ p) {
  if (block_flag(&sc->done)) return;
  const double rr_new = reduce_partials(part_rr, np_rr);
  if (rr_new * sc->inv0 < sc->tol2) {
    finish(sc, DFM_OK, sqrt(rr_new * sc->inv0));
    return;
  }
  const double beta = rr_new / sc->rho;
  GRID_LOOP(k, n) p[k] = beta * p[k] + r[k];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->beta = beta;
    sc->rz = rr_new;
    sc->it = sc->it + 1;
  }
}

// ======================================================== PBiCGSTAB (real)
// start: x = 0, r2 = r, p = r, partials of (r, r) into slot 2 and (r, r2) into slot 3
__global__ void __launch_bounds__(kVecThreads)
k_bicg_start(size_t n, const double* __restrict__ r, double* __restrict__ x, double* __restrict__ r2,
             double* __restrict__ p, double* y, double* Mp, double* part_rr, double* part_rr2) {
  double acc = 0.0;
  GRID_LOOP(k, n) {
    const double rv = r[k];
    acc += rv * rv;
    x[k] = 0.0;
    r2[k] = rv;
    p[k] = rv;
    y[k] = Sent<double>::value();
    Mp[k] = Sent<double>::value();
  }
  block_partial<kVecThreads>(acc, part_rr);
  block_partial<kVecThreads>(acc, part_rr2);
}

__global__ void k_bicg_start2(KrylovScalars* sc, const double* part_rr, int np_rr) {
  const double rr0 = reduce_partials(part_rr, np_rr);
  if (threadIdx.x == 0) {
    sc->it = 1;
    if (rr0 < 1.0e-60) {  // reference: conv_ratio = sqrt(sq0), iteration = 0, return true
      sc->conv = sqrt(rr0);
      sc->conv_it = 0;
      sc->done = 100 + DFM_OK;
    } else {
      sc->inv0 = 1.0 / rr0;
      sc->done = 0;
    }
  }
}

// alpha = (r, r2) / (AMp, r2); s = r - alpha AMp
__global__ void __launch_bounds__(kVecThreads)
k_bicg_s(size_t n, KrylovScalars* sc, const double* part_amp_r2, int np_spmv, const double* part_r_r2, int np_vec,
         const double* part_rr, const double* __restrict__ r, const double* __restrict__ AMp,
         double* __restrict__ s, double* y, double* Ms) {
  if (block_flag(&sc->done)) return;
  if (sc->it >= sc->maxit) {
    finish(sc, DFM_NOT_CONVERGED, sqrt(reduce_partials(part_rr, np_vec) * sc->inv0));
    return;
  }
  const double r_r2 = reduce_partials(part_r_r2, np_vec);
  const double alpha = r_r2 / reduce_partials(part_amp_r2, np_spmv);
  if (!isfinite(alpha)) {
    finish(sc, DFM_BREAKDOWN, NAN);
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->rho = r_r2;
    sc->alpha = alpha;
  }
  GRID_LOOP(k, n) {
    s[k] = r[k] - alpha * AMp[k];
    y[k] = Sent<double>::value();
    Ms[k] = Sent<double>::value();
  }
}

// omega = (s, AMs) / (AMs, AMs); x += alpha Mp + omega Ms; r = s - omega AMs;
// partials of (r, r) and (r, r2)
__global__ void __launch_bounds__(kVecThreads)
k_bicg_xr(size_t n, KrylovScalars* sc, const double* part_num, const double* part_den, int np_spmv,
          double* part_rr, double* part_r_r2, const double* __restrict__ Mp, const double* __restrict__ Ms,
          const double* __restrict__ s, const double* __restrict__ AMs, const double* __restrict__ r2,
          double* __restrict__ x, double* __restrict__ r) {
  if (block_flag(&sc->done)) return;
  const double omega = reduce_partials(part_num, np_spmv) / reduce_partials(part_den, np_spmv);
  if (!isfinite(omega)) {
    finish(sc, DFM_BREAKDOWN, NAN);
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->omega = omega;
  const double alpha = sc->alpha;
  double a_rr = 0.0, a_rr2 = 0.0;
  GRID_LOOP(k, n) {
    x[k] = (x[k] + alpha * Mp[k]) + omega * Ms[k];
    const double rv = s[k] - omega * AMs[k];
    r[k] = rv;
    a_rr += rv * rv;
    a_rr2 += rv * r2[k];
  }
  block_partial<kVecThreads>(a_rr, part_rr);
  block_partial<kVecThreads>(a_rr2, part_r_r2);
}

// stop test; beta = (r, r2)_new alpha / ((r, r2) omega); p = beta p + r - beta omega AMp
__global__ void __launch_bounds__(kVecThreads)
k_bicg_p(size_t n, KrylovScalars* sc, const double* part_rr, const double* part_r_r2, int np_vec,
         const double* __restrict__ r, const double* __restrict__ AMp, double* __restrict__ p, double* y,
         double* Mp) {
  if (block_flag(&sc->done)) return;
  const double rr = reduce_partials(part_rr, np_vec);
  if (rr * sc->inv0 < sc->tol2) {
    finish(sc, DFM_OK, sqrt(rr * sc->inv0));
    return;
  }
  const double tmp1 = reduce_partials(part_r_r2, np_vec);
  const double alpha = sc->alpha, omega = sc->omega;
  const double beta = tmp1 * alpha / (sc->rho * omega);
  const double bo = -beta * omega;
  GRID_LOOP(k, n) {
    p[k] = (p[k] * beta + r[k]) + bo * AMp[k];
    y[k] = Sent<double>::value();
    Mp[k] = Sent<double>::value();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->beta = beta;
    sc->it = sc->it + 1;
  }
}

// ========================================================== PCOCG (complex)
DFM_DEVINL double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
DFM_DEVINL double2 zdiv(double2 a, double2 b) {  // Com::Complex operator/ (include/delfem/complex.h)
  const double f = 1.0 / (b.x * b.x + b.y * b.y);
  return make_double2((a.x * b.x + a.y * b.y) * f, (-a.x * b.y + a.y * b.x) * f);
}

// start: x = 0, partials of |r|^2 (slot 2), y and w to the sentinel
__global__ void __launch_bounds__(kVecThreads)
k_cocg_start(size_t n2, const double* __restrict__ r, double* __restrict__ x, double* y, double* w, double* part_rr) {
  double acc = 0.0;
  GRID_LOOP(k, n2) {
    const double rv = r[k];
    acc += rv * rv;
    x[k] = 0.0;
    y[k] = Sent<double>::value();
    w[k] = Sent<double>::value();
  }
  block_partial<kVecThreads>(acc, part_rr);
}

__global__ void __launch_bounds__(kVecThreads)
k_cocg_start2(size_t n2, KrylovScalars* sc, const double* part_rr, int np_rr, const double* __restrict__ w,
              double* __restrict__ p) {
  const double rr0 = reduce_partials(part_rr, np_rr);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->it = 1;
    if (rr0 < 1.0e-30) {
      sc->conv = 0.0;
      sc->conv_it = 0;
      sc->done = 100 + DFM_OK;
    } else {
      sc->inv0 = 1.0 / rr0;
      sc->done = 0;
    }
  }
  GRID_LOOP(k, n2) p[k] = w[k];
}

// alpha = (r, w) / (p, Ap) (unconjugated); x += alpha p; r -= alpha Ap; partials of |r|^2
__global__ void __launch_bounds__(kVecThreads)
k_cocg_xr(size_t N, KrylovScalars* sc, const double* part_pap, int np_spmv, const double* part_rw, int np_rw,
          double* part_rr, int np_vec, const double2* __restrict__ p, const double2* __restrict__ Ap,
          double2* __restrict__ x, double2* __restrict__ r, double2* y, double2* w) {
  if (block_flag(&sc->done)) return;
  if (sc->it >= sc->maxit) {
    finish(sc, DFM_NOT_CONVERGED, sqrt(reduce_partials(part_rr, np_vec) * sc->inv0));
    return;
  }
  const double2 rw = make_double2(reduce_partials(part_rw, np_rw), reduce_partials(part_rw + kMaxBlocks, np_rw));
  const double2 pap =
      make_double2(reduce_partials(part_pap, np_spmv), reduce_partials(part_pap + kMaxBlocks, np_spmv));
  const double2 alpha = zdiv(rw, pap);
  if (!isfinite(alpha.x) || !isfinite(alpha.y)) {
    finish(sc, DFM_BREAKDOWN, NAN);
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->zr[0] = rw.x;
    sc->zr[1] = rw.y;
    sc->zr[2] = alpha.x;
    sc->zr[3] = alpha.y;
  }
  const double2 sent = make_double2(Sent<double>::value(), Sent<double>::value());
  double acc = 0.0;
  GRID_LOOP(k, N) {
    const double2 pk = p[k], ak = Ap[k];
    const double2 ap = zmul(alpha, pk), aa = zmul(alpha, ak);
    double2 xv = x[k], rv = r[k];
    xv.x += ap.x; xv.y += ap.y;
    rv.x -= aa.x; rv.y -= aa.y;
    x[k] = xv;
    r[k] = rv;
    acc += rv.x * rv.x + rv.y * rv.y;
    y[k] = sent;
    w[k] = sent;
  }
  block_partial<kVecThreads>(acc, part_rr);
}

// beta = (r, w)_new / (r, w); p = beta p + w
__global__ void __launch_bounds__(kVecThreads)
k_cocg_p(size_t N, KrylovScalars* sc, const double* part_rw, int np_rw, const double2* __restrict__ w,
         double2* __restrict__ p) {
  if (block_flag(&sc->done)) return;
  const double2 rw2 = make_double2(reduce_partials(part_rw, np_rw), reduce_partials(part_rw + kMaxBlocks, np_rw));
  const double2 beta = zdiv(rw2, make_double2(sc->zr[0], sc->zr[1]));
  GRID_LOOP(k, N) {
    const double2 t = zmul(p[k], beta), wk = w[k];
    p[k] = make_double2(t.x + wk.x, t.y + wk.y);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->it = sc->it + 1;
}

// ============================================================ solve plans
// vectors: PCG uses R X P Z Y; PCOCG adds Q (= Ap); PBiCGSTAB uses all
// (Z = Mp, Q = AMp).
enum { kVecR, kVecX, kVecP, kVecZ, kVecY, kVecQ, kVecR2, kVecS, kVecMs, kVecAMs, kNumVec };

static bool is_mixed(int method) { return method == DFM_PCG_MIXED || method == DFM_PCOCG_MIXED; }

static int vectors_of(int method) {
  switch (method) {
    case DFM_CG: return kVecZ + 1;  // Z holds Ap
    case DFM_PBICGSTAB: return kNumVec;
    case DFM_PCOCG: return kVecQ + 1;
    case DFM_PCG_MIXED:
    case DFM_PCOCG_MIXED: return kVecR2 + 1;  // kVecR2 keeps b for the true residual
    default: return kVecY + 1;
  }
}

// Workspace of one (M, method) pair: vectors and the captured graph, with the
// launch configuration the graph was captured with.
struct SolvePlan {
  dfm_ilu M = nullptr;
  dfm_mat A = nullptr;  // the owner of an unpreconditioned (CG) plan, which has no M
  int method = 0;
  size_t n = 0;  // doubles per vector
  double* v[kNumVec] = {};
  cudaGraphExec_t exec = nullptr;
  bool graph_failed = false;
  // capture key: everything the captured kernel arguments depend on
  int key_sweep = -1, key_lanes = -1, key_op32 = -1;
  unsigned key_gen = ~0u;
  unsigned long long key_wait = 0;
};

static std::mutex g_plan_mu;
static std::vector<SolvePlan*>& registry() {
  static std::vector<SolvePlan*> r;
  return r;
}

static void plan_drop_graph(SolvePlan* P) {
  if (P->exec) cudaGraphExecDestroy(P->exec);
  P->exec = nullptr;
  P->graph_failed = false;
}

static int plan_of(dfm_mat A, dfm_ilu M, int method, SolvePlan** out) {
  std::lock_guard<std::mutex> lock(g_plan_mu);
  dfm_mat owner = M ? nullptr : A;
  for (auto* e : registry())
    if (e->M == M && e->A == owner && e->method == method) {
      *out = e;
      return DFM_OK;
    }
  auto* P = new (std::nothrow) SolvePlan();
  if (!P) return DFM_ERR_NOMEM;
  P->M = M;
  P->A = owner;
  P->method = method;
  P->n = (size_t)A->N * A->xw();
  const size_t bytes = std::max<size_t>(P->n, 1) * sizeof(double);
  for (int k = 0; k < vectors_of(method); k++)
    if (cudaMalloc(&P->v[k], bytes) != cudaSuccess) {
      cudaGetLastError();
      for (int j = 0; j < k; j++) cudaFree(P->v[j]);
      delete P;
      return DFM_ERR_NOMEM;
    }
  registry().push_back(P);
  *out = P;
  return DFM_OK;
}

static void release_if(bool (*match)(const SolvePlan*, const void*), const void* key) {
  std::lock_guard<std::mutex> lock(g_plan_mu);
  auto& r = registry();
  for (size_t k = 0; k < r.size();) {
    if (!match(r[k], key)) { k++; continue; }
    SolvePlan* P = r[k];
    plan_drop_graph(P);
    for (double* v : P->v) cudaFree(v);
    delete P;
    r.erase(r.begin() + k);
  }
}

void solve_release(dfm_ilu M) {
  release_if([](const SolvePlan* P, const void* key) { return P->M == static_cast<dfm_ilu>(const_cast<void*>(key)); },
             M);
}

void solve_release_mat(dfm_mat A) {
  release_if([](const SolvePlan* P, const void* key) { return P->A == static_cast<dfm_mat>(const_cast<void*>(key)); },
             A);
}

// -------------------------------------------------- one iteration per method
static int enqueue_pcg(dfm_mat A, dfm_ilu M, SolvePlan* P, KrylovScalars* sc) {
  dfm_ctx c = A->ctx;
  const int gv = vec_grid(A), gs = sweep_grid(M, M->sweep);
  double *r = P->v[kVecR], *x = P->v[kVecX], *p = P->v[kVecP], *z = P->v[kVecZ], *y = P->v[kVecY];
  int rc = spmv_launch(A, 1.0, p, 0.0, z, c->part(0), gv, sc, A->lanes);
  if (rc) return rc;
  k_pcg_update_xr<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(0), gv, c->part(3), gs, c->part(2), gv, z, p,
                                                    r, x, y);
  DFM_CUDA_TRY(cudaGetLastError());
  if ((rc = ilu_fwd_launch(M, r, y, sc, M->sweep))) return rc;
  if ((rc = ilu_bwd_launch(M, y, z, r, c->part(3), sc, M->sweep))) return rc;
  k_pcg_update_p<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(3), gs, z, p);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

// r = b - A x with the FP64 values, partials of (r, r) in slot 2
static int enqueue_true_residual(dfm_mat A, SolvePlan* P, KrylovScalars* sc) {
  SpmvOpts o;
  o.yy = true;
  o.y0 = P->v[kVecR2];
  return spmv_launch(A, -1.0, P->v[kVecX], 0.0, P->v[kVecR], A->ctx->part(2), vec_grid(A), sc, A->lanes, o);
}

static int enqueue_pcg_mixed(dfm_mat A, dfm_ilu M, SolvePlan* P, KrylovScalars* sc, bool replace) {
  dfm_ctx c = A->ctx;
  const int gv = vec_grid(A), gs = sweep_grid(M, M->sweep);
  double *r = P->v[kVecR], *x = P->v[kVecX], *p = P->v[kVecP], *z = P->v[kVecZ], *y = P->v[kVecY];
  SpmvOpts o;
  o.f32 = c->mixed_op32 != 0;
  int rc = spmv_launch(A, 1.0, p, 0.0, z, c->part(0), gv, sc, A->lanes, o);
  if (rc) return rc;
  k_pcg_update_xr<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(0), gv, c->part(3), gs, c->part(2), gv, z, p,
                                                    r, x, y);
  DFM_CUDA_TRY(cudaGetLastError());
  if (replace && (rc = enqueue_true_residual(A, P, sc))) return rc;
  if ((rc = ilu_fwd_launch(M, r, y, sc, M->sweep, true, true))) return rc;
  if ((rc = ilu_bwd_launch(M, y, z, r, c->part(3), sc, M->sweep, true))) return rc;
  k_pcg_update_p<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(3), gs, z, p);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

// After the recursive residual met the tolerance (done == 99): the true
// residual decides; if it is not small enough the interrupted iteration is
// completed from the replaced residual and the solve goes on.
__global__ void k_mp_verify(KrylovScalars* sc, const double* part_rr, int np_rr) {
  const double rr = reduce_partials(part_rr, np_rr);
  if (threadIdx.x == 0) {
    if (rr * sc->inv0 < sc->tol2) {
      sc->conv = sqrt(rr * sc->inv0);
      sc->done = 100 + DFM_OK;
    } else {
      sc->done = 0;
    }
  }
}

static int mixed_verify(dfm_mat A, dfm_ilu M, SolvePlan* P, KrylovScalars* sc) {
  dfm_ctx c = A->ctx;
  const int gv = vec_grid(A), gs = sweep_grid(M, M->sweep);
  int rc = enqueue_true_residual(A, P, nullptr);
  if (rc) return rc;
  k_mp_verify<<<1, kVecThreads, 0, c->stream>>>(sc, c->part(2), gv);
  DFM_CUDA_TRY(cudaGetLastError());
  // completes the iteration if the solve goes on (kernels skip when done)
  if ((rc = ilu_fwd_launch(M, P->v[kVecR], P->v[kVecY], sc, M->sweep, false, true))) return rc;
  if ((rc = ilu_bwd_launch(M, P->v[kVecY], P->v[kVecZ], P->v[kVecR], c->part(3), sc, M->sweep, true))) return rc;
  if (P->method == DFM_PCOCG_MIXED)
    k_cocg_p<<<gv, kVecThreads, 0, c->stream>>>(A->N, sc, c->part(3), gs,
                                               reinterpret_cast<const double2*>(P->v[kVecZ]),
                                               reinterpret_cast<double2*>(P->v[kVecP]));
  else
    k_pcg_update_p<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(3), gs, P->v[kVecZ], P->v[kVecP]);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

static int enqueue_bicg(dfm_mat A, dfm_ilu M, SolvePlan* P, KrylovScalars* sc) {
  dfm_ctx c = A->ctx;
  const int gv = vec_grid(A);
  double *r = P->v[kVecR], *x = P->v[kVecX], *p = P->v[kVecP], *Mp = P->v[kVecZ], *y = P->v[kVecY];
  double *AMp = P->v[kVecQ], *r2 = P->v[kVecR2], *s = P->v[kVecS], *Ms = P->v[kVecMs], *AMs = P->v[kVecAMs];
  int rc;
  // Mp = M^-1 p; AMp = A Mp with (r2, AMp)
  if ((rc = ilu_fwd_launch(M, p, y, sc, M->sweep, false))) return rc;
  if ((rc = ilu_bwd_launch(M, y, Mp, nullptr, nullptr, sc, M->sweep))) return rc;
  SpmvOpts o1;
  o1.dot_w = r2;
  if ((rc = spmv_launch(A, 1.0, Mp, 0.0, AMp, c->part(0), gv, sc, A->lanes, o1))) return rc;
  k_bicg_s<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(0), gv, c->part(3), gv, c->part(2), r, AMp, s, y, Ms);
  DFM_CUDA_TRY(cudaGetLastError());
  // Ms = M^-1 s; AMs = A Ms with (s, AMs) and (AMs, AMs)
  if ((rc = ilu_fwd_launch(M, s, y, sc, M->sweep, false))) return rc;
  if ((rc = ilu_bwd_launch(M, y, Ms, nullptr, nullptr, sc, M->sweep))) return rc;
  SpmvOpts o2;
  o2.dot_w = s;
  o2.dot_part2 = c->part(1);
  if ((rc = spmv_launch(A, 1.0, Ms, 0.0, AMs, c->part(0), gv, sc, A->lanes, o2))) return rc;
  k_bicg_xr<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(0), c->part(1), gv, c->part(2), c->part(3), Mp, Ms,
                                              s, AMs, r2, x, r);
  DFM_CUDA_TRY(cudaGetLastError());
  k_bicg_p<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(2), c->part(3), gv, r, AMp, p, y, Mp);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

static int enqueue_cocg(dfm_mat A, dfm_ilu M, SolvePlan* P, KrylovScalars* sc, bool f32 = false,
                        bool replace = false) {
  dfm_ctx c = A->ctx;
  const int gv = vec_grid(A), gs = sweep_grid(M, M->sweep);
  double *r = P->v[kVecR], *x = P->v[kVecX], *p = P->v[kVecP], *w = P->v[kVecZ], *y = P->v[kVecY];
  double* Ap = P->v[kVecQ];
  SpmvOpts o;
  o.f32 = f32 && c->mixed_op32 != 0;
  int rc = spmv_launch(A, 1.0, p, 0.0, Ap, c->part(0), gv, sc, A->lanes, o);  // (p, Ap) re/im in slots 0/1
  if (rc) return rc;
  k_cocg_xr<<<gv, kVecThreads, 0, c->stream>>>(A->N, sc, c->part(0), gv, c->part(3), gs, c->part(2), gv,
                                              reinterpret_cast<const double2*>(p),
                                              reinterpret_cast<const double2*>(Ap), reinterpret_cast<double2*>(x),
                                              reinterpret_cast<double2*>(r), reinterpret_cast<double2*>(y),
                                              reinterpret_cast<double2*>(w));
  DFM_CUDA_TRY(cudaGetLastError());
  if (replace && (rc = enqueue_true_residual(A, P, sc))) return rc;
  if ((rc = ilu_fwd_launch(M, r, y, sc, M->sweep, true, f32))) return rc;                 // stop test on slot 2
  if ((rc = ilu_bwd_launch(M, y, w, r, c->part(3), sc, M->sweep, f32))) return rc;  // (r, w) re/im in slots 3/4
  k_cocg_p<<<gv, kVecThreads, 0, c->stream>>>(A->N, sc, c->part(3), gs, reinterpret_cast<const double2*>(w),
                                             reinterpret_cast<double2*>(p));
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

static int enqueue_cg(dfm_mat A, SolvePlan* P, KrylovScalars* sc) {
  dfm_ctx c = A->ctx;
  const int gv = vec_grid(A);
  double *r = P->v[kVecR], *x = P->v[kVecX], *p = P->v[kVecP], *q = P->v[kVecZ];
  int rc = spmv_launch(A, 1.0, p, 0.0, q, c->part(0), gv, sc, A->lanes);  // q = A p with (p, q)
  if (rc) return rc;
  k_cg_update_xr<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(0), gv, q, p, r, x, c->part(2));
  DFM_CUDA_TRY(cudaGetLastError());
  k_cg_update_p<<<gv, kVecThreads, 0, c->stream>>>(P->n, sc, c->part(2), gv, r, p);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

// k: index of the iteration inside one graph of kIterPerGraph
static int enqueue_iteration(dfm_mat A, dfm_ilu M, SolvePlan* P, KrylovScalars* sc, int k) {
  switch (P->method) {
    case DFM_CG: return enqueue_cg(A, P, sc);
    case DFM_PBICGSTAB: return enqueue_bicg(A, M, P, sc);
    case DFM_PCOCG: return enqueue_cocg(A, M, P, sc);
    case DFM_PCG_MIXED: return enqueue_pcg_mixed(A, M, P, sc, k == kIterPerGraph - 1);
    case DFM_PCOCG_MIXED: return enqueue_cocg(A, M, P, sc, true, k == kIterPerGraph - 1);
    default: return enqueue_pcg(A, M, P, sc);
  }
}

// ---------------------------------------------------------- initial steps
static int enqueue_start(dfm_mat A, dfm_ilu M, SolvePlan* P, KrylovScalars* sc) {
  dfm_ctx c = A->ctx;
  cudaStream_t s = c->stream;
  const int gv = vec_grid(A);
  double *r = P->v[kVecR], *x = P->v[kVecX], *p = P->v[kVecP], *z = P->v[kVecZ], *y = P->v[kVecY];
  int rc;
  switch (P->method) {
    case DFM_CG:
      k_cg_start<<<gv, kVecThreads, 0, s>>>(P->n, r, x, c->part(2));
      DFM_CUDA_TRY(cudaGetLastError());
      k_cg_start2<<<gv, kVecThreads, 0, s>>>(P->n, sc, c->part(2), gv, r, p);
      break;
    case DFM_PBICGSTAB:
      k_bicg_start<<<gv, kVecThreads, 0, s>>>(P->n, r, x, P->v[kVecR2], p, y, z, c->part(2), c->part(3));
      DFM_CUDA_TRY(cudaGetLastError());
      k_bicg_start2<<<1, kVecThreads, 0, s>>>(sc, c->part(2), gv);
      break;
    case DFM_PCOCG:
    case DFM_PCOCG_MIXED: {
      const bool f32 = P->method == DFM_PCOCG_MIXED;
      if (f32) DFM_CUDA_TRY(cudaMemcpyAsync(P->v[kVecR2], r, P->n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      k_cocg_start<<<gv, kVecThreads, 0, s>>>(P->n, r, x, y, z, c->part(2));
      DFM_CUDA_TRY(cudaGetLastError());
      if ((rc = ilu_fwd_launch(M, r, y, nullptr, M->sweep, true, f32))) return rc;
      if ((rc = ilu_bwd_launch(M, y, z, r, c->part(3), nullptr, M->sweep, f32))) return rc;
      k_cocg_start2<<<gv, kVecThreads, 0, s>>>(P->n, sc, c->part(2), gv, z, p);
      break;
    }
    default: {
      const bool f32 = P->method == DFM_PCG_MIXED;
      if (f32) DFM_CUDA_TRY(cudaMemcpyAsync(P->v[kVecR2], r, P->n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      k_pcg_start<<<gv, kVecThreads, 0, s>>>(P->n, r, x, y, z, c->part(2));
      DFM_CUDA_TRY(cudaGetLastError());
      if ((rc = ilu_fwd_launch(M, r, y, nullptr, M->sweep, true, f32))) return rc;
      if ((rc = ilu_bwd_launch(M, y, z, r, c->part(3), nullptr, M->sweep, f32))) return rc;
      k_pcg_start2<<<gv, kVecThreads, 0, s>>>(P->n, sc, c->part(2), gv, z, p);
      break;
    }
  }
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

// Capture kIterPerGraph iterations once per plan and launch configuration.
static void ensure_graph(dfm_mat A, dfm_ilu M, SolvePlan* P, KrylovScalars* sc) {
  dfm_ctx c = A->ctx;
  const int lanes_key = A->lanes * 2 + A->spmv_kind;
  const int sweep_key = M ? M->sweep : 0;
  const unsigned gen_key = M ? M->plan_gen : 0u;
  const bool same = P->key_sweep == sweep_key && P->key_lanes == lanes_key && P->key_gen == gen_key &&
                    P->key_wait == c->wait_ns && P->key_op32 == c->mixed_op32;
  if (!same) {
    plan_drop_graph(P);
    P->key_op32 = c->mixed_op32;
    P->key_sweep = sweep_key;
    P->key_lanes = lanes_key;
    P->key_gen = gen_key;
    P->key_wait = c->wait_ns;
  }
  if (P->exec || P->graph_failed) return;
  cudaStream_t s = c->stream;
  cudaGraph_t g = nullptr;
  bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  int erc = DFM_OK;
  if (ok) {
    for (int k = 0; k < kIterPerGraph && erc == DFM_OK; k++) erc = enqueue_iteration(A, M, P, sc, k);
    ok = (cudaStreamEndCapture(s, &g) == cudaSuccess) && erc == DFM_OK;
  }
  if (ok) ok = cudaGraphInstantiate(&P->exec, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    P->exec = nullptr;
    P->graph_failed = true;
    cudaGetLastError();  // clear a capture error; iterations are then launched directly
  }
}

// Runs `method` on A x = b.  b: N*xw doubles at `b_where`; x receives the
// solution (at x_where); r_out (device, nullable) receives the final residual.
int krylov_solve(dfm_mat A, dfm_ilu M, int method, const double* b, int b_where, double* x, int x_where,
                 double* r_out, double tol, unsigned maxit, unsigned* iters, double* conv) {
  dfm_ctx c = A->ctx;
  cudaStream_t s = c->stream;
  if (!M && method != DFM_CG) return DFM_ERR_INVALID;
  int rc = spmv_autotune(A);
  if (rc) return rc;
  if (M && (rc = ilu_autotune(M))) return rc;
  const bool f32 = is_mixed(method);
  if (f32 && c->mixed_op32 && (rc = mat_make_f32(A))) return rc;
  if (M && (rc = ilu_prepare(M, f32))) return rc;
  SolvePlan* P = nullptr;
  if ((rc = plan_of(A, M, method, &P))) return rc;
  const size_t n = P->n;
  KrylovScalars* sc = c->d_scal;
  {
    KrylovScalars h = {};
    h.maxit = maxit;
    h.tol2 = tol * tol;
    h.conv_code = f32 ? 99 : 100 + DFM_OK;
    DFM_CUDA_TRY(cudaMemcpyAsync(sc, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  }
  DFM_CUDA_TRY(cudaMemcpyAsync(P->v[kVecR], b, n * sizeof(double),
                               b_where == DFM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  if ((rc = enqueue_start(A, M, P, sc))) return rc;
  ensure_graph(A, M, P, sc);
  for (;;) {
    if (P->exec) {
      DFM_CUDA_TRY(cudaGraphLaunch(P->exec, s));
    } else {
      for (int k = 0; k < kIterPerGraph; k++)
        if ((rc = enqueue_iteration(A, M, P, sc, k))) return rc;
    }
    DFM_CUDA_TRY(cudaMemcpyAsync(c->h_scal, sc, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, s));
    DFM_CUDA_TRY(cudaStreamSynchronize(s));
    if (c->h_scal->done == 99) {  // mixed precision: confirm with the FP64 residual
      if ((rc = mixed_verify(A, M, P, sc))) return rc;
      DFM_CUDA_TRY(cudaMemcpyAsync(c->h_scal, sc, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, s));
      DFM_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (c->h_scal->done) break;
    const int code = take_code(c);
    if (code) return code;
  }
  // Solve_PBiCGSTAB returns before zeroing x when |r0|^2 < 1e-60: x is left as given
  const bool keep_x = method == DFM_PBICGSTAB && c->h_scal->done == 100 + DFM_OK && c->h_scal->conv_it == 0;
  if (!keep_x)
    DFM_CUDA_TRY(cudaMemcpyAsync(x, P->v[kVecX], n * sizeof(double),
                                 x_where == DFM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
  if (r_out) DFM_CUDA_TRY(cudaMemcpyAsync(r_out, P->v[kVecR], n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  {
    const int code = take_code(c);
    if (code) return code;
  }
  const KrylovScalars* h = c->h_scal;
  if (iters) *iters = h->conv_it;
  if (conv) *conv = h->conv;
  return h->done - 100;
}

}  // namespace dfm
