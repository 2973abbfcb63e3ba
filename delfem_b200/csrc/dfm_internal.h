// Host-side objects behind the C ABI handles (include/dfm_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "dfm_b200.h"
#include "common.cuh"
#include "sweep.h"

#define DFM_CUDA_TRY(expr)                                 \
  do {                                                     \
    cudaError_t e__ = (expr);                              \
    if (e__ != cudaSuccess) return dfm::cuda_fail(e__, #expr); \
  } while (0)

namespace dfm {

int cuda_fail(cudaError_t e, const char* what);
void ctx_retain(dfm_ctx c);
void ctx_release(dfm_ctx c);
int take_code(dfm_ctx c);
// Host (DFM_HOST, then synchronises) or device source -> device memory.
int copy_in(void* dst, const void* src, size_t bytes, int where, cudaStream_t s);

template <typename T>
inline int dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  DFM_CUDA_TRY(cudaMalloc((void**)p, count * sizeof(T)));
  return DFM_OK;
}

// Scalars of one Krylov solve, in device memory so a captured CUDA graph can
// run many iterations without the host.
struct KrylovScalars {
  int done;        // 0 running, else final dfm_status + 100 (so DFM_OK is distinguishable)
  unsigned it;     // iterations completed (0-based index of the next one)
  unsigned maxit;
  unsigned conv_it;
  double tol2;     // tol^2
  double inv0;     // 1 / |r0|^2
  double rz;       // (r, z) of the current direction
  double conv;     // final sqrt(|r|^2 / |r0|^2)
  int conv_code;   // `done` written when the recursive residual meets tol (100 = final, 99 = verify first)
  int pad_;
  double alpha, beta, omega, rho;  // BiCGSTAB / COCG extras
  double zr[4];    // complex scalars (re, im pairs)
};

// Upper bound of blocks of the grid-stride kernels (partials arrays length).
constexpr int kMaxBlocks = 148 * 16;
// Spare elements at the end of every matrix array (bulk copies round to 16 B).
constexpr size_t kArrayPad = 16;

// Row tiles of the TMA-staged SpMV (spmv.cu) for one value width.
struct SpmvTiles {
  bool valid = false;
  unsigned ntiles = 0, max_rows = 0, max_blocks = 0;
  unsigned* d_tiles = nullptr;  // ntiles + 1 row bounds
  unsigned stage_bytes = 0, vals_bytes = 0, col_bytes = 0, diag_bytes = 0, rp_bytes = 0;
  int nstage = 0;
};

}  // namespace dfm

struct dfm_ctx_s;
struct dfm_ctx_s {
  // one reference for the caller's handle and one per object created on the
  // context; dfm_ctx_destroy drops the caller's, the last one frees it (so
  // objects may outlive the handle and be destroyed in any order)
  std::atomic<int> refs{1};
  int device = 0;
  int nsm = 148;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  DevStatus* d_status = nullptr;
  unsigned long long wait_ns = 2000000000ull;
  int mixed_op32 = 0;                       // mixed-precision solves: FP32 operator values
  double* d_part = nullptr;                 // 8 partial arrays of kMaxBlocks doubles
  dfm::KrylovScalars* d_scal = nullptr;
  dfm::KrylovScalars* h_scal = nullptr;     // pinned mirror
  double* noalloc_scratch = nullptr;        // device address of noalloc.cu's static array (set on first use)
  double* part(int k) { return d_part + (size_t)k * dfm::kMaxBlocks; }
};

struct dfm_mat_s {
  dfm_ctx ctx = nullptr;
  unsigned N = 0, b = 1, ncrs = 0;
  int vt = DFM_REAL;
  unsigned* d_rowptr = nullptr;
  unsigned* d_colind = nullptr;
  double* d_diag = nullptr;
  double* d_off = nullptr;
  float* d_diag32 = nullptr;  // FP32 copies of the values for the mixed-precision solve
  float* d_off32 = nullptr;
  std::vector<unsigned> h_rowptr, h_colind;
  unsigned max_row = 0;     // most off-diagonal blocks in one row
  int lanes = 0;            // SpMV lanes per block row (0 = not tuned yet)
  int spmv_kind = 0;        // 0 lane per block, 1 TMA-staged tiles, 2 element-wise, 3 warp-staged (autotuned)
  dfm::SpmvTiles tiles[2];  // [0] FP64 values, [1] FP32 copies
  size_t vw() const { return vt == DFM_COMPLEX ? 2 : (size_t)b * b; }   // doubles per block
  size_t xw() const { return vt == DFM_COMPLEX ? 2 : b; }               // doubles per vector block
};

struct dfm_ilu_s {
  dfm_ctx ctx = nullptr;
  dfm_mat A = nullptr;      // pattern owner (rowptr/colind shared): the system matrix, or fillpat
  dfm_mat user = nullptr;   // the system matrix the preconditioner was made for
  dfm_mat fillpat = nullptr;   // ILU(k), k != 0: owned pattern-only matrix of the filled pattern
  unsigned* d_fillmap = nullptr;  // ILU(k): factor slot of each of user's off-diagonal slots
  int fill_level = 0;
  std::vector<unsigned> part_of;  // optional row partition for the range sweeps: part of every row
  unsigned nparts = 0;
  unsigned N = 0, b = 1, ncrs = 0;
  int vt = DFM_REAL;
  unsigned* d_diaind = nullptr;
  // rows sorted by forward / backward level (ascending row within a level)
  unsigned* d_order_f = nullptr;
  unsigned* d_order_b = nullptr;
  unsigned* d_lvl_f = nullptr;   // level pointers into order_f (nlev_f + 1)
  unsigned* d_lvl_b = nullptr;
  std::vector<unsigned> lev_f, lev_b, h_diaind;
  unsigned nlev_f = 0, nlev_b = 0;
  double* d_fdiag = nullptr;     // D^-1 blocks
  double* d_foff = nullptr;      // L and D^-1 U blocks
  float* d_foff32 = nullptr;     // FP32 copy of d_foff (mixed precision; D^-1 stays FP64)
  unsigned* d_flags = nullptr;   // per-row completion epochs of the numeric factorisation
  unsigned epoch = 0;
  double* d_tmp = nullptr;       // N*xw scratch: forward-sweep output of dfm_ilu_apply
  int sweep = 0;                 // 0 untuned, 1 sync-free grid, 2 single CTA, 3 CTA row ranges
  int sweep_blocks = 0;          // sync-free grid size cap (0 = all co-resident blocks)
  dfm::SweepPlan plan_f, plan_b; // mode 3 plans (forward / backward)
  dfm::SweepPlan plan32_f, plan32_b;  // mode 3 plans with FP32 values
  unsigned plan_gen = 0;         // bumped whenever the schedule or its plans change
  float sweep_ms = 0.f;          // autotuned fwd+bwd time
  bool factored = false;
  size_t vw() const { return vt == DFM_COMPLEX ? 2 : (size_t)b * b; }
  size_t xw() const { return vt == DFM_COMPLEX ? 2 : b; }
};

namespace dfm {
// spmv.cu
// Options of one SpMV launch:
//   dot_w  with dot_part: partials of (dot_w ? dot_w : x) . y     (real only)
//   dot_part2: partials of y . y beside the first dot            (real only)
//   yy: dot_part receives y . y (|y|^2 for complex) instead
//   y0: y = y0 + alpha A x (beta ignored)
//   f32: multiply with the FP32 copy of the values
// Without options a complex SpMV with dot_part writes the unconjugated x^T y
// (re in dot_part, im in dot_part + kMaxBlocks).
struct SpmvOpts {
  const double* dot_w = nullptr;
  double* dot_part2 = nullptr;
  bool yy = false;
  const double* y0 = nullptr;
  bool f32 = false;
  int kind = -1;  // -1: the matrix's tuned kernel; 0 lane per block; 1 TMA-staged tiles; 2 element-wise;
                  // 3 warp-staged
};
int spmv_launch(dfm_mat A, double alpha, const double* x, double beta, double* y, double* dot_part,
                int nblocks_hint, KrylovScalars* sc, int lanes, const SpmvOpts& o = SpmvOpts());
int mat_make_f32(dfm_mat A);
void spmv_free_tiles(dfm_mat A);
int to_f32(dfm_ctx c, const double* in, float* out, size_t n);
int spmv_autotune(dfm_mat A);
int spmv_grid(dfm_mat A);
// ilu.cu
int ilu_factor_launch(dfm_ilu M, dfm_mat A);
// fill.cu
int ilu_fill_pattern(unsigned N, const std::vector<unsigned>& rp, const std::vector<unsigned>& ci, int lev,
                     std::vector<unsigned>& frp, std::vector<unsigned>& fci, const std::vector<unsigned char>& unl,
                     unsigned bound);
int ilu_fill_values(dfm_ilu M, dfm_mat A);
// With sc, a forward sweep first stops the solve when |r|^2/|r0|^2 < tol^2
// (partials in part(2)) unless rr_check is false.
// f32: the sweeps read the FP32 copy of L / D^-1 U (D^-1 itself stays FP64).
int ilu_fwd_launch(dfm_ilu M, const double* r, double* y, KrylovScalars* sc, int sweep, bool rr_check = true,
                   bool f32 = false);
int ilu_bwd_launch(dfm_ilu M, const double* y, double* z, const double* rdot, double* dot_part,
                   KrylovScalars* sc, int sweep, bool f32 = false);
// Brings the packed sweep plans (and, with f32, the FP32 factor copy and its
// plans) up to date with the factor, outside any stream capture.
int ilu_prepare(dfm_ilu M, bool f32);
int ilu_fill_sentinel(dfm_ilu M, double* v, size_t n);
int ilu_autotune(dfm_ilu M);
int sweep_grid(dfm_ilu M, int sweep);
int ilu_wait_selftest(dfm_ctx ctx, unsigned long long limit_ns);
int set_poll_sleep(unsigned ns);
// sweep.cu
// merge: steps are pairs of levels (the second level's operands on the
// first are substituted by products with the factor; see sweep.cu)
// part: the CTAs are the parts of the ILU's row partition (G must be its
// part count) instead of balanced ranges of the natural row order
// halo: the plan of the shared-memory-only schedule (sweep_halo.cu; unmerged,
// FP64 vectors)
int sweep_plan_build(dfm_ilu M, bool fwd, int G, int val_bytes, int vec_bytes, SweepPlan* P, bool merge = false,
                     bool part = false, bool halo = false);
// sweep_halo.cu
int sweep_halo_plan_build(dfm_ilu M, bool fwd, int G, int val_bytes, SweepPlan* P, bool part, bool merge = false);
cudaError_t sweep_halo_launch(dfm_ilu M, bool fwd, const SweepPlan* P, const double* in, double* out,
                              const double* rdot, double* part, KrylovScalars* sc, const double* rr_part, int rr_n,
                              bool f32);
void sweep_plan_free(SweepPlan* P);
int sweep_plan_refresh(dfm_ilu M, SweepPlan* P);
int ilu_set_ranges(dfm_ilu M, int G, bool merge = false, bool halo = false);
int sweep_ranges_launch(dfm_ilu M, bool fwd, const double* in, double* out, const double* rdot, double* part,
                        KrylovScalars* sc, const double* rr_part, int rr_n, bool f32 = false);
// krylov.cu
// method: DFM_PCG / DFM_PBICGSTAB / DFM_PCOCG / the mixed forms, or DFM_CG
// with M == nullptr; b and x at DFM_HOST or DFM_DEVICE.
int krylov_solve(dfm_mat A, dfm_ilu M, int method, const double* b, int b_where, double* x, int x_where,
                 double* r_out, double tol, unsigned maxit, unsigned* iters, double* conv);
void solve_release(dfm_ilu M);
void solve_release_mat(dfm_mat A);  // unpreconditioned (CG) plans of A
}  // namespace dfm
