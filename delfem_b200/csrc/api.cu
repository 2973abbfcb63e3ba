// C ABI entry points (include/dfm_b200.h): handle lifetimes, host-side
// validation of patterns, the symbolic ILU(0) (m_DiaInd + level sets), and
// dispatch to the kernels.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>

#include "dfm_internal.h"

namespace dfm {

// the CUDA error behind the last DFM_ERR_CUDA / DFM_ERR_NOMEM of this host
// thread and the runtime call that returned it (a string literal)
thread_local cudaError_t g_cuda_err = cudaSuccess;
thread_local const char* g_cuda_what = "";

int cuda_fail(cudaError_t e, const char* what) {
  g_cuda_err = e;
  g_cuda_what = what;
  if (e == cudaErrorMemoryAllocation) { cudaGetLastError(); return DFM_ERR_NOMEM; }
  return DFM_ERR_CUDA;
}

int copy_in(void* dst, const void* src, size_t bytes, int where, cudaStream_t s) {
  if (bytes == 0) return DFM_OK;
  if (!src || !dst) return DFM_ERR_INVALID;
  DFM_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, where == DFM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  if (where == DFM_HOST) DFM_CUDA_TRY(cudaStreamSynchronize(s));
  return DFM_OK;
}

// Reads and clears the device status code (a timed-out wait, ...).
int take_code(dfm_ctx c) {
  DevStatus h = {};
  DFM_CUDA_TRY(cudaMemcpyAsync(&h, c->d_status, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (h.code) {
    DFM_CUDA_TRY(cudaMemsetAsync(&c->d_status->code, 0, sizeof(int), c->stream));
    DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  return h.code;
}

static int copy_out(void* dst, const void* src, size_t bytes, int where, cudaStream_t s) {
  if (bytes == 0) return DFM_OK;
  if (!src || !dst) return DFM_ERR_INVALID;
  DFM_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, where == DFM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  return DFM_OK;
}

// Level sets of the natural ordering: lev(i) = 1 + max lev(j) over the rows the
// sweep reads (j in L(i) forward, j in U(i) backward), 0 for none.  Rows are
// then listed level by level, ascending inside a level.
static unsigned make_levels(unsigned N, const std::vector<unsigned>& rowptr, const std::vector<unsigned>& colind,
                            const std::vector<unsigned>& diaind, bool fwd, std::vector<unsigned>& lev,
                            std::vector<unsigned>& order, std::vector<unsigned>& lvlptr) {
  lev.assign(N, 0);
  unsigned nl = 0;
  for (unsigned t = 0; t < N; t++) {
    const unsigned i = fwd ? t : N - 1 - t;
    const unsigned s0 = fwd ? rowptr[i] : diaind[i], s1 = fwd ? diaind[i] : rowptr[i + 1];
    unsigned l = 0;
    for (unsigned s = s0; s < s1; s++) l = std::max(l, lev[colind[s]] + 1);
    lev[i] = l;
    nl = std::max(nl, l + 1);
  }
  if (N == 0) nl = 0;
  lvlptr.assign(nl + 1, 0);
  for (unsigned i = 0; i < N; i++) lvlptr[lev[i] + 1]++;
  for (unsigned l = 0; l < nl; l++) lvlptr[l + 1] += lvlptr[l];
  order.assign(N, 0);
  std::vector<unsigned> fill(lvlptr.begin(), lvlptr.end() - (nl ? 1 : 0));
  for (unsigned i = 0; i < N; i++) order[fill[lev[i]]++] = i;
  return nl;
}

// Average duration of `reps` launches of `launch` on stream s (CUDA events).
template <typename F>
static int time_launches(cudaStream_t s, int reps, float* ms, F launch) {
  int rc = launch();  // untimed first launch
  if (rc) return rc;
  cudaEvent_t e0, e1;
  DFM_CUDA_TRY(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return DFM_ERR_CUDA;
  }
  cudaEventRecord(e0, s);
  for (int k = 0; k < reps && !rc; k++) rc = launch();
  cudaEventRecord(e1, s);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "time_launches");
  *ms = t / (float)reps;
  return DFM_OK;
}

}  // namespace dfm

using namespace dfm;

extern "C" {

int dfm_last_cuda_error(char* buf, size_t n) {
  if (buf && n) std::snprintf(buf, n, "%s: %s", g_cuda_what, cudaGetErrorName(g_cuda_err));
  return (int)g_cuda_err;
}

const char* dfm_status_string(int s) {
  switch (s) {
    case DFM_OK: return "ok";
    case DFM_ERR_INVALID: return "invalid argument";
    case DFM_ERR_CUDA: return "CUDA error";
    case DFM_ERR_IO: return "file could not be opened or read";
    case DFM_ERR_NOMEM: return "out of device memory";
    case DFM_NOT_CONVERGED: return "not converged";
    case DFM_BREAKDOWN: return "breakdown";
    case DFM_SINGULAR_PIVOT: return "singular pivot";
    case DFM_WAIT_TIMEOUT: return "device wait timeout";
    case DFM_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown";
  }
}

int dfm_abi_version(void) { return DFM_ABI_VERSION; }

int dfm_ctx_create(int device, dfm_ctx* out) {
  if (!out) return DFM_ERR_INVALID;
  *out = nullptr;
  DFM_CUDA_TRY(cudaSetDevice(device));
  dfm_ctx c = new (std::nothrow) dfm_ctx_s();
  if (!c) return DFM_ERR_NOMEM;
  c->device = device;
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
  int rc = DFM_OK;
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) rc = DFM_ERR_CUDA;
  c->stream = c->own;
  if (!rc) rc = dalloc(&c->d_status, 1);
  if (!rc) rc = dalloc(&c->d_part, (size_t)8 * kMaxBlocks);
  if (!rc) rc = dalloc(&c->d_scal, 1);
  if (!rc && cudaMallocHost((void**)&c->h_scal, sizeof(KrylovScalars)) != cudaSuccess) rc = DFM_ERR_CUDA;
  if (!rc && cudaMemset(c->d_status, 0, sizeof(DevStatus)) != cudaSuccess) rc = DFM_ERR_CUDA;
  if (!rc && cudaMemset(c->d_scal, 0, sizeof(KrylovScalars)) != cudaSuccess) rc = DFM_ERR_CUDA;
  if (rc) { dfm_ctx_destroy(c); return rc; }
  *out = c;
  return DFM_OK;
}

int dfm_ctx_destroy(dfm_ctx c) {
  if (c) ctx_release(c);
  return DFM_OK;
}

}  // extern "C"

namespace dfm {
void ctx_retain(dfm_ctx c) { c->refs.fetch_add(1, std::memory_order_relaxed); }

void ctx_release(dfm_ctx c) {
  if (c->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
  cudaSetDevice(c->device);
  if (c->own) cudaStreamSynchronize(c->own);
  cudaFree(c->d_status);
  cudaFree(c->d_part);
  cudaFree(c->d_scal);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}
}  // namespace dfm

extern "C" {

int dfm_ctx_set_stream(dfm_ctx c, void* stream) {
  if (!c) return DFM_ERR_INVALID;
  c->stream = stream ? (cudaStream_t)stream : c->own;
  return DFM_OK;
}

int dfm_ctx_sync(dfm_ctx c) {
  if (!c) return DFM_ERR_INVALID;
  DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return DFM_OK;
}

int dfm_ctx_set_wait_limit(dfm_ctx c, unsigned long long ns) {
  if (!c || ns == 0) return DFM_ERR_INVALID;
  c->wait_ns = ns;
  return DFM_OK;
}

int dfm_ctx_set_mixed_operator(dfm_ctx c, int fp32) {
  if (!c || (fp32 != 0 && fp32 != 1)) return DFM_ERR_INVALID;
  c->mixed_op32 = fp32;
  return DFM_OK;
}

int dfm_ctx_get_mixed_operator(dfm_ctx c, int* fp32) {
  if (!c || !fp32) return DFM_ERR_INVALID;
  *fp32 = c->mixed_op32;
  return DFM_OK;
}

int dfm_ctx_take_error(dfm_ctx c, int* code, int* where) {
  if (!c) return DFM_ERR_INVALID;
  DevStatus h = {};
  DFM_CUDA_TRY(cudaMemcpyAsync(&h, c->d_status, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (code) *code = h.code;
  if (where) *where = h.where;
  h.code = 0;
  h.where = 0;
  DFM_CUDA_TRY(cudaMemcpyAsync(c->d_status, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return DFM_OK;
}

int dfm_ctx_wait_selftest(dfm_ctx c, unsigned long long limit_ns) {
  if (!c || limit_ns == 0 || limit_ns > 10000000000ull) return DFM_ERR_INVALID;
  int rc = ilu_wait_selftest(c, limit_ns);
  if (rc) return rc;
  int code = 0, where = 0;
  rc = dfm_ctx_take_error(c, &code, &where);
  if (rc) return rc;
  return code;  // DFM_WAIT_TIMEOUT expected
}

// ------------------------------------------------------------- buffers
int dfm_buf_alloc(dfm_ctx c, size_t bytes, void** out) {
  if (!c || !out) return DFM_ERR_INVALID;
  *out = nullptr;
  DFM_CUDA_TRY(cudaSetDevice(c->device));
  DFM_CUDA_TRY(cudaMalloc(out, bytes ? bytes : 1));
  return DFM_OK;
}

int dfm_buf_free(dfm_ctx c, void* p) {
  if (!c) return DFM_ERR_INVALID;
  if (!p) return DFM_OK;
  DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  DFM_CUDA_TRY(cudaFree(p));
  return DFM_OK;
}

int dfm_buf_copy(dfm_ctx c, void* dst, const void* src, size_t bytes, int dir) {
  if (!c || (bytes && (!dst || !src)) || dir < DFM_H2D || dir > DFM_D2D) return DFM_ERR_INVALID;
  if (!bytes) return DFM_OK;
  const cudaMemcpyKind k =
      dir == DFM_H2D ? cudaMemcpyHostToDevice : dir == DFM_D2H ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  DFM_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, k, c->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return DFM_OK;
}

int dfm_buf_zero(dfm_ctx c, void* p, size_t bytes) {
  if (!c || (bytes && !p)) return DFM_ERR_INVALID;
  if (!bytes) return DFM_OK;
  DFM_CUDA_TRY(cudaMemsetAsync(p, 0, bytes, c->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return DFM_OK;
}

// ------------------------------------------------------------------ matrix
int dfm_mat_create(dfm_ctx c, unsigned N, unsigned b, int vt, const unsigned* rowptr, const unsigned* colind,
                   dfm_mat* out) {
  if (!c || !out || !rowptr) return DFM_ERR_INVALID;
  *out = nullptr;
  if (vt != DFM_REAL && vt != DFM_COMPLEX) return DFM_ERR_INVALID;
  if (vt == DFM_REAL && (b < 1 || b > 3)) return DFM_ERR_UNSUPPORTED;
  if (vt == DFM_COMPLEX && b != 1) return DFM_ERR_UNSUPPORTED;
  if (rowptr[0] != 0) return DFM_ERR_INVALID;
  for (unsigned i = 0; i < N; i++)
    if (rowptr[i + 1] < rowptr[i]) return DFM_ERR_INVALID;
  const unsigned ncrs = rowptr[N];
  if (ncrs && !colind) return DFM_ERR_INVALID;
  for (unsigned i = 0; i < N; i++)
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
      if (colind[s] >= N || colind[s] == i) return DFM_ERR_INVALID;
      if (s > rowptr[i] && colind[s] <= colind[s - 1]) return DFM_ERR_INVALID;
    }
  cudaSetDevice(c->device);
  dfm_mat A = new (std::nothrow) dfm_mat_s();
  if (!A) return DFM_ERR_NOMEM;
  A->ctx = c;
  ctx_retain(c);
  A->N = N;
  A->b = b;
  A->vt = vt;
  A->ncrs = ncrs;
  A->h_rowptr.assign(rowptr, rowptr + N + 1);
  A->h_colind.assign(colind, colind + ncrs);
  for (unsigned i = 0; i < N; i++) A->max_row = std::max(A->max_row, rowptr[i + 1] - rowptr[i]);
  // kArrayPad spare elements: the TMA-staged SpMV rounds its bulk copies out to 16 bytes
  int rc = dalloc(&A->d_rowptr, N + 1 + kArrayPad);
  if (!rc) rc = dalloc(&A->d_colind, ncrs + kArrayPad);
  if (!rc) rc = dalloc(&A->d_diag, (size_t)N * A->vw() + kArrayPad);
  if (!rc) rc = dalloc(&A->d_off, (size_t)ncrs * A->vw() + kArrayPad);
  if (!rc) rc = copy_in(A->d_rowptr, rowptr, sizeof(unsigned) * (N + 1), DFM_HOST, c->stream);
  if (!rc) rc = copy_in(A->d_colind, colind, sizeof(unsigned) * ncrs, DFM_HOST, c->stream);
  if (!rc) rc = dfm_mat_set_zero(A);
  if (rc) { dfm_mat_destroy(A); return rc; }
  *out = A;
  return DFM_OK;
}

int dfm_mat_destroy(dfm_mat A) {
  if (!A) return DFM_OK;
  cudaStreamSynchronize(A->ctx->stream);
  solve_release_mat(A);
  cudaFree(A->d_rowptr);
  cudaFree(A->d_colind);
  cudaFree(A->d_diag);
  cudaFree(A->d_off);
  cudaFree(A->d_diag32);
  cudaFree(A->d_off32);
  spmv_free_tiles(A);
  dfm_ctx c = A->ctx;
  delete A;
  ctx_release(c);
  return DFM_OK;
}

int dfm_mat_info(dfm_mat A, unsigned* N, unsigned* b, unsigned* ncrs, int* vt) {
  if (!A) return DFM_ERR_INVALID;
  if (N) *N = A->N;
  if (b) *b = A->b;
  if (ncrs) *ncrs = A->ncrs;
  if (vt) *vt = A->vt;
  return DFM_OK;
}

int dfm_mat_set_zero(dfm_mat A) {
  if (!A) return DFM_ERR_INVALID;
  cudaStream_t s = A->ctx->stream;
  DFM_CUDA_TRY(cudaMemsetAsync(A->d_diag, 0, sizeof(double) * A->vw() * std::max(A->N, 1u), s));
  DFM_CUDA_TRY(cudaMemsetAsync(A->d_off, 0, sizeof(double) * A->vw() * std::max(A->ncrs, 1u), s));
  return DFM_OK;
}

int dfm_mat_set_values(dfm_mat A, const double* diag, const double* off, int where) {
  if (!A) return DFM_ERR_INVALID;
  int rc = copy_in(A->d_diag, diag, sizeof(double) * A->vw() * A->N, where, A->ctx->stream);
  if (!rc) rc = copy_in(A->d_off, off, sizeof(double) * A->vw() * A->ncrs, where, A->ctx->stream);
  return rc;
}

int dfm_mat_get_values(dfm_mat A, double* diag, double* off, int where) {
  if (!A) return DFM_ERR_INVALID;
  int rc = DFM_OK;
  if (diag) rc = copy_out(diag, A->d_diag, sizeof(double) * A->vw() * A->N, where, A->ctx->stream);
  if (!rc && off) rc = copy_out(off, A->d_off, sizeof(double) * A->vw() * A->ncrs, where, A->ctx->stream);
  return rc;
}

int dfm_mat_values_device(dfm_mat A, double** diag, double** off) {
  if (!A) return DFM_ERR_INVALID;
  if (diag) *diag = A->d_diag;
  if (off) *off = A->d_off;
  return DFM_OK;
}

int dfm_mat_set_spmv_lanes(dfm_mat A, int lanes) {
  if (!A) return DFM_ERR_INVALID;
  if (lanes != 0 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) return DFM_ERR_INVALID;
  A->lanes = lanes;
  return DFM_OK;
}

int dfm_mat_set_spmv_kernel(dfm_mat A, int kernel) {
  if (!A || kernel < 0 || kernel > 3) return DFM_ERR_INVALID;
  if (kernel >= 1 && A->vt != DFM_REAL) return DFM_ERR_UNSUPPORTED;
  A->spmv_kind = kernel;
  return DFM_OK;
}

int dfm_mat_get_spmv_kernel(dfm_mat A, int* kernel) {
  if (!A || !kernel) return DFM_ERR_INVALID;
  *kernel = A->spmv_kind;
  return DFM_OK;
}

int dfm_mat_get_spmv_lanes(dfm_mat A, int* lanes) {
  if (!A || !lanes) return DFM_ERR_INVALID;
  *lanes = A->lanes;
  return DFM_OK;
}

int dfm_spmv(dfm_mat A, double alpha, const double* x, double beta, double* y) {
  if (!A || (!x && A->N) || (!y && A->N)) return DFM_ERR_INVALID;
  int rc = spmv_autotune(A);
  if (rc) return rc;
  rc = spmv_launch(A, alpha, x, beta, y, nullptr, 0, nullptr, A->lanes);
  if (rc) return rc;
  DFM_CUDA_TRY(cudaStreamSynchronize(A->ctx->stream));
  return DFM_OK;
}

int dfm_time_spmv(dfm_mat A, const double* x, double* y, int reps, float* ms) {
  if (!A || !ms || reps <= 0 || (A->N && (!x || !y))) return DFM_ERR_INVALID;
  int rc = spmv_autotune(A);
  if (rc) return rc;
  return time_launches(A->ctx->stream, reps, ms,
                       [&] { return spmv_launch(A, 1.0, x, 0.0, y, nullptr, 0, nullptr, A->lanes); });
}

// -------------------------------------------------------------------- ILU
int dfm_ilu_create(dfm_mat A, dfm_ilu* out) {
  if (!A || !out) return DFM_ERR_INVALID;
  *out = nullptr;
  dfm_ilu M = new (std::nothrow) dfm_ilu_s();
  if (!M) return DFM_ERR_NOMEM;
  M->ctx = A->ctx;
  ctx_retain(M->ctx);
  M->A = A;
  M->user = A;
  M->N = A->N;
  M->b = A->b;
  M->ncrs = A->ncrs;
  M->vt = A->vt;
  const unsigned N = A->N;
  M->h_diaind.resize(N);
  for (unsigned i = 0; i < N; i++) {  // CMatDiaFrac_BlkCrs ctor, src/matvec/matdiafrac_blkcrs.cpp:263-278
    M->h_diaind[i] = A->h_rowptr[i + 1];
    for (unsigned s = A->h_rowptr[i]; s < A->h_rowptr[i + 1]; s++)
      if (A->h_colind[s] > i) { M->h_diaind[i] = s; break; }
  }
  std::vector<unsigned> of, ob, lf, lb;
  M->nlev_f = make_levels(N, A->h_rowptr, A->h_colind, M->h_diaind, true, M->lev_f, of, lf);
  M->nlev_b = make_levels(N, A->h_rowptr, A->h_colind, M->h_diaind, false, M->lev_b, ob, lb);
  cudaStream_t s = A->ctx->stream;
  int rc = dalloc(&M->d_diaind, N);
  if (!rc) rc = dalloc(&M->d_order_f, N);
  if (!rc) rc = dalloc(&M->d_order_b, N);
  if (!rc) rc = dalloc(&M->d_lvl_f, lf.size());
  if (!rc) rc = dalloc(&M->d_lvl_b, lb.size());
  if (!rc) rc = dalloc(&M->d_fdiag, (size_t)N * M->vw());
  if (!rc) rc = dalloc(&M->d_foff, (size_t)M->ncrs * M->vw());
  if (!rc) rc = dalloc(&M->d_flags, N);
  if (!rc) rc = dalloc(&M->d_tmp, (size_t)N * M->xw());
  if (!rc) rc = copy_in(M->d_diaind, M->h_diaind.data(), sizeof(unsigned) * N, DFM_HOST, s);
  if (!rc) rc = copy_in(M->d_order_f, of.data(), sizeof(unsigned) * N, DFM_HOST, s);
  if (!rc) rc = copy_in(M->d_order_b, ob.data(), sizeof(unsigned) * N, DFM_HOST, s);
  if (!rc) rc = copy_in(M->d_lvl_f, lf.data(), sizeof(unsigned) * lf.size(), DFM_HOST, s);
  if (!rc) rc = copy_in(M->d_lvl_b, lb.data(), sizeof(unsigned) * lb.size(), DFM_HOST, s);
  if (!rc && cudaMemsetAsync(M->d_flags, 0, sizeof(unsigned) * std::max(N, 1u), s) != cudaSuccess) rc = DFM_ERR_CUDA;
  if (rc) { dfm_ilu_destroy(M); return rc; }
  *out = M;
  return DFM_OK;
}

int dfm_ilu_destroy(dfm_ilu M) {
  if (!M) return DFM_OK;
  cudaStreamSynchronize(M->ctx->stream);
  solve_release(M);
  sweep_plan_free(&M->plan_f);
  sweep_plan_free(&M->plan_b);
  sweep_plan_free(&M->plan32_f);
  sweep_plan_free(&M->plan32_b);
  cudaFree(M->d_foff32);
  cudaFree(M->d_diaind);
  cudaFree(M->d_order_f);
  cudaFree(M->d_order_b);
  cudaFree(M->d_lvl_f);
  cudaFree(M->d_lvl_b);
  cudaFree(M->d_fdiag);
  cudaFree(M->d_foff);
  cudaFree(M->d_flags);
  cudaFree(M->d_tmp);
  cudaFree(M->d_fillmap);
  if (M->fillpat) dfm_mat_destroy(M->fillpat);
  dfm_ctx c = M->ctx;
  delete M;
  ctx_release(c);
  return DFM_OK;
}

int dfm_ilu_levels(dfm_ilu M, unsigned* nf, unsigned* nb, unsigned* lev_f, unsigned* lev_b) {
  if (!M) return DFM_ERR_INVALID;
  if (nf) *nf = M->nlev_f;
  if (nb) *nb = M->nlev_b;
  if (lev_f) std::copy(M->lev_f.begin(), M->lev_f.end(), lev_f);
  if (lev_b) std::copy(M->lev_b.begin(), M->lev_b.end(), lev_b);
  return DFM_OK;
}

int dfm_ilu_factor(dfm_ilu M, dfm_mat A, unsigned* n_singular) {
  if (!M || !A || A->N != M->N || A->b != M->b || A->vt != M->vt) return DFM_ERR_INVALID;
  // the values must come in the pattern the preconditioner was made for (its size is checked)
  if (A->ncrs != M->user->ncrs) return DFM_ERR_INVALID;
  int rc = ilu_factor_launch(M, A);
  if (rc) return rc;
  DevStatus h = {};
  DFM_CUDA_TRY(cudaMemcpyAsync(&h, M->ctx->d_status, sizeof(h), cudaMemcpyDeviceToHost, M->ctx->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(M->ctx->stream));
  if (n_singular) *n_singular = h.nsing;
  if (h.code) return take_code(M->ctx);
  M->factored = true;
  if (M->vt == DFM_REAL && h.nsing > 10) return DFM_SINGULAR_PIVOT;  // nmax_sing, :774
  return DFM_OK;
}

int dfm_ilu_get_values(dfm_ilu M, double* diag, double* off, int where) {
  if (!M) return DFM_ERR_INVALID;
  int rc = DFM_OK;
  if (diag) rc = copy_out(diag, M->d_fdiag, sizeof(double) * M->vw() * M->N, where, M->ctx->stream);
  if (!rc && off) rc = copy_out(off, M->d_foff, sizeof(double) * M->vw() * M->ncrs, where, M->ctx->stream);
  return rc;
}

int dfm_ilu_set_values(dfm_ilu M, const double* diag, const double* off, int where) {
  if (!M) return DFM_ERR_INVALID;
  int rc = copy_in(M->d_fdiag, diag, sizeof(double) * M->vw() * M->N, where, M->ctx->stream);
  if (!rc) rc = copy_in(M->d_foff, off, sizeof(double) * M->vw() * M->ncrs, where, M->ctx->stream);
  if (!rc) M->factored = true;
  return rc;
}

int dfm_ilu_set_sweep(dfm_ilu M, int mode) {
  if (!M || mode < 0 || mode > 10) return DFM_ERR_INVALID;
  if (mode >= 9) return ilu_set_ranges(M, M->sweep_blocks > 0 ? M->sweep_blocks : M->ctx->nsm, mode == 10, true);
  if (mode >= 3) {
    const bool merge = mode == 5 || mode == 6 || mode == 8, nb = mode == 4 || mode == 6, pipe = mode >= 7;
    const int rc = ilu_set_ranges(M, M->sweep_blocks > 0 ? M->sweep_blocks : M->ctx->nsm, merge);
    if (rc) return rc;
    if (nb && !(M->plan_f.nb_ok && M->plan_b.nb_ok)) return DFM_ERR_UNSUPPORTED;
    M->plan_f.nb = M->plan_b.nb = nb;
    M->plan_f.pipe = M->plan_b.pipe = pipe;
    return DFM_OK;
  }
  M->sweep = mode;
  M->plan_gen++;
  return DFM_OK;
}

int dfm_ilu_set_sweep_warps(dfm_ilu M, int compute_warps, int lanes, int producer_warps) {
  if (!M || (compute_warps != 1 && compute_warps != 2 && compute_warps != 4) ||
      (lanes != 2 && lanes != 4 && lanes != 8) || producer_warps < 1 || compute_warps + producer_warps > 16)
    return DFM_ERR_INVALID;
  if (M->sweep != 3 || !M->plan_f.halo) return DFM_ERR_INVALID;  // mode 9 only
  for (SweepPlan* P : {&M->plan_f, &M->plan_b, &M->plan32_f, &M->plan32_b}) {
    P->cw = compute_warps;
    P->lpr = lanes;
    P->hw = producer_warps;
  }
  M->plan_gen++;  // captured solves hold the old launch shape
  return DFM_OK;
}

int dfm_ilu_get_sweep_warps(dfm_ilu M, int* compute_warps, int* lanes, int* producer_warps) {
  if (!M || !compute_warps || !lanes || !producer_warps) return DFM_ERR_INVALID;
  if (M->sweep != 3 || !M->plan_f.halo) return DFM_ERR_INVALID;
  *compute_warps = M->plan_f.cw;
  *lanes = M->plan_f.lpr;
  *producer_warps = M->plan_f.hw;
  return DFM_OK;
}

int dfm_ilu_set_sweep_tuning(dfm_ilu M, int max_blocks, unsigned poll_sleep_ns) {
  if (!M || max_blocks < 0 || poll_sleep_ns > 100000) return DFM_ERR_INVALID;
  M->sweep_blocks = max_blocks;
  M->plan_gen++;
  return set_poll_sleep(poll_sleep_ns);
}

int dfm_ilu_set_sweep_partition(dfm_ilu M, const unsigned* part, unsigned nparts) {
  if (!M) return DFM_ERR_INVALID;
  if (part) {
    if (nparts == 0 || nparts > (unsigned)M->ctx->nsm) return DFM_ERR_INVALID;  // one co-resident CTA per part
    for (unsigned i = 0; i < M->N; i++)
      if (part[i] >= nparts) return DFM_ERR_INVALID;
  }
  DFM_CUDA_TRY(cudaStreamSynchronize(M->ctx->stream));
  solve_release(M);  // captured solves hold the old plans
  sweep_plan_free(&M->plan_f);
  sweep_plan_free(&M->plan_b);
  sweep_plan_free(&M->plan32_f);
  sweep_plan_free(&M->plan32_b);
  if (part) {
    M->part_of.assign(part, part + M->N);
    M->nparts = nparts;
  } else {
    M->part_of.clear();
    M->nparts = 0;
  }
  M->sweep = 0;  // autotuned again on next use
  M->plan_gen++;
  return DFM_OK;
}

int dfm_ilu_get_sweep(dfm_ilu M, int* mode) {
  if (!M || !mode) return DFM_ERR_INVALID;
  *mode = M->sweep;
  if (M->sweep == 3 && M->plan_f.halo)
    *mode = M->plan_f.merged ? 10 : 9;
  else if (M->sweep == 3)
    *mode = M->plan_f.pipe ? (M->plan_f.merged ? 8 : 7) : (M->plan_f.merged ? 5 : 3) + (M->plan_f.nb ? 1 : 0);
  return DFM_OK;
}

int dfm_ilu_apply(dfm_ilu M, const double* r, double* z) {
  if (!M || (M->N && (!r || !z)) || r == z) return DFM_ERR_INVALID;
  int rc = ilu_autotune(M);
  if (rc) return rc;
  const size_t n = (size_t)M->N * M->xw();
  if ((rc = ilu_fill_sentinel(M, M->d_tmp, n))) return rc;
  if ((rc = ilu_fill_sentinel(M, z, n))) return rc;
  if ((rc = ilu_fwd_launch(M, r, M->d_tmp, nullptr, M->sweep))) return rc;
  if ((rc = ilu_bwd_launch(M, M->d_tmp, z, nullptr, nullptr, nullptr, M->sweep))) return rc;
  return take_code(M->ctx);
}

int dfm_time_ilu_apply(dfm_ilu M, const double* r, double* z, int reps, float* ms) {
  if (!M || !ms || reps <= 0 || (M->N && (!r || !z)) || r == z) return DFM_ERR_INVALID;
  int rc = ilu_autotune(M);
  if (rc) return rc;
  const size_t n = (size_t)M->N * M->xw();
  rc = time_launches(M->ctx->stream, reps, ms, [&] {
    int q = ilu_fill_sentinel(M, M->d_tmp, n);
    if (!q) q = ilu_fill_sentinel(M, z, n);
    if (!q) q = ilu_fwd_launch(M, r, M->d_tmp, nullptr, M->sweep);
    if (!q) q = ilu_bwd_launch(M, M->d_tmp, z, nullptr, nullptr, nullptr, M->sweep);
    return q;
  });
  if (rc) return rc;
  return take_code(M->ctx);
}

// ---------------------------------------------------------------- solvers
static int solve_args(dfm_mat A, dfm_ilu M, int method, const void* b, const void* x) {
  if (!A || !M || M->user != A || (A->N && (!b || !x))) return DFM_ERR_INVALID;
  const bool cplx = method == DFM_PCOCG || method == DFM_PCOCG_MIXED;
  if (cplx ? A->vt != DFM_COMPLEX : A->vt != DFM_REAL) return DFM_ERR_INVALID;
  if (!M->factored) return DFM_ERR_INVALID;
  return DFM_OK;
}

int dfm_solve_pcg(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit, unsigned* iters,
                  double* conv) {
  const int rc = solve_args(A, M, DFM_PCG, r, x);
  if (rc) return rc;
  return krylov_solve(A, M, DFM_PCG, r, DFM_DEVICE, x, DFM_DEVICE, r, tol, maxit, iters, conv);
}

int dfm_solve_pbicgstab(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit, unsigned* iters,
                        double* conv) {
  const int rc = solve_args(A, M, DFM_PBICGSTAB, r, x);
  if (rc) return rc;
  return krylov_solve(A, M, DFM_PBICGSTAB, r, DFM_DEVICE, x, DFM_DEVICE, r, tol, maxit, iters, conv);
}

int dfm_solve_pcocg(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit, unsigned* iters,
                    double* conv) {
  const int rc = solve_args(A, M, DFM_PCOCG, r, x);
  if (rc) return rc;
  return krylov_solve(A, M, DFM_PCOCG, r, DFM_DEVICE, x, DFM_DEVICE, r, tol, maxit, iters, conv);
}

int dfm_solve_pcg_mixed(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit, unsigned* iters,
                        double* conv) {
  const int rc = solve_args(A, M, DFM_PCG_MIXED, r, x);
  if (rc) return rc;
  return krylov_solve(A, M, DFM_PCG_MIXED, r, DFM_DEVICE, x, DFM_DEVICE, r, tol, maxit, iters, conv);
}

int dfm_solve_pcocg_mixed(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit, unsigned* iters,
                          double* conv) {
  const int rc = solve_args(A, M, DFM_PCOCG_MIXED, r, x);
  if (rc) return rc;
  return krylov_solve(A, M, DFM_PCOCG_MIXED, r, DFM_DEVICE, x, DFM_DEVICE, r, tol, maxit, iters, conv);
}

int dfm_solve_cg(dfm_mat A, double* r, double* x, double tol, unsigned maxit, unsigned* iters, double* conv) {
  if (!A || A->vt != DFM_REAL || (A->N && (!r || !x))) return DFM_ERR_INVALID;
  return krylov_solve(A, nullptr, DFM_CG, r, DFM_DEVICE, x, DFM_DEVICE, r, tol, maxit, iters, conv);
}

int dfm_solve_host(dfm_mat A, dfm_ilu M, int method, const double* b_host, double* x_host, double tol,
                   unsigned maxit, unsigned* iters, double* conv) {
  if (method == DFM_CG) {
    if (!A || A->vt != DFM_REAL || (A->N && (!b_host || !x_host))) return DFM_ERR_INVALID;
    return krylov_solve(A, nullptr, DFM_CG, b_host, DFM_HOST, x_host, DFM_HOST, nullptr, tol, maxit, iters, conv);
  }
  if (method < DFM_PCG || method > DFM_PCOCG_MIXED) return DFM_ERR_INVALID;
  const int rc = solve_args(A, M, method, b_host, x_host);
  if (rc) return rc;
  return krylov_solve(A, M, method, b_host, DFM_HOST, x_host, DFM_HOST, nullptr, tol, maxit, iters, conv);
}

int dfm_solve_pcg_host(dfm_mat A, dfm_ilu M, const double* b_host, double* x_host, double tol, unsigned maxit,
                       unsigned* iters, double* conv) {
  return dfm_solve_host(A, M, DFM_PCG, b_host, x_host, tol, maxit, iters, conv);
}

}  // extern "C"
