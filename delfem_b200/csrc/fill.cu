// ILU(k): the factor in its own, filled pattern.
//
// CPreconditioner_ILU::SetFillInLevel(lev) + SetLinearSystem
// (src/ls/preconditioner.cpp:57-212) builds CMatDiaFrac_BlkCrs(lev, A), whose
// pattern is A's plus the fill entries of CMatDiaFrac_BlkCrs::AddFracPtn
// (src/matvec/matdiafrac_blkcrs.cpp:1249-1377); SetValue_Initialize
// (include/delfem/matvec/matdiafrac_blkcrs.h:90-117) then copies A's values
// into it (zero elsewhere) and DoILUDecomp factors it over that pattern.
//
// Here the fill pattern is computed on the host, once, and held by an
// internal pattern-only matrix that the ILU object's factor, level sets and
// sweep plans use exactly as they use A's pattern for ILU(0); the numeric
// factor starts from a device scatter of A's blocks through a precomputed
// slot map, then runs the same factor kernel.
#include <algorithm>
#include <new>

#include "dfm_internal.h"

namespace dfm {

// The fill pattern, row by row.  Row i starts from A's entries (level 0).  Its
// entries k < i are taken as pivots in ascending order - fill entries too, as
// they are added - when lev(i,k) + 1 <= lev; each such pivot adds every j of
// row k's upper part (already final) with lev(k,j) + 1 <= lev and j != i, at
// level max(lev(i,k), lev(k,j)) + 1.  An entry that row i holds already keeps
// the level it has (AddFracPtn's sorted list inserts only new columns, see
// CListRLN::Insert in include/delfem/matvec/matdiafrac_blkcrs.h:207-257), so
// a column's level is that of the first pivot reaching it.  lev = -1: no limit.
// Rows flagged in `unl` (CPreconditioner_ILU::SetFillBlk, AddFracPtn(lev,
// aBlkFill), src/matvec/matdiafrac_blkcrs.cpp:1379-1500) lift the limit: a
// candidate (i, j) with i, j < bound is kept at any level when row i or row j
// is flagged, so a pivot cannot be skipped on its own level in a row that may
// take such fill.  `bound` is the first segment's row count in a joined
// multi-segment system (only that segment's diagonal matrix gets the list).
// The row is a linked list over column numbers; `level[c]` is kNone for
// columns not in it.
int ilu_fill_pattern(unsigned N, const std::vector<unsigned>& rp, const std::vector<unsigned>& ci, int lev,
                     std::vector<unsigned>& frp, std::vector<unsigned>& fci, const std::vector<unsigned char>& unl,
                     unsigned bound) {
  constexpr unsigned kNone = 0xffffffffu;
  const size_t ncrs = rp[N];
  frp.assign(N + 1, 0);
  fci.clear();
  const bool dense = N > 0 && ncrs == (size_t)N * (N - 1);
  const bool flags = !unl.empty();
  if ((lev == 0 && !flags) || ncrs == 0 || dense) {  // AddFracPtn returns at once
    fci.assign(ci.begin(), ci.begin() + ncrs);
    frp = rp;
    return DFM_OK;
  }
  std::vector<unsigned> flev, upper(N);  // levels of the final entries; first upper slot per row
  fci.reserve(ncrs * 2);
  flev.reserve(ncrs * 2);
  std::vector<unsigned> level(N, kNone), next(N, kNone);
  const auto within = [lev](unsigned l) { return lev < 0 || l + 1 <= (unsigned)lev; };
  for (unsigned i = 0; i < N; i++) {
    unsigned head = kNone, last = kNone;
    for (size_t s = rp[i]; s < rp[i + 1]; s++) {
      const unsigned c = ci[s];
      level[c] = 0;
      next[c] = kNone;
      (last == kNone ? head : next[last]) = c;
      last = c;
    }
    const bool may_flag = flags && i < bound, flag_i = may_flag && unl[i];
    for (unsigned k = head; k != kNone; k = next[k]) {
      const unsigned lik = level[k];
      if (!may_flag && !within(lik)) continue;
      if (k >= i) break;
      unsigned at = k;  // insertion point: every new column lies after k
      for (size_t s = upper[k]; s < frp[k + 1]; s++) {
        const unsigned lkj = flev[s], j = fci[s];
        const bool free_ij = may_flag && j < bound && (flag_i || unl[j]);
        if (!(free_ij || within(std::max(lik, lkj))) || j == i || level[j] != kNone) continue;
        while (next[at] != kNone && next[at] < j) at = next[at];
        next[j] = next[at];
        next[at] = j;
        level[j] = std::max(lik, lkj) + 1;
        at = j;
      }
    }
    upper[i] = kNone;
    for (unsigned c = head; c != kNone; c = next[c]) {
      if (upper[i] == kNone && c > i) upper[i] = (unsigned)fci.size();
      fci.push_back(c);
      flev.push_back(level[c]);
      level[c] = kNone;
    }
    if (fci.size() > 0xfffffff0u) return DFM_ERR_NOMEM;  // slots are 32-bit
    frp[i + 1] = (unsigned)fci.size();
    if (upper[i] == kNone) upper[i] = frp[i + 1];
  }
  return DFM_OK;
}

// foff[map[s]] = off[s], one b*b block per A slot (the rest of foff is zero)
__global__ void k_fill_scatter(size_t ncrs, unsigned vw, const unsigned* __restrict__ map,
                               const double* __restrict__ off, double* __restrict__ foff) {
  const size_t n = ncrs * vw;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t s = e / vw, q = e - s * vw;
    foff[(size_t)map[s] * vw + q] = off[e];
  }
}

int ilu_fill_values(dfm_ilu M, dfm_mat A) {
  cudaStream_t s = M->ctx->stream;
  const size_t vw = M->vw();
  DFM_CUDA_TRY(cudaMemsetAsync(M->d_foff, 0, sizeof(double) * vw * M->ncrs, s));
  if (A->ncrs == 0) return DFM_OK;
  const size_t n = (size_t)A->ncrs * vw;
  const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)M->ctx->nsm * 8);
  k_fill_scatter<<<grid, 256, 0, s>>>(A->ncrs, (unsigned)vw, M->d_fillmap, A->d_off, M->d_foff);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

}  // namespace dfm

using namespace dfm;

extern "C" {

int dfm_ilu_create_fill(dfm_mat A, int lev, dfm_ilu* out) { return dfm_ilu_create_fill_rows(A, lev, nullptr, 0, 0, out); }

int dfm_ilu_create_fill_rows(dfm_mat A, int lev, const unsigned* rows, size_t nrows, unsigned bound, dfm_ilu* out) {
  if (!A || !out || lev < -1 || (nrows && !rows)) return DFM_ERR_INVALID;
  *out = nullptr;
  std::vector<unsigned char> unl;
  if (nrows) {
    if (bound == 0 || bound > A->N) return DFM_ERR_INVALID;
    unl.assign(A->N, 0);
    for (size_t t = 0; t < nrows; t++) {
      if (rows[t] >= bound) return DFM_ERR_INVALID;
      unl[rows[t]] = 1;
    }
  }
  if (lev == 0 && !nrows) return dfm_ilu_create(A, out);
  // complex matrices: CZPreconditioner_ILU::SetFillInLevel, whose fill pattern
  // (CZMatDiaFrac_BlkCrs::AddFracPtn, src/matvec/zmatdiafrac_blkcrs.cpp:263-441)
  // is the real one's
  std::vector<unsigned> frp, fci;
  int rc = ilu_fill_pattern(A->N, A->h_rowptr, A->h_colind, lev, frp, fci, unl, bound);
  if (rc) return rc;
  // the pattern-only matrix that the factor, level sets and sweep plans use
  dfm_mat P = new (std::nothrow) dfm_mat_s();
  if (!P) return DFM_ERR_NOMEM;
  dfm_ctx c = A->ctx;
  P->ctx = c;
  ctx_retain(c);
  P->N = A->N;
  P->b = A->b;
  P->vt = A->vt;
  P->ncrs = frp[A->N];
  P->h_rowptr = std::move(frp);
  P->h_colind = std::move(fci);
  for (unsigned i = 0; i < P->N; i++) P->max_row = std::max(P->max_row, P->h_rowptr[i + 1] - P->h_rowptr[i]);
  std::vector<unsigned> map(A->ncrs);
  for (unsigned i = 0; i < A->N; i++) {  // A's row is a sorted subset of the factor's
    unsigned t = P->h_rowptr[i];
    for (unsigned s = A->h_rowptr[i]; s < A->h_rowptr[i + 1]; s++) {
      while (P->h_colind[t] != A->h_colind[s]) t++;
      map[s] = t;
    }
  }
  cudaSetDevice(c->device);
  rc = dalloc(&P->d_rowptr, P->N + 1 + kArrayPad);
  if (!rc) rc = dalloc(&P->d_colind, P->ncrs + kArrayPad);
  if (!rc) rc = copy_in(P->d_rowptr, P->h_rowptr.data(), sizeof(unsigned) * (P->N + 1), DFM_HOST, c->stream);
  if (!rc) rc = copy_in(P->d_colind, P->h_colind.data(), sizeof(unsigned) * P->ncrs, DFM_HOST, c->stream);
  dfm_ilu M = nullptr;
  if (!rc) rc = dfm_ilu_create(P, &M);
  if (rc) {
    dfm_mat_destroy(P);
    return rc;
  }
  M->user = A;
  M->fillpat = P;
  M->fill_level = lev;
  rc = dalloc(&M->d_fillmap, std::max<size_t>(A->ncrs, 1));
  if (!rc) rc = copy_in(M->d_fillmap, map.data(), sizeof(unsigned) * A->ncrs, DFM_HOST, c->stream);
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = DFM_ERR_CUDA;
  if (rc) {
    dfm_ilu_destroy(M);
    return rc;
  }
  *out = M;
  return DFM_OK;
}

int dfm_ilu_pattern(dfm_ilu M, unsigned* rowptr, unsigned* colind, unsigned* ncrs) {
  if (!M) return DFM_ERR_INVALID;
  const dfm_mat P = M->A;
  if (ncrs) *ncrs = P->ncrs;
  if (rowptr) std::copy(P->h_rowptr.begin(), P->h_rowptr.end(), rowptr);
  if (colind) std::copy(P->h_colind.begin(), P->h_colind.end(), colind);
  return DFM_OK;
}

}  // extern "C"
