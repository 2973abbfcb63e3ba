// The stored boundary matrix of Fem::Ls::CLinearSystem_Save
// (include/delfem/femls/linearsystem_fieldsave.h:59-97,
// src/femls/linearsystem_fieldsave.cpp:64-260), host only.
//
// CLinearSystem_Save keeps, beside the eliminated system, a matrix B with the
// pattern CMat_BlkCrs::SetPatternBoundary gives it (src/matvec/mat_blkcrs.cpp:
// 1177-1265: block rows with at least one free DOF, block columns with at
// least one fixed DOF), filled by the same element matrices as K (so its
// entries are K's values before the Dirichlet elimination), then masked by
// SetBoundaryConditionInverse_Colum (free columns zeroed, :876-907) and
// SetBoundaryCondition_Row (fixed rows zeroed, :910-951).  MakeResidual
// (src/femls/linearsystem_fieldsave.cpp:206-246) is then r = Force - B u: with
// B in this library's block-CRS layout that product is dfm_spmv(B, -1, u, 1, r)
// with r holding Force.
//
// Here B is built from K's values (before dfm_apply_dirichlet) in the
// library's layout: the same off-diagonal entries in the same (ascending)
// column order as the reference's pattern, the diagonal block in the separate
// diagonal array (the reference lists it first in its row; its masked values
// are the same, and a block it leaves out is all zero here).
#include "dfm_internal.h"

extern "C" {

int dfm_boundary_matrix(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind, const double* diag,
                        const double* off, const int* flags, unsigned* brow, unsigned* bcol, double* bdiag,
                        double* boff, unsigned* bncrs) {
  if (!rowptr || !flags || !bncrs || b < 1 || (N && (!diag)) || rowptr[0] != 0) return DFM_ERR_INVALID;
  const unsigned ncrs = rowptr[N];
  if (ncrs && (!colind || !off)) return DFM_ERR_INVALID;
  std::vector<char> free_any(N, 0), fixed_any(N, 0);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) {
      if (flags[(size_t)i * b + d] == 0) free_any[i] = 1;
      else fixed_any[i] = 1;
    }
  for (unsigned i = 0; i < N; i++) {
    if (rowptr[i + 1] < rowptr[i]) return DFM_ERR_INVALID;
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++)
      if (colind[s] >= N || colind[s] == i) return DFM_ERR_INVALID;
  }
  unsigned nb = 0;
  for (unsigned i = 0; i < N; i++) {
    if (!free_any[i]) continue;
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++)
      if (fixed_any[colind[s]]) nb++;
  }
  *bncrs = nb;
  if (!brow) return DFM_OK;  // size query
  const size_t bb = (size_t)b * b;
  // kept entry (r, c) of block (i, j): row DOF (i, r) free and column DOF (j, c) fixed
  auto masked = [&](unsigned i, unsigned j, const double* src, double* dst) {
    for (unsigned r = 0; r < b; r++)
      for (unsigned c = 0; c < b; c++)
        dst[r * b + c] = (flags[(size_t)i * b + r] == 0 && flags[(size_t)j * b + c] != 0) ? src[r * b + c] : 0.0;
  };
  unsigned k = 0;
  brow[0] = 0;
  for (unsigned i = 0; i < N; i++) {
    if (bdiag) masked(i, i, diag + i * bb, bdiag + i * bb);
    if (free_any[i])
      for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
        const unsigned j = colind[s];
        if (!fixed_any[j]) continue;
        if (bcol) bcol[k] = j;
        if (boff) masked(i, j, off + (size_t)s * bb, boff + (size_t)k * bb);
        k++;
      }
    brow[i + 1] = k;
  }
  return DFM_OK;
}

}  // extern "C"
