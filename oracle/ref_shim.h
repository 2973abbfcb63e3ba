/* C-ABI shim over the reference's own CPU linear-solve path (DelFEM, built from
 * its sources by oracle/Makefile into oracle/_ref/libdfm_refshim.so).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker and the timed CPU
 * baseline; nothing in the product (delfem_b200/) links or calls it.
 *
 * Two levels:
 *  - field level: a mesh goes through Fem::Field::CFieldWorld::AddMesh,
 *    Fem::Ls::CLinearSystem_Field / CZLinearSystem, LsSol::CPreconditioner_ILU /
 *    CZPreconditioner_ILU and LsSol::Solve_PCG / Solve_PBiCGSTAB /
 *    Fem::Ls::Solve_PCOCG, in the call order of
 *    src/femeqn/eqnsys_scalar.cpp:213-359 and test_glut/helmholtz2d/main.cpp:82-121;
 *  - matrix level: arbitrary block-CRS arrays go into MatVec::CMatDia_BlkCrs /
 *    CMatDiaFrac_BlkCrs and LsSol::CLinearSystem directly.
 *
 * Array layout everywhere is the reference's: rowptr[N+1] (m_colInd_Blk),
 * colind[ncrs] (m_rowPtr_Blk, off-diagonal only, ascending per row), diagonal
 * blocks diag[N*b*b], off-diagonal blocks off[ncrs*b*b], each block row-major.
 * Complex values are interleaved (re, im) doubles.
 * All functions return 0 on success, non-zero on failure. */
#ifndef DFM_REF_SHIM_H
#define DFM_REF_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif

enum {
  DFM_REF_POISSON2D = 1,   /* Fem::Eqn::AddLinSys_Poisson, P1 triangles, b=1      */
  DFM_REF_SOLID2D = 2,     /* Fem::Eqn::AddLinSys_LinearSolid2D_Static, P1, b=2   */
  DFM_REF_SOLID3D = 3,     /* Fem::Eqn::AddLinSys_LinearSolid3D_Static, P1 tet, b=3 */
  DFM_REF_HELMHOLTZ2D = 4  /* Fem::Eqn::AddLinSys_Helmholtz + SommerfeltRadiationBC, complex b=1 */
};
enum { DFM_REF_PCG = 0, DFM_REF_PBICGSTAB = 1, DFM_REF_PCOCG = 2, DFM_REF_CG = 3 /* matrix level only */ };

typedef struct dfm_ref_sys dfm_ref_sys;

/* Mesh: coord[nnode*ndim]; elem[nelem*nnoel] (TRI nnoel=3, TET nnoel=4);
 * bnd[nbnd*bnd_nnoel] (BAR 2 / TRI 3, or nbnd=0).  The boundary array is a
 * Dirichlet partial field (all DOFs fixed) for the real kinds and carries the
 * Sommerfeld radiation condition for DFM_REF_HELMHOLTZ2D. */
dfm_ref_sys* dfm_ref_create(int kind, int ndim, int nnode, const double* coord,
                            int nnoel, int nelem, const int* elem,
                            int bnd_nnoel, int nbnd, const int* bnd);
void dfm_ref_destroy(dfm_ref_sys* s);
int dfm_ref_dims(const dfm_ref_sys* s, unsigned* N, unsigned* b, unsigned* ncrs);
int dfm_ref_pattern(const dfm_ref_sys* s, unsigned* rowptr, unsigned* colind);
/* params: POISSON2D {alpha, source}; SOLID2D {lambda, myu, rho, gx, gy};
 * SOLID3D {lambda, myu, rho, gx, gy, gz}; HELMHOLTZ2D {wave_length}.
 * elem_coef (may be NULL; POISSON2D/SOLID2D only): per-element multiplier of the
 * element matrix, assembled by a restatement of the element loop into the
 * reference's own matrix through CMatDia_BlkCrs::Mearge.
 * nodal_load (may be NULL): added to the residual before FinalizeMarge. */
int dfm_ref_assemble(dfm_ref_sys* s, const double* params, const double* elem_coef,
                     const double* nodal_load, double* res_norm, double* seconds);
int dfm_ref_get_system(const dfm_ref_sys* s, double* diag, double* off, double* rhs);
int dfm_ref_get_bcflag(const dfm_ref_sys* s, int* flags);
int dfm_ref_ilu(dfm_ref_sys* s, double* seconds);
int dfm_ref_get_ilu(const dfm_ref_sys* s, double* diag, double* off);
/* Restores r = b (saved after assembly), runs the solver, copies the update x. */
int dfm_ref_solve(dfm_ref_sys* s, int method, double tol, unsigned maxit,
                  unsigned* iters, double* conv, double* x, double* seconds);

/* ---- matrix level (real, fixed block size b) ---- */
int dfm_ref_mat_spmv(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                     const double* diag, const double* off, double alpha, const double* x,
                     double beta, double* y);
/* Returns 0 if DoILUDecomp succeeded, 1 if it gave up (more than 10 singular pivots). */
int dfm_ref_mat_ilu0(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                     const double* diag, const double* off, double* fdiag, double* foff);
int dfm_ref_mat_precond(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                        const double* fdiag, const double* foff, double* vec);
/* CMatDiaFrac_BlkCrs(lev, A): the ILU(lev) fill pattern (AddFracPtn) and,
 * after SetValue_Initialize + DoILUDecomp, the factor in it.  *fncrs gets the
 * pattern's size; with frowptr == NULL or cap < *fncrs nothing else is written
 * and 2 is returned.  Otherwise 0 (1 when DoILUDecomp gave up). */
int dfm_ref_mat_iluk(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                     const double* diag, const double* off, int lev, unsigned cap, unsigned* frowptr,
                     unsigned* fcolind, double* fdiag, double* foff, unsigned* fncrs);
/* The same through CMatDiaFrac_BlkCrs(0, A) + AddFracPtn(lev, aBlkFill) +
 * MakePatternFinalize (the SetFillBlk path) when nrows > 0. */
int dfm_ref_mat_iluk_rows(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                          const double* diag, const double* off, int lev, unsigned nrows, const unsigned* rows,
                          unsigned cap, unsigned* frowptr, unsigned* fcolind, double* fdiag, double* foff,
                          unsigned* fncrs);
/* LsSol::CLinearSystem + CPreconditioner_ILU(0) + Solve_PCG / Solve_PBiCGSTAB.
 * Returns 0 when the solver reported convergence, 3 when it did not, 1 on ILU failure. */
int dfm_ref_mat_solve(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                      const double* diag, const double* off, const double* rhs, int method,
                      double tol, unsigned maxit, unsigned* iters, double* conv, double* x,
                      double* t_ilu, double* t_solve);
/* The same with CPreconditioner_ILU::SetFillInLevel(lev). */
int dfm_ref_mat_solve_lev(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                          const double* diag, const double* off, const double* rhs, int method,
                          double tol, unsigned maxit, int lev, unsigned* iters, double* conv, double* x,
                          double* t_ilu, double* t_solve);

/* ---- matrix level (complex, b = 1) ---- */
int dfm_ref_zmat_spmv(unsigned N, const unsigned* rowptr, const unsigned* colind,
                      const double* diag, const double* off, double alpha, const double* x,
                      double beta, double* y);
/* CZMatDia_BlkCrs(file_path): pattern and values as read by the reference
 * (*N, *ncrs always; the arrays when rowptr != NULL and cap >= *ncrs, else 2). */
int dfm_ref_zmat_read(const char* path, unsigned cap, unsigned* N, unsigned* ncrs, unsigned* rowptr,
                      unsigned* colind, double* diag, double* off);
/* CLinearSystem_Save's boundary matrix over K (values before elimination)
 * and MakeResidual's r = force - B u, computed by the reference's CMat_BlkCrs
 * (SetPatternBoundary, the two BC masks, MatVec).  *bncrs always; B row by row
 * (brow[N+1], bcol, bval, diagonal block first as the reference stores it) when
 * brow != NULL and cap >= *bncrs. */
int dfm_ref_boundary_residual(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                              const double* diag, const double* off, const int* flags, const double* force,
                              const double* u, unsigned cap, unsigned* brow, unsigned* bcol, double* bval,
                              unsigned* bncrs, double* r);
/* Msh::CMesher2D (want2d) or Msh::CMesh3D ReadFromFile_GiDMsh: node
 * coordinates (2 or 3 per node) and the element array, 0-based.  Sizes always;
 * the arrays when coord != NULL and they fit the caps (else 2); 1 when the
 * reference's reader returned false. */
int dfm_ref_gid_read(const char* path, int want2d, unsigned cap_node, unsigned cap_elem, unsigned* nnode,
                     unsigned* nelem, int* nnoel, double* coord, int* elem);
int dfm_ref_gid_boundary(const char* path, int want2d, unsigned cap_facet, unsigned cap_group, unsigned cap_vertex,
                         unsigned* nfacet, unsigned* ngroup, unsigned* nvertex, unsigned* facet, unsigned* group_ptr,
                         unsigned* group_id, unsigned* vertex, unsigned* vertex_id, unsigned* group_ends);
int dfm_ref_zmat_ilu0(unsigned N, const unsigned* rowptr, const unsigned* colind,
                      const double* diag, const double* off, double* fdiag, double* foff);

/* The stored-matrix Newmark systems through the reference's classes:
 * scheme 1 CLinearSystem_SaveDiaM_Newmark + AddLinSys_Diffusion (p = rho,
 * alpha, source; b = 1), scheme 2 CLinearSystem_SaveDiaM_NewmarkBeta +
 * AddLinSys_LinearSolid2D_NonStatic_Save_NewmarkBeta (p = lambda, myu, rho, gx,
 * gy; b = 2) on P1 triangles, the boundary bars fixed.  The field is set from
 * u, v (a), assembled, finalized; out: the stored matrix (library layout over
 * the mesh pattern), force, BC flags, MakeResidual's r and norm.  Then the
 * update vector is set to x and UpdateValueOfField runs: u, v, a and x are
 * overwritten with the field's new state and the final update vector. */
int dfm_ref_newmark(int scheme, int nnode, const double* coord, int nelem, const int* elem, int nbnd,
                    const int* bnd, const double* p, double dt, double gamma, double beta, double* u, double* v,
                    double* a, double* x, double* bdiag, double* boff, double* force, int* flags, double* r,
                    double* norm);

/* Complex ILU(k): CZMatDiaFrac_BlkCrs(lev, A) pattern and factor (as
 * dfm_ref_mat_iluk). */
int dfm_ref_zmat_iluk(unsigned N, const unsigned* rowptr, const unsigned* colind, const double* diag,
                      const double* off, int lev, unsigned cap, unsigned* frowptr, unsigned* fcolind, double* fdiag,
                      double* foff, unsigned* fncrs);
/* The field-level system's preconditioner at fill level lev (SetFillInLevel +
 * SetLinearSystem); factored by the next dfm_ref_ilu. */
int dfm_ref_set_fill(dfm_ref_sys* s, int lev);

/* CMat_BlkCrs::MatVec on a rectangular block matrix (nrow x ncol blocks of
 * brow x bcol), y updated in place. */
int dfm_ref_rmat_spmv(unsigned nrow, unsigned ncol, unsigned brow, unsigned bcol, const unsigned* rowptr,
                      const unsigned* colind, const double* val, double alpha, const double* x, double beta,
                      double* y);

#ifdef __cplusplus
}
#endif
#endif
