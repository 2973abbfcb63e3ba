/* dfm_oracle - plain-C restatement of the reference's linear-solve path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels and the "port"
 * CPU baseline.  It is pinned bit-for-bit against the reference's own code
 * (oracle/_ref/libdfm_refshim.so, built from the DelFEM sources) by
 * tests/test_oracle_pin.py and against the committed fixtures in tests/golden/.
 *
 * Layout: the reference's block-CRS with a separate diagonal
 * (include/delfem/matvec/mat_blkcrs.h:183-185, matdia_blkcrs.h:114):
 * rowptr[N+1], colind[ncrs] (off-diagonal, ascending per row), diag[N*b*b],
 * off[ncrs*b*b], blocks row-major.  Complex values are interleaved (re, im).
 * Block sizes b = 1, 2, 3 (the closed-form paths of the reference). */
#ifndef DFM_ORACLE_H
#define DFM_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Pattern: MakePointSurElem + MakePointSurPoint(isnt_self) + Sort
 * (src/femfield/elem_ary.cpp:225-244, :675-724, :821-892; include/delfem/indexed_array.h:113-131).
 * Call with colind == NULL to get the count in *ncrs. */
int dfo_pattern(int nnode, int nnoel, int nelem, const int* elem, unsigned* rowptr,
                unsigned* colind, unsigned* ncrs);
/* m_DiaInd of CMatDiaFrac_BlkCrs (src/matvec/matdiafrac_blkcrs.cpp:263-278). */
void dfo_diaind(unsigned N, const unsigned* rowptr, const unsigned* colind, unsigned* diaind);
/* ILU(k) symbolic fill: CMatDiaFrac_BlkCrs::AddFracPtn(lev_fill)
 * (src/matvec/matdiafrac_blkcrs.cpp:1249-1377).  frowptr[N+1] is filled; the
 * column and level arrays are allocated here (free with dfo_free).
 * lev_fill = -1: no limit. */
int dfo_iluk_pattern(unsigned N, const unsigned* rowptr, const unsigned* colind, int lev_fill,
                     unsigned* frowptr, unsigned** fcolind, unsigned** flev);
/* AddFracPtn(lev_fill, aBlkFill) (src/matvec/matdiafrac_blkcrs.cpp:1379-1500,
 * CPreconditioner_ILU::SetFillBlk): fill through a listed row, or into one, is
 * kept at any level; flags act on pairs i, j < bound.  -1: a row >= bound. */
int dfo_iluk_pattern_rows(unsigned N, const unsigned* rowptr, const unsigned* colind, int lev_fill,
                          unsigned nrows, const unsigned* rows, unsigned bound, unsigned* frowptr,
                          unsigned** fcolind, unsigned** flev);
void dfo_free(void* p);
/* SetValue_Initialize (include/delfem/matvec/matdiafrac_blkcrs.h:90-117): A's
 * values into the fill pattern, zero elsewhere. */
void dfo_iluk_init(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                   const double* diag, const double* off, const unsigned* frowptr,
                   const unsigned* fcolind, double* fdiag, double* foff);
/* Level sets of the forward (L) and backward (U) sweeps in the natural order:
 * lev_f(i) = 1 + max lev_f(j) over j in L(i) (0 when L(i) is empty),
 * lev_b(i) = 1 + max lev_b(j) over j in U(i).  Returns the number of levels. */
unsigned dfo_levels_fwd(unsigned N, const unsigned* rowptr, const unsigned* colind,
                        const unsigned* diaind, unsigned* lev);
unsigned dfo_levels_bwd(unsigned N, const unsigned* rowptr, const unsigned* colind,
                        const unsigned* diaind, unsigned* lev);

/* Element assembly into (diag, off, res), which the caller zeroes first
 * (CLinearSystem::InitializeMarge, src/ls/linearsystem.cpp:74-88).
 * coef (nullable) multiplies each element matrix (per-element alpha / E);
 * u (nullable) is the current field, res += f_e - K_e u_e. */
void dfo_asm_poisson_tri(const unsigned* rowptr, const unsigned* colind, int nelem,
                         const int* elem, const double* coord, double alpha, double source,
                         const double* coef, const double* u, double* diag, double* off,
                         double* res);
void dfo_asm_solid2d_tri(const unsigned* rowptr, const unsigned* colind, int nelem,
                         const int* elem, const double* coord, double lambda, double myu,
                         double rho, double gx, double gy, const double* coef, const double* u,
                         double* diag, double* off, double* res);
void dfo_asm_solid3d_tet(const unsigned* rowptr, const unsigned* colind, int nelem,
                         const int* elem, const double* coord, double lambda, double myu,
                         double rho, double gx, double gy, double gz, const double* u,
                         double* diag, double* off, double* res);
void dfo_asm_helmholtz_tri(const unsigned* rowptr, const unsigned* colind, int nelem,
                           const int* elem, const double* coord, double wave_length,
                           const double* u, double* diag, double* off, double* res);
void dfo_asm_sommerfeld_bar(const unsigned* rowptr, const unsigned* colind, int nbar,
                            const int* bar, const double* coord, double wave_length,
                            const double* u, double* diag, double* off, double* res);

/* Dirichlet elimination (SetBoundaryCondition, src/matvec/matdia_blkcrs.cpp:261-343)
 * + CBCFlag::SetZeroToBCDof on the residual. flags[N*b], non-zero = fixed. */
void dfo_apply_bc(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                  const int* flags, double* diag, double* off, double* res);

/* y = beta*y + alpha*A x (CMatDia_BlkCrs::MatVec, src/matvec/matdia_blkcrs.cpp:921-1094). */
void dfo_spmv(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
              const double* diag, const double* off, double alpha, const double* x,
              double beta, double* y);
/* In-place ILU(0) numeric factor (DoILUDecomp, src/matvec/matdiafrac_blkcrs.cpp:769-1102).
 * Returns the number of singular pivots; the reference gives up (returns
 * false) when that count exceeds 10, and so does this (return value > 10). */
unsigned dfo_ilu0(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                  const unsigned* diaind, double* diag, double* off);
/* vec <- U^-1 L^-1 vec in place (Forward/BackwardSubstitution, :332-663). */
void dfo_fwd(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
             const unsigned* diaind, const double* fdiag, const double* foff, double* vec);
void dfo_bwd(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
             const unsigned* diaind, const double* foff, double* vec);

/* LsSol::Solve_PCG (src/ls/solver_ls_iter.cpp:100-172) with the ILU(0) factor.
 * r holds b on entry (overwritten by the recursive residual), x gets the
 * solution.  *iters = 0-based iteration index at convergence (reference
 * convention); *conv = final relative residual.  Returns 1 when converged.
 * hist (nullable, length maxit) receives sqrt(|r|^2/|r0|^2) per iteration. */
int dfo_pcg(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
            const unsigned* diaind, const double* diag, const double* off, const double* fdiag,
            const double* foff, double* r, double* x, double tol, unsigned maxit,
            unsigned* iters, double* conv, double* hist);
/* dfo_pcg with a factor in its own (filled) pattern frowptr / fcolind / fdiaind. */
int dfo_pcg_fill(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind, const double* diag,
                 const double* off, const unsigned* frowptr, const unsigned* fcolind, const unsigned* fdiaind,
                 const double* fdiag, const double* foff, double* r, double* x, double tol, unsigned maxit,
                 unsigned* iters, double* conv, double* hist);
/* LsSol::Solve_PBiCGSTAB (src/ls/solver_ls_iter.cpp:291-408); *iters is the
 * 1-based iitr at convergence, as in the reference. */
/* LsSol::Solve_CG (no preconditioner), returns the reference's bool. */
int dfo_cg(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind, const double* diag,
           const double* off, double* r, double* x, double tol, unsigned maxit, unsigned* iters, double* conv);
int dfo_pbicgstab(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                  const unsigned* diaind, const double* diag, const double* off,
                  const double* fdiag, const double* foff, double* r, double* x, double tol,
                  unsigned maxit, unsigned* iters, double* conv);

/* ---- complex, b = 1 ---- */
void dfo_zspmv(unsigned N, const unsigned* rowptr, const unsigned* colind, const double* diag,
               const double* off, double alpha, const double* x, double beta, double* y);
/* CZMatDiaFrac_BlkCrs::DoILUDecomp (src/matvec/zmatdiafrac_blkcrs.cpp:192-261).
 * The reference blocks on getchar() for |pivot|^2 < 1e-20; this returns the
 * count of such pivots instead (and inverts them anyway, as the reference does
 * after the keypress). */
unsigned dfo_zilu0(unsigned N, const unsigned* rowptr, const unsigned* colind,
                   const unsigned* diaind, double* diag, double* off);
void dfo_zfwdbwd(unsigned N, const unsigned* rowptr, const unsigned* colind,
                 const unsigned* diaind, const double* fdiag, const double* foff, double* vec);
/* Fem::Ls::Solve_PCOCG (src/femls/zsolver_ls_iter.cpp:171-267); *iters is the
 * 1-based iitr at convergence (mx_iter when not converged), as in the reference. */
int dfo_pcocg(unsigned N, const unsigned* rowptr, const unsigned* colind, const unsigned* diaind,
              const double* diag, const double* off, const double* fdiag, const double* foff,
              double* r, double* x, double tol, unsigned maxit, unsigned* iters, double* conv);

/* Stored-matrix Newmark systems: SetBoundaryCondition_Row, MakeResidual and
   UpdateValueOfField of CLinearSystem_SaveDiaM_Newmark (scheme 1) and
   _NewmarkBeta (scheme 2). */
void dfo_mat_zero_rows(unsigned N, unsigned b, const unsigned* rowptr, const int* flags, double* diag, double* off);
void dfo_newmark_residual(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind, const double* diag,
                          const double* off, int scheme, double dt, double gamma, double beta, const double* force,
                          const double* u, const double* v, const double* a, const int* flags, double* t, double* r,
                          double* norm);
void dfo_newmark_update(size_t n, int scheme, double dt, double gamma, double beta, const int* flags, double* x,
                        double* u, double* v, double* a);

/* Complex ILU(k): SetValue_Initialize over the filled pattern, and
   Fem::Ls::Solve_PCOCG with a factor in its own pattern. */
void dfo_ziluk_init(unsigned N, const unsigned* rowptr, const unsigned* colind, const double* diag,
                    const double* off, const unsigned* frowptr, const unsigned* fcolind, double* fdiag,
                    double* foff);
int dfo_pcocg_fill(unsigned N, const unsigned* rowptr, const unsigned* colind, const double* diag,
                   const double* off, const unsigned* frowptr, const unsigned* fcolind, const unsigned* fdiaind,
                   const double* fdiag, const double* foff, double* r, double* x, double tol, unsigned maxit,
                   unsigned* iters, double* conv);

/* CMat_BlkCrs::MatVec (rectangular block-CRS, not transposed). */
void dfo_rmat_spmv(unsigned nrow, unsigned brow, unsigned bcol, const unsigned* rowptr, const unsigned* colind,
                   const double* val, double alpha, const double* x, double beta, double* y);

#ifdef __cplusplus
}
#endif
#endif
