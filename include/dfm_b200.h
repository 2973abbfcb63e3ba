/* dfm_b200.h - C ABI of the B200-native DelFEM linear-solve path.
 *
 * One shared library (delfem_b200/_lib/libdfm_b200.so, sm_100a) replaces the
 * reference's CPU hot path behind its own interfaces:
 *   LsSol::ILinearSystem(Preconditioner)_Sol  include/delfem/ls/linearsystem_interface_solver.h:39-82
 *   LsSol::CPreconditioner(_ILU)               include/delfem/ls/preconditioner.h:46-108
 *   LsSol::Solve_PCG / Solve_PBiCGSTAB         include/delfem/ls/solver_ls_iter.h:35-45
 *   Fem::Ls::Solve_PCOCG                       include/delfem/femls/zsolver_ls_iter.h:53-54
 *   MatVec::CMatDia_BlkCrs / CMatDiaFrac_BlkCrs include/delfem/matvec/matdia_blkcrs.h:44-118,
 *                                              include/delfem/matvec/matdiafrac_blkcrs.h:40-313
 * The C++ adapters in include/dfm_b200_lsol.hpp mirror those classes on top of
 * this ABI.
 *
 * Conventions
 *  - Storage is the reference's block-CRS with a separate diagonal: rowptr[N+1]
 *    (its m_colInd_Blk), colind[ncrs] (its m_rowPtr_Blk: off-diagonal columns,
 *    strictly ascending per row), diag[N*b*b], off[ncrs*b*b], each b x b block
 *    row-major; complex matrices (b = 1) store interleaved (re, im) doubles.
 *  - Vectors passed to compute calls are DEVICE pointers (cudaMalloc'd or
 *    torch tensors) of N*b doubles (2*N for complex).  Calls ending in _host
 *    take host pointers and include the copies.
 *  - Every call returns a dfm_status; nothing exits, asserts or waits for input.
 *  - Calls on one context are issued on its stream and are not re-entrant.
 */
#ifndef DFM_B200_H
#define DFM_B200_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

#define DFM_ABI_VERSION 1

#if defined(__GNUC__)
#define DFM_API __attribute__((visibility("default")))
#else
#define DFM_API
#endif

typedef enum dfm_status {
  DFM_OK = 0,
  DFM_ERR_INVALID = 1,       /* bad argument or inconsistent pattern (validated on the host) */
  DFM_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  DFM_ERR_NOMEM = 3,         /* device allocation failed */
  DFM_NOT_CONVERGED = 4,     /* max_iter reached (the reference's `false` of Solve_PCG) */
  DFM_BREAKDOWN = 5,         /* p.Ap <= 0, rho == 0 or a non-finite scalar */
  DFM_SINGULAR_PIVOT = 6,    /* more than 10 singular ILU pivots (reference nmax_sing) */
  DFM_WAIT_TIMEOUT = 7,      /* a bounded device-side wait ran out */
  DFM_ERR_UNSUPPORTED = 8,   /* block size / value type not supported by this entry */
  DFM_ERR_IO = 9             /* a file could not be opened or read */
} dfm_status;

enum { DFM_REAL = 0, DFM_COMPLEX = 1 };
enum { DFM_HOST = 0, DFM_DEVICE = 1 };
enum { DFM_PCG = 0, DFM_PBICGSTAB = 1, DFM_PCOCG = 2, DFM_PCG_MIXED = 3, DFM_PCOCG_MIXED = 4, DFM_CG = 5 };

typedef struct dfm_ctx_s* dfm_ctx;
typedef struct dfm_mat_s* dfm_mat;
typedef struct dfm_ilu_s* dfm_ilu;
typedef struct dfm_mesh_s* dfm_mesh;
typedef struct dfm_batch_s* dfm_batch;
typedef struct dfm_rmat_s* dfm_rmat;

DFM_API const char* dfm_status_string(int status);
/* The CUDA error code behind this host thread's last DFM_ERR_CUDA or
 * DFM_ERR_NOMEM (cudaSuccess if none), with "<runtime call>: <error name>"
 * written to buf[n] (nullable).  No reference counterpart: the reference has
 * no device code. */
DFM_API int dfm_last_cuda_error(char* buf, size_t n);
DFM_API int dfm_abi_version(void);

/* ---- context: device, stream, device status word ---------------------- */
DFM_API int dfm_ctx_create(int device, dfm_ctx* out);
/* Releases the caller's handle.  Every matrix, ILU, mesh, batch and
 * rectangular matrix created on the context holds it too, so they may be
 * destroyed before or after it, in any order; the context's stream and
 * buffers go with the last of them. */
DFM_API int dfm_ctx_destroy(dfm_ctx ctx);
/* Issue work on `stream` (a cudaStream_t; NULL restores the context's own). */
DFM_API int dfm_ctx_set_stream(dfm_ctx ctx, void* stream);
DFM_API int dfm_ctx_sync(dfm_ctx ctx);
/* Time limit of every device-side spin-wait (default 2 s). */
DFM_API int dfm_ctx_set_wait_limit(dfm_ctx ctx, unsigned long long ns);
/* Operator values of the mixed-precision solves (dfm_solve_pcg_mixed,
 * dfm_solve_pcocg_mixed): 0 = FP64 (default), 1 = FP32 copies. */
DFM_API int dfm_ctx_set_mixed_operator(dfm_ctx ctx, int fp32);
DFM_API int dfm_ctx_get_mixed_operator(dfm_ctx ctx, int* fp32);
/* First device-side error since the last call (code, kernel id); clears it. */
DFM_API int dfm_ctx_take_error(dfm_ctx ctx, int* code, int* where);
/* Failure-detection self test: one kernel waits on a flag nothing sets, under
 * the given limit, and must come back with DFM_WAIT_TIMEOUT. */
DFM_API int dfm_ctx_wait_selftest(dfm_ctx ctx, unsigned long long limit_ns);

/* ---- device buffers (for callers built without the CUDA toolkit) -------- */
/* dfm_buf_copy directions; the copy is complete when the call returns. */
enum { DFM_H2D = 0, DFM_D2H = 1, DFM_D2D = 2 };
DFM_API int dfm_buf_alloc(dfm_ctx ctx, size_t bytes, void** out);
DFM_API int dfm_buf_free(dfm_ctx ctx, void* p);
DFM_API int dfm_buf_copy(dfm_ctx ctx, void* dst, const void* src, size_t bytes, int direction);
DFM_API int dfm_buf_zero(dfm_ctx ctx, void* p, size_t bytes);

/* ---- vector operations: CVector_Blk on the device ----------------------- */
/* The solver-side vector steps of LsSol::CLinearSystem (DOT / COPY / SCAL /
 * AXPY, src/ls/linearsystem.cpp:298-415, over MatVec::CVector_Blk,
 * src/matvec/vector_blk.cpp:37-112) on device arrays of n doubles, issued on
 * the context's stream.  dfm_vec_dot returns the value on the host (it
 * synchronises; fixed summation order, so equal inputs give equal bits);
 * the others only enqueue.  dfm_vec_scal multiplies (NaN * 0 stays NaN, as
 * in the reference). */
DFM_API int dfm_vec_dot(dfm_ctx ctx, size_t n, const double* x, const double* y, double* out);
DFM_API int dfm_vec_copy(dfm_ctx ctx, size_t n, const double* x, double* y);          /* y := x */
DFM_API int dfm_vec_scal(dfm_ctx ctx, size_t n, double alpha, double* x);             /* x := alpha x */
DFM_API int dfm_vec_axpy(dfm_ctx ctx, size_t n, double alpha, const double* x, double* y); /* y += alpha x */
/* y[i b + c] := x[idx[i] b + c] for the nblk blocks of b doubles (idx a
 * device array of nblk block indices, y not aliasing x): a vector into or out
 * of a block ordering, as COrdering_Blk::OrderingVector_OldToNew / _NewToOld
 * (src/matvec/ordering_blk.cpp:136-170) with idx the new-to-old or the
 * old-to-new map.  Enqueued on the context's stream. */
DFM_API int dfm_vec_gather(dfm_ctx ctx, size_t nblk, unsigned b, const unsigned* idx, const double* x, double* y);

/* ---- matrix: CMatDia_BlkCrs on the device ------------------------------ */
/* Pattern from host arrays; validated (monotone rowptr, in-range, strictly
 * ascending off-diagonal columns, no diagonal entry) as CMatDia_BlkCrs::AddPattern
 * (src/matvec/matdia_blkcrs.cpp:346-505) requires.  b in {1,2,3} (real) or 1 (complex). */
DFM_API int dfm_mat_create(dfm_ctx ctx, unsigned N, unsigned b, int value_type,
                   const unsigned* rowptr, const unsigned* colind, dfm_mat* out);
DFM_API int dfm_mat_destroy(dfm_mat A);
DFM_API int dfm_mat_info(dfm_mat A, unsigned* N, unsigned* b, unsigned* ncrs, int* value_type);
/* CMatDia_BlkCrs::SetZero (src/matvec/matdia_blkcrs.cpp:139-163). */
DFM_API int dfm_mat_set_zero(dfm_mat A);
DFM_API int dfm_mat_set_values(dfm_mat A, const double* diag, const double* off, int where);
DFM_API int dfm_mat_get_values(dfm_mat A, double* diag, double* off, int where);
/* Device addresses of the value arrays (owned by A). */
DFM_API int dfm_mat_values_device(dfm_mat A, double** diag, double** off);
/* Lanes per block row of the SpMV (4, 8, 16, 32); 0 = autotuned on first use. */
DFM_API int dfm_mat_set_spmv_lanes(dfm_mat A, int lanes);
DFM_API int dfm_mat_get_spmv_lanes(dfm_mat A, int* lanes);
/* SpMV kernel: 0 = a lane per block (direct loads), 1 = row tiles staged in
 * shared memory by TMA bulk copies, 2 = element-wise coalesced loads of each
 * row's contiguous values, 3 = each warp stages its rows' contiguous value run
 * in shared memory with coalesced 16-byte loads (1, 2 and 3 real matrices
 * only).  Autotuned together with the lanes. */
DFM_API int dfm_mat_set_spmv_kernel(dfm_mat A, int kernel);
DFM_API int dfm_mat_get_spmv_kernel(dfm_mat A, int* kernel);

/* y = beta*y + alpha*A x  (CMatDia_BlkCrs::MatVec, src/matvec/matdia_blkcrs.cpp:921-1094;
 * complex: CZMatDia_BlkCrs::MatVec, src/matvec/zmatdia_blkcrs.cpp:737-801).
 * beta == 0 writes y without reading it. */
DFM_API int dfm_spmv(dfm_mat A, double alpha, const double* x, double beta, double* y);
/* Measurement hook, no counterpart in the reference: `reps` back-to-back
 * launches of y = A x (the tuned kernel) on the context's stream between one
 * pair of CUDA events, after one untimed launch; *ms = average per launch. */
DFM_API int dfm_time_spmv(dfm_mat A, const double* x, double* y, int reps, float* ms);

/* ---- rectangular block matrices: CMat_BlkCrs (segment couplings) -------- */
/* MatVec::CMat_BlkCrs (include/delfem/matvec/mat_blkcrs.h:44-190), the
 * coupling of two segments of a linear system (CLinearSystem::GetMatrix(i, j),
 * i != j): nrow x ncol blocks of brow x bcol values (1..3 each), every block
 * in the CRS list, row-major blocks; pattern from host arrays (rowptr[nrow+1],
 * colind ascending per row, no repeats; validated). */
DFM_API int dfm_rmat_create(dfm_ctx ctx, unsigned nrow, unsigned ncol, unsigned brow, unsigned bcol,
                            const unsigned* rowptr, const unsigned* colind, dfm_rmat* out);
DFM_API int dfm_rmat_destroy(dfm_rmat R);
/* val[nnz*brow*bcol] at DFM_HOST or DFM_DEVICE. */
DFM_API int dfm_rmat_set_values(dfm_rmat R, const double* val, int where);
/* y (nrow*brow) = beta y + alpha R x (x: ncol*bcol), CMat_BlkCrs::MatVec
 * (src/matvec/mat_blkcrs.cpp:955-1175); beta == 0 writes y without reading it. */
DFM_API int dfm_rmat_spmv(dfm_rmat R, double alpha, const double* x, double beta, double* y);

/* Reads a complex matrix with scalar blocks from the reference's text format
 * (CZMatDia_BlkCrs(const std::string& file_path), src/matvec/zmatdia_blkcrs.cpp:
 * 108-173): "nblk nnz", then nnz lines "icol irow re im", icol = row.  Host
 * only.  With rowptr == NULL it reports *N and *ncrs (off-diagonal entries);
 * then rowptr[N+1], colind[ncrs], diag[2N] and off[2 ncrs] (re, im
 * interleaved; each nullable) receive the matrix, ready for dfm_mat_create
 * (DFM_COMPLEX) and dfm_mat_set_values.  Rows without entries are empty with
 * a zero diagonal and each row's columns come out ascending; a repeated
 * off-diagonal column, an index out of range or a decreasing row is
 * DFM_ERR_INVALID, an unreadable file DFM_ERR_IO. */
DFM_API int dfm_zmat_read_text(const char* path, unsigned* N, unsigned* ncrs, unsigned* rowptr, unsigned* colind,
                               double* diag, double* off);

/* Reads a GiD ASCII mesh as the reference's readers do
 * (Msh::CMesh3D::ReadFromFile_GiDMsh, src/msh/mesh3d.cpp:601-800;
 * Msh::CMesher2D::ReadFromFile_GiDMsh, src/msh/mesher2d.cpp:2464-2640).  Host
 * only.  Tetrahedra / hexahedra: 3-D coordinates.  Triangles /
 * quadrilaterals: 2-D coordinates, a planar 3-D node cloud projected by
 * dropping its axis of least variance as the 2-D mesher does (a non-planar
 * one is DFM_ERR_INVALID).  With coord == NULL it reports *ndim, *nnode,
 * *nnoel and *nelem; then coord[nnode*ndim] and elem[nelem*nnoel] (0-based,
 * nullable) receive the mesh, ready for dfm_mesh_create; dfm_gid_boundary
 * derives the reference's boundary facets from it.  Malformed input is
 * DFM_ERR_INVALID, an unreadable file DFM_ERR_IO. */
DFM_API int dfm_gid_read_mesh(const char* path, int* ndim, unsigned* nnode, double* coord, int* nnoel,
                              unsigned* nelem, int* elem);

/* The boundary facets the reference's GiD readers derive from the elements
 * (host only), on a mesh as dfm_gid_read_mesh returns it:
 *  - ndim 3, nnoel 4 (tetrahedra; Msh::CMesh3D::ReadFromFile_GiDMsh,
 *    src/msh/mesh3d.cpp:744-778): facets are the triangles of faces that no
 *    other tetrahedron shares with the opposite orientation (Msh::MakeTetSurTet
 *    + MakeOuterBoundTet, src/msh/meshkernel3d.cpp:102-230, 514-539), in
 *    (tetrahedron, face) order, nodes counter-clockwise from outside; groups
 *    are the colours of Msh::MakeColorCoding_Tri3D (:905-947): flat patches
 *    grown across shared edges whose unit normals have a dot product above
 *    crt_dot (0.2 in the reader), each group's facets ascending;
 *  - ndim 2, nnoel 3 or 4 (Msh::CMesher2D::ReadFromFile_GiDMsh,
 *    src/msh/mesher2d.cpp:2581-2760): facets are the outer bars (edges no
 *    other element shares; MakeOuterBoundTri / Quad,
 *    src/msh/meshkernel2d.cpp:1272-1323) in (element, edge) order; groups are
 *    the bar arrays of Msh::ColorCodeBarAry (:1941-2018): chains in walking
 *    order that end at a node without exactly two bars or where successive
 *    unit directions have a dot product at most crt_dot (0.8 there);
 *    vertex[] holds the chains' end nodes ascending (the reader's vertices)
 *    and group_ends[2 g] / [2 g + 1] the indices into vertex[] of chain g's
 *    first and last node (the bar array's id_se);
 *  - ndim 3, nnoel 8 (hexahedra): no facets (the reference derives none).
 * The reference numbers the element array 1, then the groups 2, 3, ... and
 * (2-D) the vertices after them.  With facet == NULL it reports *nnofa (nodes
 * per facet), *nfacet, *ngroup and *nvertex; then facet[nfacet*nnofa],
 * group_ptr[ngroup+1], group_facet[nfacet], vertex[nvertex] and
 * group_ends[2*ngroup] (each but facet nullable) receive them.  Node indices
 * out of range or an element with a repeated node are DFM_ERR_INVALID. */
DFM_API int dfm_gid_boundary(int ndim, unsigned nnode, const double* coord, int nnoel, unsigned nelem,
                             const int* elem, double crt_dot, int* nnofa, unsigned* nfacet, unsigned* facet,
                             unsigned* ngroup, unsigned* group_ptr, unsigned* group_facet, unsigned* nvertex,
                             unsigned* vertex, unsigned* group_ends);

/* The stored boundary matrix B of Fem::Ls::CLinearSystem_Save
 * (src/femls/linearsystem_fieldsave.cpp:64-260; pattern CMat_BlkCrs::
 * SetPatternBoundary, src/matvec/mat_blkcrs.cpp:1177-1265; masks
 * SetBoundaryConditionInverse_Colum / SetBoundaryCondition_Row, :876-951),
 * host only: from K's values BEFORE dfm_apply_dirichlet (rowptr, colind, diag,
 * off in the library's layout) and the flags (N*b, nonzero = fixed), B keeps
 * the entries of free rows and fixed columns.  With brow == NULL it reports
 * *bncrs; then brow[N+1], bcol[*bncrs], bdiag[N*b*b], boff[*bncrs*b*b]
 * (each but brow nullable) receive B for dfm_mat_create + dfm_mat_set_values.
 * CLinearSystem_Save::MakeResidual (:206-246), r = Force - B u, is then
 * dfm_spmv(B, -1, u, 1, r) with r holding Force. */
DFM_API int dfm_boundary_matrix(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                                const double* diag, const double* off, const int* flags, unsigned* brow,
                                unsigned* bcol, double* bdiag, double* boff, unsigned* bncrs);

/* ---- time integration with a stored matrix ------------------------------- */
/* Fem::Ls::CLinearSystem_SaveDiaM_Newmark (first order, scheme 1: the update
 * is the velocity) and CLinearSystem_SaveDiaM_NewmarkBeta (second order,
 * scheme 2: the update is the acceleration), src/femls/linearsystem_fieldsave.
 * cpp:367-880.  B is their stored matrix: the element matrices K_e merged
 * into the full pattern (diagonal blocks included), with the rows of fixed
 * DOFs zeroed by dfm_mat_zero_rows (CMat_BlkCrs::SetBoundaryCondition_Row,
 * src/matvec/mat_blkcrs.cpp:910-951) in FinalizeMarge.  Device vectors of
 * N*b doubles; flags: device int[N*b], nonzero = fixed.  Real matrices. */
DFM_API int dfm_mat_zero_rows(dfm_mat B, const int* flags);
/* MakeResidual (:446-520, :706-794): t = u + dt(1-gamma) v (scheme 1) or
 * t = u + dt v + dt^2(1/2-beta) a (scheme 2; a unused by scheme 1), then
 * r = force - B t with r = 0 at fixed DOFs; *norm (nullable) = |r|.  t is the
 * caller's work vector; r may alias force.  Synchronises (the norm). */
DFM_API int dfm_newmark_residual(dfm_mat B, int scheme, double dt, double gamma, double beta, const double* force,
                                 const double* u, const double* v, const double* a, const int* flags, double* t,
                                 double* r, double* norm);
/* UpdateValueOfField (:522-566, :796-877) after the solve of the update x:
 * scheme 1: free DOFs u += dt(1-gamma) v + dt gamma x, fixed DOFs x = v, then
 * v = x; scheme 2: free DOFs u += dt v + dt^2(1/2-beta) a + dt^2 beta x and
 * v += dt(1-gamma) a + gamma dt x, fixed DOFs x = a, then a = x.  The
 * reference's arithmetic term by term (bit-identical). */
DFM_API int dfm_newmark_update(dfm_ctx ctx, size_t n, int scheme, double dt, double gamma, double beta,
                               const int* flags, double* x, double* u, double* v, double* a);

/* ---- element assembly: CLinearSystem_Field + Fem::Eqn::AddLinSys_* ------- */
/* A P1 mesh resident on the device: coord[nnode*ndim], elem[nelem*nnoel]
 * (triangles nnoel = 3 in 2D, tetrahedra 4 in 3D) and optional boundary bars
 * bar[nbar*2] (the Sommerfeld boundary of the Helmholtz problem).  Host arrays;
 * the node -> element adjacency used by the gather assembly is built here. */
DFM_API int dfm_mesh_create(dfm_ctx ctx, int ndim, unsigned nnode, const double* coord, unsigned nnoel,
                    unsigned nelem, const int* elem, unsigned nbar, const int* bar, dfm_mesh* out);
DFM_API int dfm_mesh_destroy(dfm_mesh mesh);
/* The mesh's block pattern as CMatDia_BlkCrs::AddPattern builds it
 * (src/matvec/matdia_blkcrs.cpp:346-505): row i lists, ascending, every other
 * node sharing an element with node i.  Host arrays: rowptr[nnode+1] and
 * colind[*ncrs]; call with colind NULL first to learn *ncrs. */
DFM_API int dfm_mesh_pattern(dfm_mesh mesh, unsigned* rowptr, unsigned* colind, size_t* ncrs);
/* Each assemble call is InitializeMarge (matrix and residual zeroed,
 * src/ls/linearsystem.cpp:74-89) + the element loop + nodal loads
 * added to the residual afterwards.  A's pattern must hold every element's node
 * pairs (dfm pattern from the same mesh); entries outside it are skipped as in
 * CMatDia_BlkCrs::Mearge (src/matvec/matdia_blkcrs.cpp:165-258).  Results are
 * bit-identical to the reference's.  Device pointers: elem_coef[nelem]
 * (per-element multiplier of the material constants, nullable), u (current
 * field, nullable = 0: res = f - K u), load (nodal loads, nullable), rhs (out,
 * N*b doubles, 2N for complex).  Row length <= 63 off-diagonal blocks. */
/* AddLinearSystem_Poisson2D_P1, src/femeqn/eqn_poisson.cpp:49-125 (b = 1). */
DFM_API int dfm_assemble_poisson2d(dfm_mesh mesh, dfm_mat A, double alpha, double source,
                           const double* elem_coef, const double* u, const double* load, double* rhs);
/* AddLinSys_LinearSolid2D_Static_P1, src/femeqn/eqn_linear_solid2d.cpp:505-598 (b = 2). */
DFM_API int dfm_assemble_solid2d(dfm_mesh mesh, dfm_mat A, double lambda, double myu, double rho, double gx,
                         double gy, const double* elem_coef, const double* u, const double* load, double* rhs);
/* AddLinSys_LinearSolid3D_Static_P1, src/femeqn/eqn_linear_solid3d.cpp:241-334 (b = 3). */
DFM_API int dfm_assemble_solid3d(dfm_mesh mesh, dfm_mat A, double lambda, double myu, double rho, double gx,
                         double gy, double gz, const double* u, const double* load, double* rhs);
/* AddLinearSystem_Helmholtz2D_P1 (src/femeqn/eqn_helmholtz.cpp:51-137) followed by
 * AddLinearSystem_SommerfeltRadiationBC2D_B1 (:437-512) on the mesh's bars; complex A. */
DFM_API int dfm_assemble_helmholtz2d(dfm_mesh mesh, dfm_mat A, double wave_length, const double* u,
                             const double* load, double* rhs);
/* Dirichlet elimination of FinalizeMarge (src/ls/linearsystem.cpp:92-122:
 * CMatDia_BlkCrs::SetBoundaryCondition, src/matvec/matdia_blkcrs.cpp:261-343,
 * and CBCFlag::SetZeroToBCDof): rows and
 * columns of fixed DOFs zeroed, unit diagonal, residual zeroed.  flags: device
 * int[N*b], nonzero = fixed; rhs nullable.  Real matrices. */
DFM_API int dfm_apply_dirichlet(dfm_mat A, const int* flags, double* rhs);
/* No counterpart in the reference: the element kernel of the adjoint of
 * K(coef) u = f, where each element matrix is linear in its coefficient
 * (K_e = coef_e K_e^0 for the Poisson alpha and the solid lambda, myu pair):
 * grad[e] = -lambda_e^T K_e^0 u_e with K_e^0 the element matrix at the given
 * base constants.  lam, u: device vectors (N*b), grad: device nelem. */
DFM_API int dfm_coef_grad_poisson2d(dfm_mesh mesh, double alpha, const double* lam, const double* u,
                            double* grad);
DFM_API int dfm_coef_grad_solid2d(dfm_mesh mesh, double lambda, double myu, const double* lam, const double* u,
                          double* grad);

/* ---- ILU(0): CPreconditioner_ILU / CMatDiaFrac_BlkCrs ------------------- */
/* Symbolic ILU(0) (CMatDiaFrac_BlkCrs(0, A), src/matvec/matdiafrac_blkcrs.cpp:227-287)
 * plus the level sets of both sweeps in the natural order. */
DFM_API int dfm_ilu_create(dfm_mat A, dfm_ilu* out);
/* ILU(k) (CPreconditioner_ILU::SetFillInLevel(lev) + SetLinearSystem,
 * src/ls/preconditioner.cpp:57-212): the factor's pattern is A's plus the fill
 * entries of CMatDiaFrac_BlkCrs::AddFracPtn (src/matvec/matdiafrac_blkcrs.cpp:
 * 1249-1377) up to level lev (-1: no limit), identical to the reference's;
 * dfm_ilu_factor then starts from A's values in it (SetValue_Initialize) and
 * factors over it.  lev = 0 is dfm_ilu_create.  Complex matrices too
 * (CZPreconditioner_ILU::SetFillInLevel, include/delfem/femls/zpreconditioner.h:75,
 * whose CZMatDiaFrac_BlkCrs::AddFracPtn, src/matvec/zmatdiafrac_blkcrs.cpp:
 * 263-441, fills as the real one does).  Batches (dfm_batch_create) take
 * ILU(0) objects only. */
DFM_API int dfm_ilu_create_fill(dfm_mat A, int lev, dfm_ilu* out);
/* ILU(k) with unlimited fill through some block rows (CPreconditioner_ILU::
 * SetFillBlk, include/delfem/ls/preconditioner.h:80, applied by
 * CMatDiaFrac_BlkCrs::AddFracPtn(lev, aBlkFill), src/matvec/
 * matdiafrac_blkcrs.cpp:1379-1500): a fill candidate (i, j) is kept whatever
 * its level when row i or row j is one of rows[0..nrows) and i, j < bound;
 * otherwise the rule of dfm_ilu_create_fill.  bound = N for one matrix; for
 * segments joined into one matrix, the first segment's block rows (the
 * reference hands the list to that segment's diagonal matrix only).  Rows may
 * repeat; a row >= bound is DFM_ERR_INVALID.  nrows = 0 is
 * dfm_ilu_create_fill. */
DFM_API int dfm_ilu_create_fill_rows(dfm_mat A, int lev, const unsigned* rows, size_t nrows, unsigned bound,
                                     dfm_ilu* out);
/* The factor's pattern (host arrays, nullable): rowptr[N+1], colind[*ncrs];
 * the off-diagonal values of dfm_ilu_get_values/set_values follow it. */
DFM_API int dfm_ilu_pattern(dfm_ilu M, unsigned* rowptr, unsigned* colind, unsigned* ncrs);
DFM_API int dfm_ilu_destroy(dfm_ilu M);
/* Level counts; lev_fwd / lev_bwd (host, N entries each, nullable) get the level of every row. */
DFM_API int dfm_ilu_levels(dfm_ilu M, unsigned* nlev_fwd, unsigned* nlev_bwd, unsigned* lev_fwd,
                   unsigned* lev_bwd);
/* Numeric ILU(0) of A on the device (DoILUDecomp, :769-1102), bit-identical to the
 * reference.  Returns DFM_SINGULAR_PIVOT when more than 10 pivots are singular. */
DFM_API int dfm_ilu_factor(dfm_ilu M, dfm_mat A, unsigned* n_singular);
DFM_API int dfm_ilu_get_values(dfm_ilu M, double* diag, double* off, int where);
DFM_API int dfm_ilu_set_values(dfm_ilu M, const double* diag, const double* off, int where);
/* z = U^-1 L^-1 r (ForwardSubstitution + BackwardSubstitution, :332-663).  r != z. */
DFM_API int dfm_ilu_apply(dfm_ilu M, const double* r, double* z);
/* Measurement hook, no counterpart in the reference: `reps` back-to-back
 * dfm_ilu_apply launch sequences (forward + backward sweep) timed as
 * dfm_time_spmv does; *ms = average per application. */
DFM_API int dfm_time_ilu_apply(dfm_ilu M, const double* r, double* z, int reps, float* ms);
/* No counterpart in the reference.  The same z = U^-1 L^-1 r as dfm_ilu_apply,
 * for callers that cannot allocate device memory at the point of use (code
 * that enqueues work on a stream it must not stall - cudaMalloc and cudaFree
 * can synchronise the device -, a host framework that owns every device
 * allocation, callbacks under an allocator lock): it allocates nothing,
 * keeping its intermediate vector in a static device array of 4 MiB
 * (N * doubles-per-row <= 524,288, else DFM_ERR_INVALID) that every GPU
 * loading the library holds until exit.  It enqueues the two sweeps on the
 * context's stream and returns without waiting; device-side errors surface
 * through dfm_ctx_take_error.  All calls share the array, so calls whose
 * kernels overlap on the GPU race on it.  The first call on a context looks
 * up the array's address with the context's device current; make it before
 * any stream capture.  Runs the one-CTA level-barrier schedule. */
DFM_API int dfm_ilu_apply_static(dfm_ilu M, const double* r, double* z);
/* Sweep schedule: 0 = autotuned, 1 = sync-free across the GPU, 2 = one CTA with
 * level barriers, 3 = contiguous row ranges per CTA (shared-memory slice, TMA-
 * streamed level data, a CTA barrier per level; the CTA count is the max_blocks
 * of dfm_ilu_set_sweep_tuning, default one per SM), 4 = the row ranges of 3
 * without level barriers (each row waits on its own operands), 5 and 6 = 3 and
 * 4 with the levels taken in pairs (the second level's operands on the first
 * substituted by products with the factor, recomputed after every
 * factorization: half the sequential steps, results equal to rounding), 7 and
 * 8 = 3 and 5 with the row groups in two halves taking alternate levels, the
 * idle half fetching its next row's operands before the level barrier (same
 * results as 3 and 5), 9 = the row ranges of 3 with the level path in shared
 * memory only: a few compute warps synchronised by a named barrier take the
 * rows of each level while producer warps stream the level data by TMA and
 * prefetch the operands owned by other CTAs into a shared-memory halo (results
 * equal to those of 3 to rounding), 10 = 9 with the levels taken in pairs as
 * in 5 (half the sequential steps; the second level reads the first level's
 * right-hand sides through the products with the factor; results equal to
 * rounding).  Complex matrices run 3-10 as real 2x2 blocks [re -im; im re]. */
DFM_API int dfm_ilu_set_sweep(dfm_ilu M, int mode);
/* No counterpart in the reference (its sweeps are sequential).  A row
 * partition for the range-partitioned sweep schedules: CTA c takes the rows
 * with part[i] == c (part has N entries, nparts <= the GPU's SM count: one
 * co-resident CTA per part).  The sweeps' results do not depend on it.  A
 * caller that knows the geometry can shorten the chains of dependencies that
 * cross CTAs, e.g. with compact patches across the direction the levels
 * advance in.  The autotuner times the partition beside balanced ranges of the
 * natural order and keeps the faster; explicit range modes (dfm_ilu_set_sweep
 * 3-8) use it.  part == NULL clears it.  Resets the schedule to autotuned. */
DFM_API int dfm_ilu_set_sweep_partition(dfm_ilu M, const unsigned* part, unsigned nparts);
/* No counterpart in the reference.  A partition for dfm_ilu_set_sweep_partition
 * from node coordinates (host, coord[nnode*ndim]): a grid of at most max_parts
 * patches across the longest bounding-box axis, so that every line of nodes
 * along that axis lies in one part.  *nparts gets the grid's cell count. */
DFM_API int dfm_sweep_partition_patches(unsigned nnode, int ndim, const double* coord, unsigned max_parts,
                                        unsigned* part, unsigned* nparts);
DFM_API int dfm_ilu_get_sweep(dfm_ilu M, int* mode);
/* No counterpart in the reference.  The launch shape of schedules 9 and 10
 * (valid while one of them is the schedule): compute warps 1, 2 or 4, lanes per row 2, 4 or 8,
 * producer warps (compute + producer <= 16).  The autotuner picks one; this
 * pins it (a row's sum runs over `lanes` lanes, so the lanes decide its
 * summation order). */
DFM_API int dfm_ilu_set_sweep_warps(dfm_ilu M, int compute_warps, int lanes, int producer_warps);
DFM_API int dfm_ilu_get_sweep_warps(dfm_ilu M, int* compute_warps, int* lanes, int* producer_warps);
/* Sync-free schedule knobs: cap on the number of co-resident blocks (0 = all
 * that fit) and the back-off between polls of a waiting lane in ns (global). */
DFM_API int dfm_ilu_set_sweep_tuning(dfm_ilu M, int max_blocks, unsigned poll_sleep_ns);

/* ---- Krylov solvers ------------------------------------------------------ */
/* Common to the solvers: x = 0 initial guess; r holds b on entry and the
 * recursive residual on exit; *conv = |r|/|r0| at exit; the stop test is the
 * reference's |r|^2/|r0|^2 < tol^2 on the recursive residual.  Reductions are
 * deterministic (same inputs, same bits), the iterations run as replays of a
 * captured CUDA graph with all scalars on the device.  DFM_NOT_CONVERGED at
 * max_iter (where the reference's PBiCGSTAB and PCOCG still return true),
 * DFM_BREAKDOWN on a non-finite step. */
/* LsSol::Solve_PCG (src/ls/solver_ls_iter.cpp:100-172) preconditioned by M.
 * *iters follows the reference: the 0-based index of the converged iteration. */
DFM_API int dfm_solve_pcg(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit,
                  unsigned* iters, double* conv);
/* LsSol::Solve_CG (src/ls/solver_ls_iter.cpp:31-97): conjugate gradients
 * without a preconditioner, on A alone.  *iters is the 0-based index of the
 * converged iteration (max_iter when it is reached: DFM_NOT_CONVERGED here,
 * where the reference returns true and leaves conv_ratio at the tolerance);
 * |r0|^2 < 1e-60 returns at once with *conv = |r0|.  Real matrices. */
DFM_API int dfm_solve_cg(dfm_mat A, double* r, double* x, double tol, unsigned maxit, unsigned* iters,
                         double* conv);
/* LsSol::Solve_PBiCGSTAB (src/ls/solver_ls_iter.cpp:291-408): shadow residual
 * r0, *iters 1-based.  Real matrices. */
DFM_API int dfm_solve_pbicgstab(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit,
                        unsigned* iters, double* conv);
/* Fem::Ls::Solve_PCOCG (src/femls/zsolver_ls_iter.cpp:171-267): complex
 * symmetric CG with unconjugated products, *iters 1-based.  Complex matrices;
 * r and x are interleaved (re, im). */
DFM_API int dfm_solve_pcocg(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit,
                    unsigned* iters, double* conv);
/* No counterpart in the reference: PCG whose ILU(0) sweeps read FP32 copies of
 * the L / D^-1 U blocks (D^-1 pivots, vectors, dots and scalars stay FP64),
 * inside FP64 iterative refinement done as residual replacement - the true
 * residual b - A x with the FP64 values replaces the recursive one every 16
 * iterations and whenever the latter meets tol, and only a true residual
 * below tol ends the solve.  The SpMV of the recurrences uses A's FP64 values
 * unless dfm_ctx_set_mixed_operator(ctx, 1) selects FP32 copies of them too
 * (which pays only where cond(A) * 2^-24 << 1: on stiff systems the FP32
 * operator loses conjugacy and costs iterations).  Same arguments and
 * conventions as dfm_solve_pcg (x = 0 start, *iters 0-based); real matrices. */
DFM_API int dfm_solve_pcg_mixed(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit,
                        unsigned* iters, double* conv);
/* The same scheme for PCOCG on complex matrices: complex64 factor values in
 * the ILU sweeps (and in the SpMV under dfm_ctx_set_mixed_operator(ctx, 1)),
 * complex128 vectors, dots, scalars and D^-1, complex128 residual
 * replacement; conventions of dfm_solve_pcocg. */
DFM_API int dfm_solve_pcocg_mixed(dfm_mat A, dfm_ilu M, double* r, double* x, double tol, unsigned maxit,
                          unsigned* iters, double* conv);
/* ---- batched solves (no counterpart in the reference) -------------------- */
/* A batch of independent systems stored as one block-diagonal matrix: instance
 * k owns block rows [row_off[k], row_off[k+1]) of M's matrix (row_off: host,
 * ninst + 1 entries, row_off[ninst] = N) and no entry crosses an instance
 * boundary (checked).  M's ILU(0) factor is then the per-instance factors. */
DFM_API int dfm_batch_create(dfm_ilu M, unsigned ninst, const unsigned* row_off, dfm_batch* out);
DFM_API int dfm_batch_destroy(dfm_batch batch);
/* Lanes per row of the batched SpMV (4, 8, 16, 32) and rows per chunk (the
 * tile of the per-instance reductions); 0, 0 = autotuned on the next solve. */
DFM_API int dfm_batch_set_tuning(dfm_batch batch, int lanes, int chunk_rows);
DFM_API int dfm_batch_get_tuning(dfm_batch batch, int* lanes, int* chunk_rows);
/* Schedule: 0 = autotuned on the next solve, 1 = every phase one launch over
 * all instances with the iteration captured as a CUDA graph, 2 = one
 * persistent launch in which each CTA (cta_threads 256/512/1024, cta_lanes
 * 2/4/8 lanes per row) solves whole instances taken from a queue. */
DFM_API int dfm_batch_set_schedule(dfm_batch batch, int schedule, int cta_threads, int cta_lanes);
DFM_API int dfm_batch_get_schedule(dfm_batch batch, int* schedule, int* cta_threads, int* cta_lanes);
/* Every instance runs Solve_PCG's algorithm with its own scalars, stop test
 * and iteration count, all instances advancing in the same launches; stopped
 * instances are masked.  b (N*b doubles) and x at DFM_HOST or DFM_DEVICE;
 * iters, conv, status: host arrays of ninst (nullable), status per instance
 * (DFM_OK, DFM_NOT_CONVERGED, DFM_BREAKDOWN).  Returns DFM_OK when every
 * instance converged, else the worst instance status. */
DFM_API int dfm_batch_solve_pcg(dfm_batch batch, const double* b, int b_where, double* x, int x_where,
                        double tol, unsigned maxit, unsigned* iters, double* conv, int* status);

/* End-to-end variants with HOST buffers (b copied in, x copied out, inside the
 * call); method is any DFM_PCG ... DFM_CG (M is ignored for DFM_CG). */
DFM_API int dfm_solve_host(dfm_mat A, dfm_ilu M, int method, const double* b_host, double* x_host, double tol,
                   unsigned maxit, unsigned* iters, double* conv);
DFM_API int dfm_solve_pcg_host(dfm_mat A, dfm_ilu M, const double* b_host, double* x_host, double tol,
                       unsigned maxit, unsigned* iters, double* conv);

#ifdef __cplusplus
}
#endif
#endif
