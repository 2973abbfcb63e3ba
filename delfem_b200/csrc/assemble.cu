// Element assembly into the block-CRS matrix and the residual, and the
// Dirichlet elimination, on the device.
//
// Reference element loops (one element at a time, Mearge scatter-add):
//   AddLinearSystem_Poisson2D_P1            src/femeqn/eqn_poisson.cpp:49-125
//   AddLinSys_LinearSolid2D_Static_P1       src/femeqn/eqn_linear_solid2d.cpp:505-598
//   AddLinSys_LinearSolid3D_Static_P1       src/femeqn/eqn_linear_solid3d.cpp:241-334
//   AddLinearSystem_Helmholtz2D_P1          src/femeqn/eqn_helmholtz.cpp:51-137
//   AddLinearSystem_SommerfeltRadiationBC2D_B1  src/femeqn/eqn_helmholtz.cpp:437-512
//   CMatDia_BlkCrs::Mearge                  src/matvec/matdia_blkcrs.cpp:165-258
//   CMatDia_BlkCrs::SetBoundaryCondition    src/matvec/matdia_blkcrs.cpp:261-343
//   CBCFlag::SetZeroToBCDof                 include/delfem/matvec/bcflag_blk.h:102-129
//
// Gather formulation: one warp owns a node (a block row).  Its lanes compute
// the element-matrix rows of up to 32 surrounding elements at once (elements in
// ascending order, from a node->element adjacency built at mesh set-up) into
// shared memory; then lane j, which owns slot j of the row (the last slot is
// the diagonal block), adds every contribution to that slot in element order.
// Each slot therefore receives the same additions in the same order as in the
// reference's sequential scatter, and with this file compiled without FMA
// contraction (-fmad=false) the assembled values are bit-identical.  The row's
// blocks are contiguous, so the final stores are coalesced.
#include <algorithm>
#include <new>

#include "dfm_internal.h"

struct dfm_mesh_s {
  dfm_ctx ctx = nullptr;
  int ndim = 2;
  unsigned nnode = 0, nnoel = 3, nelem = 0, nbar = 0;
  double* d_coord = nullptr;
  int* d_elem = nullptr;
  int* d_bar = nullptr;
  unsigned* d_esup_ptr = nullptr;  // node -> elements (ascending)
  unsigned* d_esup = nullptr;
  unsigned* d_bsup_ptr = nullptr;  // node -> boundary bars (ascending)
  unsigned* d_bsup = nullptr;
  std::vector<int> h_elem;         // host copies for the pattern
  std::vector<unsigned> h_esup_ptr, h_esup;
};

namespace dfm {

constexpr int kAsmWarps = 4;  // warps (nodes) per CTA

// ---------------------------------------------------- element geometry (ref. order)
DFM_DEVINL double tri_area(const double* p0, const double* p1, const double* p2) {
  return 0.5 * ((p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]));
}
DFM_DEVINL void tri_dldx(double d[3][2], const double* p0, const double* p1, const double* p2) {
  const double area = tri_area(p0, p1, p2);
  const double tmp1 = 0.5 / area;
  d[0][0] = tmp1 * (p1[1] - p2[1]);
  d[1][0] = tmp1 * (p2[1] - p0[1]);
  d[2][0] = tmp1 * (p0[1] - p1[1]);
  d[0][1] = tmp1 * (p2[0] - p1[0]);
  d[1][1] = tmp1 * (p0[0] - p2[0]);
  d[2][1] = tmp1 * (p1[0] - p0[0]);
}
DFM_DEVINL double tet_volume(const double* p0, const double* p1, const double* p2, const double* p3) {
  double v = (p1[0] - p0[0]) * ((p2[1] - p0[1]) * (p3[2] - p0[2]) - (p3[1] - p0[1]) * (p2[2] - p0[2]))
           - (p1[1] - p0[1]) * ((p2[0] - p0[0]) * (p3[2] - p0[2]) - (p3[0] - p0[0]) * (p2[2] - p0[2]))
           + (p1[2] - p0[2]) * ((p2[0] - p0[0]) * (p3[1] - p0[1]) - (p3[0] - p0[0]) * (p2[1] - p0[1]));
  v *= 0.1666666666666;  // the reference's truncated 1/6 (include/delfem/femeqn/ker_emat_tet.h:32-40)
  return v;
}
DFM_DEVINL void tet_dldx(double d[4][3], const double* p0, const double* p1, const double* p2, const double* p3) {
  const double vol = tet_volume(p0, p1, p2, p3);
  const double t = 1.0 / (vol * 6.0);
  d[0][0] = -t * ((p2[1] - p1[1]) * (p3[2] - p1[2]) - (p3[1] - p1[1]) * (p2[2] - p1[2]));
  d[0][1] = +t * ((p2[0] - p1[0]) * (p3[2] - p1[2]) - (p3[0] - p1[0]) * (p2[2] - p1[2]));
  d[0][2] = -t * ((p2[0] - p1[0]) * (p3[1] - p1[1]) - (p3[0] - p1[0]) * (p2[1] - p1[1]));
  d[1][0] = +t * ((p3[1] - p2[1]) * (p0[2] - p2[2]) - (p0[1] - p2[1]) * (p3[2] - p2[2]));
  d[1][1] = -t * ((p3[0] - p2[0]) * (p0[2] - p2[2]) - (p0[0] - p2[0]) * (p3[2] - p2[2]));
  d[1][2] = +t * ((p3[0] - p2[0]) * (p0[1] - p2[1]) - (p0[0] - p2[0]) * (p3[1] - p2[1]));
  d[2][0] = -t * ((p0[1] - p3[1]) * (p1[2] - p3[2]) - (p1[1] - p3[1]) * (p0[2] - p3[2]));
  d[2][1] = +t * ((p0[0] - p3[0]) * (p1[2] - p3[2]) - (p1[0] - p3[0]) * (p0[2] - p3[2]));
  d[2][2] = -t * ((p0[0] - p3[0]) * (p1[1] - p3[1]) - (p1[0] - p3[0]) * (p0[1] - p3[1]));
  d[3][0] = +t * ((p1[1] - p0[1]) * (p2[2] - p0[2]) - (p2[1] - p0[1]) * (p1[2] - p0[2]));
  d[3][1] = -t * ((p1[0] - p0[0]) * (p2[2] - p0[2]) - (p2[0] - p0[0]) * (p1[2] - p0[2]));
  d[3][2] = +t * ((p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]));
}

// ------------------------------------------------ element kinds (row `a` only)
struct AsmParams {
  double p[6];          // kind parameters (alpha,source | lambda,myu,rho,g.. | wave_length)
  const double* coef;   // per-element multiplier or nullptr
  const double* u;      // current field or nullptr (res += f_e - K_e u_e)
};

enum { K_POISSON = 0, K_SOLID2D = 1, K_SOLID3D = 2, K_HELM = 3, K_SOMMER = 4 };

template <int KIND> struct Kind;

// Poisson P1 triangle, b = 1
template <> struct Kind<K_POISSON> {
  static constexpr int NNO = 3, NDIM = 2, BW = 1, RW = 1;  // block width (doubles), residual width
  DFM_DEVINL static void row(const AsmParams& P, unsigned e, const int* no, const double* X, int a, double* blk,
                             double* res) {
    const double *p0 = X + 2 * no[0], *p1 = X + 2 * no[1], *p2 = X + 2 * no[2];
    const double area = tri_area(p0, p1, p2);
    double d[3][2];
    tri_dldx(d, p0, p1, p2);
    const double alpha = P.coef ? P.p[0] * P.coef[e] : P.p[0];
    double em[3];
    for (int c = 0; c < 3; c++) em[c] = alpha * area * (d[a][0] * d[c][0] + d[a][1] * d[c][1]);
    for (int c = 0; c < 3; c++) blk[c] = em[c];
    double r = P.p[1] * area * 0.33333333333333333;
    if (P.u)
      for (int c = 0; c < 3; c++) r -= em[c] * P.u[no[c]];
    res[0] = r;
  }
};

// linear solid P1 triangle, b = 2 (plane stress via lambda*)
template <> struct Kind<K_SOLID2D> {
  static constexpr int NNO = 3, NDIM = 2, BW = 4, RW = 2;
  DFM_DEVINL static void row(const AsmParams& P, unsigned e, const int* no, const double* X, int a, double* blk,
                             double* res) {
    const double *p0 = X + 2 * no[0], *p1 = X + 2 * no[1], *p2 = X + 2 * no[2];
    const double lambda = P.coef ? P.p[0] * P.coef[e] : P.p[0];
    const double myu = P.coef ? P.p[1] * P.coef[e] : P.p[1];
    const double area = tri_area(p0, p1, p2);
    double d[3][2];
    tri_dldx(d, p0, p1, p2);
    double em[3][4];
    for (int c = 0; c < 3; c++) {
      em[c][0] = area * (lambda + myu) * d[a][0] * d[c][0];
      em[c][1] = area * (lambda * d[a][0] * d[c][1] + myu * d[c][0] * d[a][1]);
      em[c][2] = area * (lambda * d[a][1] * d[c][0] + myu * d[c][1] * d[a][0]);
      em[c][3] = area * (lambda + myu) * d[a][1] * d[c][1];
      const double dtmp1 = (d[a][1] * d[c][1] + d[a][0] * d[c][0]) * area * myu;
      em[c][0] += dtmp1;
      em[c][3] += dtmp1;
    }
    for (int c = 0; c < 3; c++)
      for (int q = 0; q < 4; q++) blk[c * 4 + q] = em[c][q];
    double r0 = area * P.p[2] * P.p[3] * 0.33333333333333333;
    double r1 = area * P.p[2] * P.p[4] * 0.33333333333333333;
    if (P.u)
      for (int c = 0; c < 3; c++) {
        const double* uc = P.u + 2 * no[c];
        r0 -= em[c][0] * uc[0] + em[c][1] * uc[1];
        r1 -= em[c][2] * uc[0] + em[c][3] * uc[1];
      }
    res[0] = r0;
    res[1] = r1;
  }
};

// linear solid P1 tetrahedron, b = 3
template <> struct Kind<K_SOLID3D> {
  static constexpr int NNO = 4, NDIM = 3, BW = 9, RW = 3;
  DFM_DEVINL static void row(const AsmParams& P, unsigned, const int* no, const double* X, int a, double* blk,
                             double* res) {
    const double *p0 = X + 3 * no[0], *p1 = X + 3 * no[1], *p2 = X + 3 * no[2], *p3 = X + 3 * no[3];
    const double lambda = P.p[0], myu = P.p[1];
    const double vol = tet_volume(p0, p1, p2, p3);
    double d[4][3];
    tet_dldx(d, p0, p1, p2, p3);
    for (int c = 0; c < 4; c++) {
      double* m = blk + c * 9;
      for (int r = 0; r < 3; r++)
        for (int s = 0; s < 3; s++) m[r * 3 + s] = vol * (lambda * d[a][r] * d[c][s] + myu * d[c][r] * d[a][s]);
      const double dtmp1 = d[a][0] * d[c][0] + d[a][1] * d[c][1] + d[a][2] * d[c][2];
      m[0] += vol * myu * dtmp1;
      m[4] += vol * myu * dtmp1;
      m[8] += vol * myu * dtmp1;
    }
    for (int r = 0; r < 3; r++) {
      double v = vol * P.p[2] * P.p[3 + r] * 0.25;
      if (P.u)
        for (int c = 0; c < 4; c++) {
          const double* uc = P.u + 3 * no[c];
          const double* m = blk + c * 9 + r * 3;
          v -= m[0] * uc[0] + m[1] * uc[1] + m[2] * uc[2];
        }
      res[r] = v;
    }
  }
};

// Helmholtz P1 triangle, complex b = 1 (blocks and residual as (re, im))
template <> struct Kind<K_HELM> {
  static constexpr int NNO = 3, NDIM = 2, BW = 2, RW = 2;
  DFM_DEVINL static void row(const AsmParams& P, unsigned, const int* no, const double* X, int a, double* blk,
                             double* res) {
    const double *p0 = X + 2 * no[0], *p1 = X + 2 * no[1], *p2 = X + 2 * no[2];
    const double area = tri_area(p0, p1, p2);
    double d[3][2];
    tri_dldx(d, p0, p1, p2);
    double em[3];
    for (int c = 0; c < 3; c++) em[c] = area * (d[a][0] * d[c][0] + d[a][1] * d[c][1]);
    const double k = 2 * 3.1416 / P.p[0];  // the reference's truncated pi (eqn_helmholtz.cpp:113)
    const double tmp_val = k * k * area / 12.0;
    em[a] -= tmp_val;
    for (int c = 0; c < 3; c++) em[c] -= tmp_val;
    for (int c = 0; c < 3; c++) {
      blk[2 * c] = em[c];
      blk[2 * c + 1] = 0.0;
    }
    double rr = 0.0, ri = 0.0;
    if (P.u)
      for (int c = 0; c < 3; c++) {  // res -= em * u (complex, em real)
        const double ur = P.u[2 * no[c]], ui = P.u[2 * no[c] + 1];
        const double pr = em[c] * ur - 0.0 * ui, pi = em[c] * ui + 0.0 * ur;
        rr -= pr;
        ri -= pi;
      }
    res[0] = rr;
    res[1] = ri;
  }
};

// Sommerfeld radiation condition on a boundary bar, complex b = 1
template <> struct Kind<K_SOMMER> {
  static constexpr int NNO = 2, NDIM = 2, BW = 2, RW = 2;
  DFM_DEVINL static void row(const AsmParams& P, unsigned, const int* no, const double* X, int a, double* blk,
                             double* res) {
    const double *c0 = X + 2 * no[0], *c1 = X + 2 * no[1];
    const double elen = sqrt((c0[0] - c1[0]) * (c0[0] - c1[0]) + (c0[1] - c1[1]) * (c0[1] - c1[1]));
    const double k = 2 * 3.1416 / P.p[0];
    const double s1 = k / 6.0 * elen, s2 = -1 / (2.0 * elen * k);
    const double t1r = s1 * 0.0, t1i = s1 * 1.0, t2r = s2 * 0.0, t2i = s2 * 1.0;
    const double dr = 2 * t1r + t2r, di = 2 * t1i + t2i;  // tmp_val1*2 + tmp_val2
    const double orr = t1r - t2r, oi = t1i - t2i;         // tmp_val1 - tmp_val2
    for (int c = 0; c < 2; c++) {
      blk[2 * c] = (c == a) ? dr : orr;
      blk[2 * c + 1] = (c == a) ? di : oi;
    }
    double rr = 0.0, ri = 0.0;
    if (P.u)
      for (int c = 0; c < 2; c++) {
        const double er = blk[2 * c], ei = blk[2 * c + 1];
        const double ur = P.u[2 * no[c]], ui = P.u[2 * no[c] + 1];
        rr -= er * ur - ei * ui;
        ri -= er * ui + ei * ur;
      }
    res[0] = rr;
    res[1] = ri;
  }
};

DFM_DEVINL int find_slot_asm(const unsigned* colind, unsigned s0, unsigned s1, unsigned j) {
  while (s0 < s1) {
    const unsigned m = (s0 + s1) >> 1;
    const unsigned c = __ldg(colind + m);
    if (c == j) return (int)m;
    if (c < j) s0 = m + 1; else s1 = m;
  }
  return -1;
}

// One batch of up to 32 elements of one kind around node i: lanes compute rows
// into shared memory (blk: [k][c][BW], tgt: [k][c] = slot or -1); then every lane
// adds the contributions to its own slots in element order.
template <int KIND, int NSLOT_REG>
DFM_DEVINL void gather_kind(const AsmParams& P, unsigned i, const unsigned* ptr, const unsigned* lst, const int* elem,
                            const double* X, const unsigned* colind, unsigned s0, unsigned s1, double* sblk, int* stgt,
                            double* sres, double (&acc)[NSLOT_REG][Kind<KIND>::BW], double* racc, int lane) {
  using K = Kind<KIND>;
  constexpr int NNO = K::NNO, BW = K::BW, RW = K::RW;
  const unsigned nslot = s1 - s0 + 1;
  const unsigned e0 = ptr[i], e1 = ptr[i + 1];
  for (unsigned eb = e0; eb < e1; eb += 32) {
    const unsigned nb = min(32u, e1 - eb);
    if ((unsigned)lane < nb) {
      const unsigned e = lst[eb + lane];
      int no[NNO];
      int a = 0;
      for (int c = 0; c < NNO; c++) {
        no[c] = elem[(size_t)e * NNO + c];
        if ((unsigned)no[c] == i) a = c;
      }
      K::row(P, e, no, X, a, sblk + (size_t)lane * NNO * BW, sres + lane * RW);
      for (int c = 0; c < NNO; c++) {
        int t;
        if (c == a) t = (int)nslot - 1;
        else {
          const int s = find_slot_asm(colind, s0, s1, (unsigned)no[c]);
          t = (s < 0) ? -1 : s - (int)s0;  // not in the pattern: skipped, as in Mearge
        }
        stgt[lane * NNO + c] = t;
      }
    }
    __syncwarp();
#pragma unroll
    for (int p = 0; p < NSLOT_REG; p++) {
      const int j = lane + 32 * p;
      if (j >= (int)nslot) continue;
      for (unsigned k = 0; k < nb; k++)
        for (int c = 0; c < NNO; c++)
          if (stgt[k * NNO + c] == j)
            for (int q = 0; q < BW; q++) acc[p][q] += sblk[((size_t)k * NNO + c) * BW + q];
    }
    if (lane == 0)
      for (unsigned k = 0; k < nb; k++)
        for (int q = 0; q < RW; q++) racc[q] += sres[k * RW + q];
    __syncwarp();
  }
}

template <int KIND, int KIND2>
__global__ void __launch_bounds__(32 * kAsmWarps)
k_assemble(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind, double* diag,
           double* off, double* rhs, AsmParams P, const double* __restrict__ X, const int* __restrict__ elem,
           const unsigned* __restrict__ esup_ptr, const unsigned* __restrict__ esup, AsmParams P2,
           const int* __restrict__ elem2, const unsigned* __restrict__ esup2_ptr, const unsigned* __restrict__ esup2,
           const double* __restrict__ load) {
  using K = Kind<KIND>;
  constexpr int NNO = K::NNO, BW = K::BW, RW = K::RW;
  constexpr int NSLOT_REG = 2;  // up to 64 slots per row
  __shared__ double s_blk[kAsmWarps][32 * NNO * BW];
  __shared__ int s_tgt[kAsmWarps][32 * NNO];
  __shared__ double s_res[kAsmWarps][32 * RW];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (unsigned i = blockIdx.x * kAsmWarps + w; i < N; i += gridDim.x * kAsmWarps) {
    const unsigned s0 = rowptr[i], s1 = rowptr[i + 1];
    double acc[NSLOT_REG][BW];
#pragma unroll
    for (int p = 0; p < NSLOT_REG; p++)
#pragma unroll
      for (int q = 0; q < BW; q++) acc[p][q] = 0.0;  // SetZero
    double racc[RW];
#pragma unroll
    for (int q = 0; q < RW; q++) racc[q] = 0.0;     // SetVectorZero
    gather_kind<KIND, NSLOT_REG>(P, i, esup_ptr, esup, elem, X, colind, s0, s1, s_blk[w], s_tgt[w], s_res[w], acc,
                                 racc, lane);
    if (KIND2 >= 0 && esup2_ptr) {  // second element array after the first (Helmholtz bars)
      using K2 = Kind<(KIND2 >= 0 ? KIND2 : KIND)>;
      static_assert(K2::BW == BW && K2::RW == RW, "element kinds of one system share the block width");
      gather_kind<(KIND2 >= 0 ? KIND2 : KIND), NSLOT_REG>(P2, i, esup2_ptr, esup2, elem2, X, colind, s0, s1,
                                                           s_blk[w], s_tgt[w], s_res[w], acc, racc, lane);
    }
    const unsigned nslot = s1 - s0 + 1;
#pragma unroll
    for (int p = 0; p < NSLOT_REG; p++) {
      const unsigned j = lane + 32 * p;
      if (j >= nslot) continue;
      double* out = (j == nslot - 1) ? diag + (size_t)i * BW : off + (size_t)(s0 + j) * BW;
#pragma unroll
      for (int q = 0; q < BW; q++) out[q] = acc[p][q];
    }
    if (lane == 0)  // nodal loads after all element contributions
#pragma unroll
      for (int q = 0; q < RW; q++) rhs[(size_t)i * RW + q] = load ? racc[q] + load[(size_t)i * RW + q] : racc[q];
  }
}

// Dirichlet elimination: rows and columns of fixed DOFs zeroed, diagonal 1,
// residual zeroed (one thread per stored entry).
__global__ void k_dirichlet(unsigned N, unsigned b, const unsigned* __restrict__ rowptr,
                            const unsigned* __restrict__ colind, const int* __restrict__ flags, double* diag,
                            double* off, double* rhs) {
  const unsigned bb = b * b;
  const size_t ncrs = rowptr[N];
  const size_t ndiag = (size_t)N * bb, noff = ncrs * bb;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < ndiag + noff + (size_t)N * b;
       t += (size_t)gridDim.x * blockDim.x) {
    if (t < ndiag) {
      const unsigned i = (unsigned)(t / bb), r = (unsigned)(t % bb) / b, c = (unsigned)(t % bb) % b;
      const bool fr = flags[(size_t)i * b + r] != 0, fc = flags[(size_t)i * b + c] != 0;
      if (fr || fc) diag[t] = (r == c && fr) ? 1.0 : 0.0;
    } else if (t < ndiag + noff) {
      const size_t u = t - ndiag;
      const size_t s = u / bb;
      const unsigned r = (unsigned)(u % bb) / b, c = (unsigned)(u % bb) % b;
      // row of slot s: binary search in rowptr
      unsigned lo = 0, hi = N;
      while (hi - lo > 1) {
        const unsigned m = (lo + hi) >> 1;
        if (rowptr[m] <= s) lo = m; else hi = m;
      }
      const unsigned j = colind[s];
      if (flags[(size_t)lo * b + r] || flags[(size_t)j * b + c]) off[u] = 0.0;
    } else {
      const size_t k = t - ndiag - noff;
      if (rhs && flags[k]) rhs[k] = 0.0;
    }
  }
}

// Adjoint element kernel: grad_e = -lambda_e^T (dK_e/dcoef_e) u_e, where the
// element matrix is linear in its coefficient (K_e = coef_e K_e^0, K_e^0 the
// matrix at the base constants P.p, as the assembly computes it).
template <int KIND>
__global__ void k_coef_grad(unsigned nelem, AsmParams P, const double* __restrict__ X, const int* __restrict__ elem,
                            const double* __restrict__ lam, const double* __restrict__ u, double* __restrict__ grad) {
  using K = Kind<KIND>;
  constexpr int NNO = K::NNO, BW = K::BW, RW = K::RW;
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
    int no[NNO];
#pragma unroll
    for (int c = 0; c < NNO; c++) no[c] = elem[(size_t)e * NNO + c];
    double g = 0.0;
#pragma unroll
    for (int a = 0; a < NNO; a++) {
      double blk[NNO * BW], res[RW];
      K::row(P, e, no, X, a, blk, res);
#pragma unroll
      for (int r = 0; r < RW; r++) {
        double v = 0.0;  // (K_e^0 u_e) at node a, component r
#pragma unroll
        for (int c = 0; c < NNO; c++)
#pragma unroll
          for (int s = 0; s < RW; s++) v += blk[c * BW + r * RW + s] * u[(size_t)no[c] * RW + s];
        g += lam[(size_t)no[a] * RW + r] * v;
      }
    }
    grad[e] = -g;
  }
}

static void node_adjacency(unsigned nnode, unsigned nnoel, unsigned nelem, const int* elem, std::vector<unsigned>& ptr,
                           std::vector<unsigned>& lst) {
  ptr.assign(nnode + 1, 0);
  for (size_t k = 0; k < (size_t)nelem * nnoel; k++) ptr[elem[k] + 1]++;
  for (unsigned i = 0; i < nnode; i++) ptr[i + 1] += ptr[i];
  lst.assign(ptr[nnode], 0);
  std::vector<unsigned> fill(ptr.begin(), ptr.end() - 1);
  for (unsigned e = 0; e < nelem; e++)
    for (unsigned k = 0; k < nnoel; k++) lst[fill[elem[(size_t)e * nnoel + k]]++] = e;
}

template <typename T>
static int up(T** d, const T* h, size_t n, cudaStream_t s) {
  DFM_CUDA_TRY(cudaMalloc((void**)d, sizeof(T) * std::max<size_t>(n, 1)));
  if (n) DFM_CUDA_TRY(cudaMemcpyAsync(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice, s));
  return DFM_OK;
}

template <int KIND, int KIND2>
static int launch_asm(dfm_mesh G, dfm_mat A, const AsmParams& P, const AsmParams& P2, const double* load,
                      double* rhs) {
  if (A->N == 0) return DFM_OK;
  const int grid = std::max(1, (int)std::min<unsigned>((A->N + kAsmWarps - 1) / kAsmWarps, 148u * 16u));
  k_assemble<KIND, KIND2><<<grid, 32 * kAsmWarps, 0, A->ctx->stream>>>(
      A->N, A->d_rowptr, A->d_colind, A->d_diag, A->d_off, rhs, P, G->d_coord, G->d_elem, G->d_esup_ptr, G->d_esup,
      P2, G->d_bar, KIND2 >= 0 ? G->d_bsup_ptr : nullptr, G->d_bsup, load);
  DFM_CUDA_TRY(cudaGetLastError());
  DFM_CUDA_TRY(cudaStreamSynchronize(A->ctx->stream));
  return take_code(A->ctx);
}

static bool rows_fit(dfm_mat A) { return A->max_row + 1 <= 64; }  // slots held in registers

}  // namespace dfm

using namespace dfm;

extern "C" {

int dfm_mesh_create(dfm_ctx c, int ndim, unsigned nnode, const double* coord, unsigned nnoel, unsigned nelem,
                    const int* elem, unsigned nbar, const int* bar, dfm_mesh* out) {
  if (!c || !out || !coord || (nelem && !elem) || (nbar && !bar)) return DFM_ERR_INVALID;
  *out = nullptr;
  if (!((ndim == 2 && nnoel == 3) || (ndim == 3 && nnoel == 4))) return DFM_ERR_UNSUPPORTED;
  for (size_t k = 0; k < (size_t)nelem * nnoel; k++)
    if (elem[k] < 0 || (unsigned)elem[k] >= nnode) return DFM_ERR_INVALID;
  for (size_t k = 0; k < (size_t)nbar * 2; k++)
    if (bar[k] < 0 || (unsigned)bar[k] >= nnode) return DFM_ERR_INVALID;
  dfm_mesh G = new (std::nothrow) dfm_mesh_s();
  if (!G) return DFM_ERR_NOMEM;
  G->ctx = c;
  ctx_retain(c);
  G->ndim = ndim;
  G->nnode = nnode;
  G->nnoel = nnoel;
  G->nelem = nelem;
  G->nbar = nbar;
  std::vector<unsigned> ep, el, bp, bl;
  node_adjacency(nnode, nnoel, nelem, elem, ep, el);
  node_adjacency(nnode, 2, nbar, bar, bp, bl);
  cudaStream_t s = c->stream;
  int rc = up(&G->d_coord, coord, (size_t)nnode * ndim, s);
  if (!rc) rc = up(&G->d_elem, elem, (size_t)nelem * nnoel, s);
  if (!rc) rc = up(&G->d_bar, bar, (size_t)nbar * 2, s);
  if (!rc) rc = up(&G->d_esup_ptr, ep.data(), ep.size(), s);
  if (!rc) rc = up(&G->d_esup, el.data(), el.size(), s);
  if (!rc) rc = up(&G->d_bsup_ptr, bp.data(), bp.size(), s);
  if (!rc) rc = up(&G->d_bsup, bl.data(), bl.size(), s);
  if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = DFM_ERR_CUDA;
  if (rc) {
    dfm_mesh_destroy(G);
    return rc;
  }
  G->h_elem.assign(elem, elem + (size_t)nelem * nnoel);
  G->h_esup_ptr.swap(ep);
  G->h_esup.swap(el);
  *out = G;
  return DFM_OK;
}

// Block pattern of the mesh: node i's row lists every other node sharing an
// element with it, ascending (CMatDia_BlkCrs::AddPattern over the field's
// element connectivity, src/matvec/matdia_blkcrs.cpp:346-505).
int dfm_mesh_pattern(dfm_mesh G, unsigned* rowptr, unsigned* colind, size_t* ncrs) {
  if (!G || !ncrs) return DFM_ERR_INVALID;
  const unsigned n = G->nnode, nno = G->nnoel;
  std::vector<unsigned> mark(n, 0xffffffffu), row;
  size_t total = 0;
  if (rowptr) rowptr[0] = 0;
  for (unsigned i = 0; i < n; i++) {
    row.clear();
    for (unsigned k = G->h_esup_ptr[i]; k < G->h_esup_ptr[i + 1]; k++) {
      const int* no = G->h_elem.data() + (size_t)G->h_esup[k] * nno;
      for (unsigned a = 0; a < nno; a++) {
        const unsigned j = (unsigned)no[a];
        if (j != i && mark[j] != i) {
          mark[j] = i;
          row.push_back(j);
        }
      }
    }
    std::sort(row.begin(), row.end());
    if (colind) std::copy(row.begin(), row.end(), colind + total);
    total += row.size();
    if (total > 0xffffffffull) return DFM_ERR_UNSUPPORTED;
    if (rowptr) rowptr[i + 1] = (unsigned)total;
  }
  *ncrs = total;
  return DFM_OK;
}

int dfm_mesh_destroy(dfm_mesh G) {
  if (!G) return DFM_OK;
  cudaStreamSynchronize(G->ctx->stream);
  cudaFree(G->d_coord);
  cudaFree(G->d_elem);
  cudaFree(G->d_bar);
  cudaFree(G->d_esup_ptr);
  cudaFree(G->d_esup);
  cudaFree(G->d_bsup_ptr);
  cudaFree(G->d_bsup);
  dfm_ctx c = G->ctx;
  delete G;
  ctx_release(c);
  return DFM_OK;
}

int dfm_assemble_poisson2d(dfm_mesh G, dfm_mat A, double alpha, double source, const double* elem_coef,
                           const double* u, const double* load, double* rhs) {
  if (!G || !A || !rhs || G->ndim != 2 || A->b != 1 || A->vt != DFM_REAL || G->nnode != A->N) return DFM_ERR_INVALID;
  if (!rows_fit(A)) return DFM_ERR_UNSUPPORTED;
  AsmParams P = {{alpha, source, 0, 0, 0, 0}, elem_coef, u};
  return launch_asm<K_POISSON, -1>(G, A, P, P, load, rhs);
}

int dfm_assemble_solid2d(dfm_mesh G, dfm_mat A, double lambda, double myu, double rho, double gx, double gy,
                         const double* elem_coef, const double* u, const double* load, double* rhs) {
  if (!G || !A || !rhs || G->ndim != 2 || A->b != 2 || A->vt != DFM_REAL || G->nnode != A->N) return DFM_ERR_INVALID;
  if (!rows_fit(A)) return DFM_ERR_UNSUPPORTED;
  AsmParams P = {{lambda, myu, rho, gx, gy, 0}, elem_coef, u};
  return launch_asm<K_SOLID2D, -1>(G, A, P, P, load, rhs);
}

int dfm_assemble_solid3d(dfm_mesh G, dfm_mat A, double lambda, double myu, double rho, double gx, double gy,
                         double gz, const double* u, const double* load, double* rhs) {
  if (!G || !A || !rhs || G->ndim != 3 || A->b != 3 || A->vt != DFM_REAL || G->nnode != A->N) return DFM_ERR_INVALID;
  if (!rows_fit(A)) return DFM_ERR_UNSUPPORTED;
  AsmParams P = {{lambda, myu, rho, gx, gy, gz}, nullptr, u};
  return launch_asm<K_SOLID3D, -1>(G, A, P, P, load, rhs);
}

int dfm_assemble_helmholtz2d(dfm_mesh G, dfm_mat A, double wave_length, const double* u, const double* load,
                             double* rhs) {
  if (!G || !A || !rhs || G->ndim != 2 || A->vt != DFM_COMPLEX || G->nnode != A->N) return DFM_ERR_INVALID;
  if (!rows_fit(A)) return DFM_ERR_UNSUPPORTED;
  AsmParams P = {{wave_length, 0, 0, 0, 0, 0}, nullptr, u};
  if (G->nbar) return launch_asm<K_HELM, K_SOMMER>(G, A, P, P, load, rhs);
  return launch_asm<K_HELM, -1>(G, A, P, P, load, rhs);
}

int dfm_coef_grad_poisson2d(dfm_mesh G, double alpha, const double* lam, const double* u, double* grad) {
  if (!G || !lam || !u || !grad || G->ndim != 2) return DFM_ERR_INVALID;
  if (G->nelem == 0) return DFM_OK;
  AsmParams P = {{alpha, 0, 0, 0, 0, 0}, nullptr, nullptr};
  const int grid = (int)std::min<unsigned>((G->nelem + 255) / 256, (unsigned)G->ctx->nsm * 8);
  k_coef_grad<K_POISSON><<<grid, 256, 0, G->ctx->stream>>>(G->nelem, P, G->d_coord, G->d_elem, lam, u, grad);
  DFM_CUDA_TRY(cudaGetLastError());
  DFM_CUDA_TRY(cudaStreamSynchronize(G->ctx->stream));
  return DFM_OK;
}

int dfm_coef_grad_solid2d(dfm_mesh G, double lambda, double myu, const double* lam, const double* u,
                          double* grad) {
  if (!G || !lam || !u || !grad || G->ndim != 2) return DFM_ERR_INVALID;
  if (G->nelem == 0) return DFM_OK;
  AsmParams P = {{lambda, myu, 0, 0, 0, 0}, nullptr, nullptr};
  const int grid = (int)std::min<unsigned>((G->nelem + 255) / 256, (unsigned)G->ctx->nsm * 8);
  k_coef_grad<K_SOLID2D><<<grid, 256, 0, G->ctx->stream>>>(G->nelem, P, G->d_coord, G->d_elem, lam, u, grad);
  DFM_CUDA_TRY(cudaGetLastError());
  DFM_CUDA_TRY(cudaStreamSynchronize(G->ctx->stream));
  return DFM_OK;
}

int dfm_apply_dirichlet(dfm_mat A, const int* flags, double* rhs) {
  if (!A || !flags || A->vt != DFM_REAL) return DFM_ERR_INVALID;
  if (A->N == 0) return DFM_OK;
  const size_t total = (size_t)A->N * A->b * A->b + (size_t)A->ncrs * A->b * A->b + (size_t)A->N * A->b;
  const int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)A->ctx->nsm * 16);
  k_dirichlet<<<grid, 256, 0, A->ctx->stream>>>(A->N, A->b, A->d_rowptr, A->d_colind, flags, A->d_diag, A->d_off, rhs);
  DFM_CUDA_TRY(cudaGetLastError());
  DFM_CUDA_TRY(cudaStreamSynchronize(A->ctx->stream));
  return DFM_OK;
}

}  // extern "C"
