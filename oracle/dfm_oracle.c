/* dfm_oracle.c - plain-C restatement of the reference's linear-solve path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the "port" CPU baseline).  Every
 * routine follows the reference function cited beside it, with the same
 * floating-point operation order, and the file is compiled with
 * -ffp-contract=off, so its results are bit-identical to the reference's own
 * code built the same way (pinned by tests/test_oracle_pin.py).
 * See dfm_oracle.h for the layout conventions. */
#include "dfm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ pattern */

int dfo_pattern(int nnode, int nnoel, int nelem, const int* elem, unsigned* rowptr,
                unsigned* colind, unsigned* ncrs) {
  /* node -> elements, elements in increasing order (MakePointSurElem, elem_ary.cpp:675-724) */
  unsigned* esi = (unsigned*)calloc((size_t)nnode + 1, sizeof(unsigned));
  for (int e = 0; e < nelem; e++)
    for (int k = 0; k < nnoel; k++) esi[elem[(size_t)e * nnoel + k] + 1]++;
  for (int i = 0; i < nnode; i++) esi[i + 1] += esi[i];
  unsigned* es = (unsigned*)malloc(sizeof(unsigned) * (esi[nnode] + 1));
  unsigned* fill = (unsigned*)malloc(sizeof(unsigned) * ((size_t)nnode + 1));
  memcpy(fill, esi, sizeof(unsigned) * ((size_t)nnode + 1));
  for (int e = 0; e < nelem; e++)
    for (int k = 0; k < nnoel; k++) es[fill[elem[(size_t)e * nnoel + k]]++] = (unsigned)e;
  /* node -> nodes, self excluded (MakePointSurPoint with isnt_self, :821-892) */
  int* mark = (int*)malloc(sizeof(int) * (size_t)nnode);
  for (int i = 0; i < nnode; i++) mark[i] = -1;
  unsigned cnt = 0;
  if (rowptr) rowptr[0] = 0;
  for (int i = 0; i < nnode; i++) {
    mark[i] = i;
    const unsigned r0 = cnt;
    for (unsigned q = esi[i]; q < esi[i + 1]; q++) {
      const int* en = elem + (size_t)es[q] * nnoel;
      for (int k = 0; k < nnoel; k++) {
        const int j = en[k];
        if (mark[j] != i) {
          mark[j] = i;
          if (colind) colind[cnt] = (unsigned)j;
          cnt++;
        }
      }
    }
    if (colind) { /* ascending per row (CIndexedArray::Sort, indexed_array.h:113-131) */
      for (unsigned a = r0 + 1; a < cnt; a++) {
        const unsigned v = colind[a];
        unsigned b = a;
        while (b > r0 && colind[b - 1] > v) { colind[b] = colind[b - 1]; b--; }
        colind[b] = v;
      }
    }
    if (rowptr) rowptr[i + 1] = cnt;
  }
  *ncrs = cnt;
  free(mark); free(fill); free(es); free(esi);
  return 0;
}

void dfo_diaind(unsigned N, const unsigned* rowptr, const unsigned* colind, unsigned* diaind) {
  for (unsigned i = 0; i < N; i++) {
    diaind[i] = rowptr[i + 1];
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++)
      if (colind[s] > i) { diaind[i] = s; break; }
  }
}

/* ILU(k) symbolic fill, CMatDiaFrac_BlkCrs::AddFracPtn(lev_fill)
 * (src/matvec/matdiafrac_blkcrs.cpp:1249-1377) with its sorted row list
 * CListRLN (include/delfem/matvec/matdiafrac_blkcrs.h:185-300).  Row i starts
 * from A's entries at level 0.  Its pivots k < i are visited in ascending
 * order, fill entries included as they appear; a pivot is used only when
 * lev(i,k) + 1 <= lev_fill, and then every j of row k's upper part (of the
 * already finished fill pattern) with lev(k,j) + 1 <= lev_fill and j != i is
 * added with level max(lev(i,k), lev(k,j)) + 1 - unless row i holds j
 * already, whose level is then left as it is (CListRLN::Insert returns
 * without touching it).  lev_fill = -1 means no limit.  Here the sorted list
 * is a linked list over column numbers (next[]) with a per-column level
 * (ABSENT when not in the row); the resulting pattern is the same. */
#define DFO_ABSENT 0xffffffffu
int dfo_iluk_pattern(unsigned N, const unsigned* rowptr, const unsigned* colind, int lev_fill,
                     unsigned* frowptr, unsigned** fcolind_out, unsigned** flev_out) {
  return dfo_iluk_pattern_rows(N, rowptr, colind, lev_fill, 0, NULL, N, frowptr, fcolind_out, flev_out);
}

/* The same with CMatDiaFrac_BlkCrs::AddFracPtn(lev_fill, aBlkFill)
 * (src/matvec/matdiafrac_blkcrs.cpp:1379-1500): a row listed in aBlkFill has
 * the fill flag -1, and a candidate (i, j) is dropped only when its level
 * exceeds lev_fill and neither row i nor row j is flagged; the pivot loop
 * therefore cannot skip a pivot on its level alone when row i may take
 * flagged fill.  Flags apply to pairs with i, j < bound (the rows of the
 * matrix that AddFracPtn saw when this one is a joined system).  The early
 * return for lev_fill == 0 needs an empty list. */
int dfo_iluk_pattern_rows(unsigned N, const unsigned* rowptr, const unsigned* colind, int lev_fill,
                          unsigned nrows, const unsigned* rows, unsigned bound, unsigned* frowptr,
                          unsigned** fcolind_out, unsigned** flev_out) {
  const unsigned ncrs0 = rowptr[N];
  size_t cap = (size_t)ncrs0 * 4 + 16, nf = 0;
  unsigned* fcol = (unsigned*)malloc(cap * sizeof(unsigned));
  unsigned* flev = (unsigned*)malloc(cap * sizeof(unsigned));
  unsigned* fdia = (unsigned*)malloc((N ? N : 1) * sizeof(unsigned));
  unsigned* lv = (unsigned*)malloc((N ? N : 1) * sizeof(unsigned));
  unsigned* nx = (unsigned*)malloc((N ? N : 1) * sizeof(unsigned));
  const unsigned END = DFO_ABSENT;
  unsigned char* flag = (unsigned char*)calloc(N ? N : 1, 1);
  for (unsigned t = 0; t < nrows; t++) {
    if (rows[t] >= bound || bound > N) {
      free(fcol); free(flev); free(fdia); free(lv); free(nx); free(flag);
      return -1;
    }
    flag[rows[t]] = 1;
  }
  const int no_fill = (lev_fill == 0 && nrows == 0) || ncrs0 == 0 || (size_t)ncrs0 == (size_t)N * (N ? N - 1 : 0);
  for (unsigned j = 0; j < N; j++) lv[j] = DFO_ABSENT;
  frowptr[0] = 0;
  for (unsigned i = 0; i < N; i++) {
    /* the row's list: A's entries, ascending, level 0 */
    unsigned head = END, tail = END;
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
      const unsigned c = colind[s];
      lv[c] = 0;
      nx[c] = END;
      if (tail == END) head = c; else nx[tail] = c;
      tail = c;
    }
    if (!no_fill) {
      const int flagged_i = i < bound && flag[i];
      const int may_flag = nrows > 0 && i < bound;  /* row i can take fill of a flagged row j */
      for (unsigned k = head; k != END; k = nx[k]) {
        const unsigned lik = lv[k];
        if (!may_flag && lev_fill != -1 && lik + 1 > (unsigned)lev_fill) continue;
        if (k >= i) break;
        unsigned hint = k; /* every new j lies after k */
        for (unsigned s = fdia[k]; s < frowptr[k + 1]; s++) {
          const unsigned lkj = flev[s];
          const unsigned j = fcol[s];
          const unsigned lmax = lik > lkj ? lik : lkj;
          const int unlimited = lev_fill == -1 || (j < bound && (flagged_i || flag[j]));
          if (!unlimited && lmax + 1 > (unsigned)lev_fill) continue;
          if (j == i || lv[j] != DFO_ABSENT) continue;
          while (nx[hint] != END && nx[hint] < j) hint = nx[hint];
          nx[j] = nx[hint];
          nx[hint] = j;
          lv[j] = (lik > lkj ? lik : lkj) + 1;
          hint = j;
        }
      }
    }
    /* finish the row (CListRLN::Finalize): entries in order, m_DiaInd */
    fdia[i] = END;
    for (unsigned c = head; c != END; c = nx[c]) {
      if (nf == cap) {
        cap *= 2;
        fcol = (unsigned*)realloc(fcol, cap * sizeof(unsigned));
        flev = (unsigned*)realloc(flev, cap * sizeof(unsigned));
      }
      if (fdia[i] == END && c > i) fdia[i] = (unsigned)nf;
      fcol[nf] = c;
      flev[nf] = lv[c];
      nf++;
    }
    frowptr[i + 1] = (unsigned)nf;
    if (fdia[i] == END) fdia[i] = (unsigned)nf;
    for (unsigned c = head; c != END; c = nx[c]) lv[c] = DFO_ABSENT;
  }
  free(fdia);
  free(lv);
  free(nx);
  free(flag);
  *fcolind_out = fcol;
  if (flev_out) *flev_out = flev; else free(flev);
  return 0;
}

void dfo_free(void* p) { free(p); }

/* CMatDiaFrac_BlkCrs::SetValue_Initialize (include/delfem/matvec/matdiafrac_blkcrs.h:90-117):
 * the factor's values are zero except where A has an entry, which is copied. */
void dfo_iluk_init(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                   const double* diag, const double* off, const unsigned* frowptr,
                   const unsigned* fcolind, double* fdiag, double* foff) {
  const size_t bb = (size_t)b * b;
  memcpy(fdiag, diag, sizeof(double) * bb * N);
  memset(foff, 0, sizeof(double) * bb * frowptr[N]);
  for (unsigned i = 0; i < N; i++) {
    unsigned t = frowptr[i];
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
      while (fcolind[t] != colind[s]) t++; /* A's row is a sorted subset of the factor's */
      memcpy(foff + t * bb, off + s * bb, sizeof(double) * bb);
    }
  }
}

unsigned dfo_levels_fwd(unsigned N, const unsigned* rowptr, const unsigned* colind,
                        const unsigned* diaind, unsigned* lev) {
  unsigned nl = 0;
  for (unsigned i = 0; i < N; i++) {
    unsigned l = 0;
    for (unsigned s = rowptr[i]; s < diaind[i]; s++) {
      const unsigned c = lev[colind[s]] + 1;
      if (c > l) l = c;
    }
    lev[i] = l;
    if (l + 1 > nl) nl = l + 1;
  }
  return nl;
}

unsigned dfo_levels_bwd(unsigned N, const unsigned* rowptr, const unsigned* colind,
                        const unsigned* diaind, unsigned* lev) {
  unsigned nl = 0;
  for (unsigned ii = N; ii > 0; ii--) {
    const unsigned i = ii - 1;
    unsigned l = 0;
    for (unsigned s = diaind[i]; s < rowptr[i + 1]; s++) {
      const unsigned c = lev[colind[s]] + 1;
      if (c > l) l = c;
    }
    lev[i] = l;
    if (l + 1 > nl) nl = l + 1;
  }
  return nl;
}

/* ------------------------------------------------------------ element kernels */

/* TriArea / TriDlDx (src/femeqn/ker_emat_tri.cpp:13-52) */
static double tri_area(const double* p0, const double* p1, const double* p2) {
  return 0.5 * ((p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]));
}
static void tri_dldx(double dldx[3][2], const double* p0, const double* p1, const double* p2) {
  const double area = tri_area(p0, p1, p2);
  const double tmp1 = 0.5 / area;
  dldx[0][0] = tmp1 * (p1[1] - p2[1]);
  dldx[1][0] = tmp1 * (p2[1] - p0[1]);
  dldx[2][0] = tmp1 * (p0[1] - p1[1]);
  dldx[0][1] = tmp1 * (p2[0] - p1[0]);
  dldx[1][1] = tmp1 * (p0[0] - p2[0]);
  dldx[2][1] = tmp1 * (p1[0] - p0[0]);
}
/* TetVolume / TetDlDx (include/delfem/femeqn/ker_emat_tet.h:32-77), including
 * the reference's truncated 1/6 constant. */
static double tet_volume(const double* p0, const double* p1, const double* p2, const double* p3) {
  double v = (p1[0] - p0[0]) * ((p2[1] - p0[1]) * (p3[2] - p0[2]) - (p3[1] - p0[1]) * (p2[2] - p0[2]))
           - (p1[1] - p0[1]) * ((p2[0] - p0[0]) * (p3[2] - p0[2]) - (p3[0] - p0[0]) * (p2[2] - p0[2]))
           + (p1[2] - p0[2]) * ((p2[0] - p0[0]) * (p3[1] - p0[1]) - (p3[0] - p0[0]) * (p2[1] - p0[1]));
  v *= 0.1666666666666;
  return v;
}
static void tet_dldx(double d[4][3], const double* p0, const double* p1, const double* p2, const double* p3) {
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

static long find_slot(const unsigned* rowptr, const unsigned* colind, unsigned i, unsigned j) {
  for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++)
    if (colind[s] == j) return (long)s;
  return -1;
}

/* CMatDia_BlkCrs::Mearge (src/matvec/matdia_blkcrs.cpp:165-258): element block
 * (a,c) of an nno-node element adds into the diagonal block (a == c) or the
 * off-diagonal slot of node c in node a's row; a missing slot is skipped. */
static void merge_blocks(const unsigned* rowptr, const unsigned* colind, int nno, const int* no,
                         int bb, const double* emat, double* diag, double* off) {
  for (int a = 0; a < nno; a++) {
    const unsigned i = (unsigned)no[a];
    for (int c = 0; c < nno; c++) {
      const double* in = emat + (size_t)(a * nno + c) * bb;
      double* out;
      if (a == c) out = diag + (size_t)i * bb;
      else {
        const long s = find_slot(rowptr, colind, i, (unsigned)no[c]);
        if (s < 0) continue;
        out = off + (size_t)s * bb;
      }
      for (int k = 0; k < bb; k++) out[k] += in[k];
    }
  }
}

/* AddLinearSystem_Poisson2D_P1 (src/femeqn/eqn_poisson.cpp:49-125) */
void dfo_asm_poisson_tri(const unsigned* rowptr, const unsigned* colind, int nelem,
                         const int* elem, const double* coord, double alpha, double source,
                         const double* coef, const double* u, double* diag, double* off,
                         double* res) {
  for (int e = 0; e < nelem; e++) {
    const int* no = elem + 3 * (size_t)e;
    const double *p0 = coord + 2 * no[0], *p1 = coord + 2 * no[1], *p2 = coord + 2 * no[2];
    const double area = tri_area(p0, p1, p2);
    double dldx[3][2];
    tri_dldx(dldx, p0, p1, p2);
    const double a = coef ? alpha * coef[e] : alpha;
    double emat[3][3], eres[3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        emat[i][j] = a * area * (dldx[i][0] * dldx[j][0] + dldx[i][1] * dldx[j][1]);
    for (int i = 0; i < 3; i++) eres[i] = source * area * 0.33333333333333333;
    if (u)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) eres[i] -= emat[i][j] * u[no[j]];
    merge_blocks(rowptr, colind, 3, no, 1, &emat[0][0], diag, off);
    for (int i = 0; i < 3; i++) res[no[i]] += eres[i];
  }
}

/* AddLinSys_LinearSolid2D_Static_P1 (src/femeqn/eqn_linear_solid2d.cpp:505-598) */
void dfo_asm_solid2d_tri(const unsigned* rowptr, const unsigned* colind, int nelem,
                         const int* elem, const double* coord, double lambda0, double myu0,
                         double rho, double gx, double gy, const double* coef, const double* u,
                         double* diag, double* off, double* res) {
  for (int e = 0; e < nelem; e++) {
    const int* no = elem + 3 * (size_t)e;
    const double *p0 = coord + 2 * no[0], *p1 = coord + 2 * no[1], *p2 = coord + 2 * no[2];
    const double lambda = coef ? lambda0 * coef[e] : lambda0;
    const double myu = coef ? myu0 * coef[e] : myu0;
    const double area = tri_area(p0, p1, p2);
    double dldx[3][2];
    tri_dldx(dldx, p0, p1, p2);
    double emat[3][3][2][2], eres[3][2];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        emat[i][j][0][0] = area * (lambda + myu) * dldx[i][0] * dldx[j][0];
        emat[i][j][0][1] = area * (lambda * dldx[i][0] * dldx[j][1] + myu * dldx[j][0] * dldx[i][1]);
        emat[i][j][1][0] = area * (lambda * dldx[i][1] * dldx[j][0] + myu * dldx[j][1] * dldx[i][0]);
        emat[i][j][1][1] = area * (lambda + myu) * dldx[i][1] * dldx[j][1];
        const double dtmp1 = (dldx[i][1] * dldx[j][1] + dldx[i][0] * dldx[j][0]) * area * myu;
        emat[i][j][0][0] += dtmp1;
        emat[i][j][1][1] += dtmp1;
      }
    for (int i = 0; i < 3; i++) {
      eres[i][0] = area * rho * gx * 0.33333333333333333;
      eres[i][1] = area * rho * gy * 0.33333333333333333;
    }
    if (u)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          const double* uj = u + 2 * no[j];
          eres[i][0] -= emat[i][j][0][0] * uj[0] + emat[i][j][0][1] * uj[1];
          eres[i][1] -= emat[i][j][1][0] * uj[0] + emat[i][j][1][1] * uj[1];
        }
    merge_blocks(rowptr, colind, 3, no, 4, &emat[0][0][0][0], diag, off);
    for (int i = 0; i < 3; i++) {
      res[2 * no[i] + 0] += eres[i][0];
      res[2 * no[i] + 1] += eres[i][1];
    }
  }
}

/* AddLinSys_LinearSolid3D_Static_P1 (src/femeqn/eqn_linear_solid3d.cpp:241-334) */
void dfo_asm_solid3d_tet(const unsigned* rowptr, const unsigned* colind, int nelem,
                         const int* elem, const double* coord, double lambda, double myu,
                         double rho, double gx, double gy, double gz, const double* u,
                         double* diag, double* off, double* res) {
  for (int e = 0; e < nelem; e++) {
    const int* no = elem + 4 * (size_t)e;
    const double *p0 = coord + 3 * no[0], *p1 = coord + 3 * no[1], *p2 = coord + 3 * no[2],
                 *p3 = coord + 3 * no[3];
    const double vol = tet_volume(p0, p1, p2, p3);
    double d[4][3];
    tet_dldx(d, p0, p1, p2, p3);
    double emat[4][4][3][3], eres[4][3];
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++)
            emat[i][j][r][c] = vol * (lambda * d[i][r] * d[j][c] + myu * d[j][r] * d[i][c]);
        const double dtmp1 = d[i][0] * d[j][0] + d[i][1] * d[j][1] + d[i][2] * d[j][2];
        emat[i][j][0][0] += vol * myu * dtmp1;
        emat[i][j][1][1] += vol * myu * dtmp1;
        emat[i][j][2][2] += vol * myu * dtmp1;
      }
    for (int i = 0; i < 4; i++) {
      eres[i][0] = vol * rho * gx * 0.25;
      eres[i][1] = vol * rho * gy * 0.25;
      eres[i][2] = vol * rho * gz * 0.25;
      if (u)
        for (int j = 0; j < 4; j++) {
          const double* uj = u + 3 * no[j];
          for (int r = 0; r < 3; r++)
            eres[i][r] -= emat[i][j][r][0] * uj[0] + emat[i][j][r][1] * uj[1] + emat[i][j][r][2] * uj[2];
        }
    }
    merge_blocks(rowptr, colind, 4, no, 9, &emat[0][0][0][0], diag, off);
    for (int i = 0; i < 4; i++)
      for (int r = 0; r < 3; r++) res[3 * no[i] + r] += eres[i][r];
  }
}

/* complex helpers, Com::Complex arithmetic (include/delfem/complex.h:82-156) */
typedef struct { double re, im; } zc;
static zc zmul(zc a, zc b) { zc r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static zc zsub(zc a, zc b) { zc r = {a.re - b.re, a.im - b.im}; return r; }
static zc zadd(zc a, zc b) { zc r = {a.re + b.re, a.im + b.im}; return r; }
static zc zld(const double* p) { zc r = {p[0], p[1]}; return r; }
static void zst(double* p, zc v) { p[0] = v.re; p[1] = v.im; }
static zc zinv(double d, zc c) { /* operator/(double, Complex) */
  const double fact = d / (c.re * c.re + c.im * c.im);
  zc r = {fact * c.re, -fact * c.im};
  return r;
}

/* AddLinearSystem_Helmholtz2D_P1 (src/femeqn/eqn_helmholtz.cpp:51-137) */
void dfo_asm_helmholtz_tri(const unsigned* rowptr, const unsigned* colind, int nelem,
                           const int* elem, const double* coord, double wave_length,
                           const double* u, double* diag, double* off, double* res) {
  for (int e = 0; e < nelem; e++) {
    const int* no = elem + 3 * (size_t)e;
    const double *p0 = coord + 2 * no[0], *p1 = coord + 2 * no[1], *p2 = coord + 2 * no[2];
    const double area = tri_area(p0, p1, p2);
    double dldx[3][2];
    tri_dldx(dldx, p0, p1, p2);
    double emat[3][3][2];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        emat[i][j][0] = area * (dldx[i][0] * dldx[j][0] + dldx[i][1] * dldx[j][1]);
        emat[i][j][1] = 0.0;
      }
    const double k = 2 * 3.1416 / wave_length;
    const double tmp_val = k * k * area / 12.0;
    for (int i = 0; i < 3; i++) {
      emat[i][i][0] -= tmp_val; /* Complex -= double: real part only */
      for (int j = 0; j < 3; j++) emat[i][j][0] -= tmp_val;
    }
    if (u)
      for (int i = 0; i < 3; i++) {
        zc r = {0.0, 0.0};
        for (int j = 0; j < 3; j++) r = zsub(r, zmul(zld(emat[i][j]), zld(u + 2 * no[j])));
        zst(res + 2 * no[i], zadd(zld(res + 2 * no[i]), r));
      }
    merge_blocks(rowptr, colind, 3, no, 2, &emat[0][0][0], diag, off);
  }
}

/* AddLinearSystem_SommerfeltRadiationBC2D_B1 (src/femeqn/eqn_helmholtz.cpp:437-512) */
void dfo_asm_sommerfeld_bar(const unsigned* rowptr, const unsigned* colind, int nbar,
                            const int* bar, const double* coord, double wave_length,
                            const double* u, double* diag, double* off, double* res) {
  for (int e = 0; e < nbar; e++) {
    const int* no = bar + 2 * (size_t)e;
    const double *c0 = coord + 2 * no[0], *c1 = coord + 2 * no[1];
    const double elen = sqrt((c0[0] - c1[0]) * (c0[0] - c1[0]) + (c0[1] - c1[1]) * (c0[1] - c1[1]));
    const double k = 2 * 3.1416 / wave_length;
    /* tmp_val1 = (k/6*elen)*i, tmp_val2 = -1/(2*elen*k)*i, as Com::Complex products */
    const zc I = {0.0, 1.0};
    const double s1 = k / 6.0 * elen, s2 = -1 / (2.0 * elen * k);
    zc t1 = {s1 * I.re, s1 * I.im}, t2 = {s2 * I.re, s2 * I.im};
    zc t1x2 = {2 * t1.re, 2 * t1.im}; /* tmp_val1*2 : Complex*double */
    double emat[2][2][2];
    zst(emat[0][0], zadd(t1x2, t2));
    zst(emat[0][1], zsub(t1, t2));
    zst(emat[1][0], zsub(t1, t2));
    zst(emat[1][1], zadd(t1x2, t2));
    if (u)
      for (int i = 0; i < 2; i++) {
        zc r = {0.0, 0.0};
        for (int j = 0; j < 2; j++) r = zsub(r, zmul(zld(emat[i][j]), zld(u + 2 * no[j])));
        zst(res + 2 * no[i], zadd(zld(res + 2 * no[i]), r));
      }
    merge_blocks(rowptr, colind, 2, no, 2, &emat[0][0][0], diag, off);
  }
}

/* ------------------------------------------------------------------- BC */

void dfo_apply_bc(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                  const int* flags, double* diag, double* off, double* res) {
  const unsigned bb = b * b;
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) {
      if (!flags[i * b + d]) continue;
      for (unsigned k = 0; k < b; k++) diag[i * bb + k * b + d] = 0.0;
      for (unsigned k = 0; k < b; k++) diag[i * bb + d * b + k] = 0.0;
      diag[i * bb + d * b + d] = 1.0;
      for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++)
        for (unsigned k = 0; k < b; k++) off[(size_t)s * bb + d * b + k] = 0.0;
    }
  for (unsigned s = 0; s < rowptr[N]; s++) {
    const unsigned j = colind[s];
    for (unsigned d = 0; d < b; d++) {
      if (!flags[j * b + d]) continue;
      for (unsigned k = 0; k < b; k++) off[(size_t)s * bb + k * b + d] = 0.0;
    }
  }
  if (res)
    for (unsigned i = 0; i < N * b; i++)
      if (flags[i]) res[i] = 0.0;
}

/* ----------------------------------------------------------------- SpMV */

void dfo_spmv(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
              const double* diag, const double* off, double alpha, const double* x,
              double beta, double* y) {
  if (b == 1) {
    for (unsigned i = 0; i < N; i++) {
      double yi = y[i] * beta;
      for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) yi += alpha * off[s] * x[colind[s]];
      yi += alpha * diag[i] * x[i];
      y[i] = yi;
    }
  } else if (b == 2) {
    for (unsigned i = 0; i < N; i++) {
      double y0 = y[2 * i] * beta, y1 = y[2 * i + 1] * beta;
      for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
        const double* m = off + 4 * (size_t)s;
        const double* xj = x + 2 * colind[s];
        y0 += alpha * (m[0] * xj[0] + m[1] * xj[1]);
        y1 += alpha * (m[2] * xj[0] + m[3] * xj[1]);
      }
      const double* m = diag + 4 * (size_t)i;
      const double* xi = x + 2 * i;
      y0 += alpha * (m[0] * xi[0] + m[1] * xi[1]);
      y1 += alpha * (m[2] * xi[0] + m[3] * xi[1]);
      y[2 * i] = y0; y[2 * i + 1] = y1;
    }
  } else {
    for (unsigned i = 0; i < N; i++) {
      double y0 = y[3 * i] * beta, y1 = y[3 * i + 1] * beta, y2 = y[3 * i + 2] * beta;
      for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
        const double* m = off + 9 * (size_t)s;
        const double* xj = x + 3 * colind[s];
        y0 += alpha * (m[0] * xj[0] + m[1] * xj[1] + m[2] * xj[2]);
        y1 += alpha * (m[3] * xj[0] + m[4] * xj[1] + m[5] * xj[2]);
        y2 += alpha * (m[6] * xj[0] + m[7] * xj[1] + m[8] * xj[2]);
      }
      const double* m = diag + 9 * (size_t)i;
      const double* xi = x + 3 * i;
      y0 += alpha * (m[0] * xi[0] + m[1] * xi[1] + m[2] * xi[2]);
      y1 += alpha * (m[3] * xi[0] + m[4] * xi[1] + m[5] * xi[2]);
      y2 += alpha * (m[6] * xi[0] + m[7] * xi[1] + m[8] * xi[2]);
      y[3 * i] = y0; y[3 * i + 1] = y1; y[3 * i + 2] = y2;
    }
  }
}

/* ------------------------------------------------------------------ ILU(0) */

/* CalcInvMat3 (src/matvec/matdiafrac_blkcrs.cpp:138-160) */
static void inv3(double* a) {
  const double det = a[0] * a[4] * a[8] + a[3] * a[7] * a[2] + a[6] * a[1] * a[5]
                   - a[0] * a[7] * a[5] - a[6] * a[4] * a[2] - a[3] * a[1] * a[8];
  const double inv_det = 1.0 / det;
  double t[9];
  for (int i = 0; i < 9; i++) t[i] = a[i];
  a[0] = inv_det * (t[4] * t[8] - t[5] * t[7]);
  a[1] = inv_det * (t[2] * t[7] - t[1] * t[8]);
  a[2] = inv_det * (t[1] * t[5] - t[2] * t[4]);
  a[3] = inv_det * (t[5] * t[6] - t[3] * t[8]);
  a[4] = inv_det * (t[0] * t[8] - t[2] * t[6]);
  a[5] = inv_det * (t[2] * t[3] - t[0] * t[5]);
  a[6] = inv_det * (t[3] * t[7] - t[4] * t[6]);
  a[7] = inv_det * (t[1] * t[6] - t[0] * t[7]);
  a[8] = inv_det * (t[0] * t[4] - t[1] * t[3]);
}

unsigned dfo_ilu0(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                  const unsigned* diaind, double* diag, double* off) {
  const unsigned bb = b * b;
  long* pos = (long*)malloc(sizeof(long) * (N ? N : 1));
  for (unsigned j = 0; j < N; j++) pos[j] = -1;
  unsigned nsing = 0;
  for (unsigned i = 0; i < N; i++) {
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) pos[colind[s]] = (long)s;
    /* row i -= L_ik * (D^-1 U)_kj over the pattern, k ascending */
    for (unsigned ik = rowptr[i]; ik < diaind[i]; ik++) {
      const unsigned k = colind[ik];
      const double* l = off + (size_t)ik * bb;
      for (unsigned kj = diaind[k]; kj < rowptr[k + 1]; kj++) {
        const unsigned j = colind[kj];
        const double* u = off + (size_t)kj * bb;
        double* a;
        if (j != i) {
          if (pos[j] < 0) continue;
          a = off + (size_t)pos[j] * bb;
        } else a = diag + (size_t)i * bb;
        if (b == 1) {
          a[0] -= l[0] * u[0];
        } else if (b == 2) {
          a[0] -= l[0] * u[0] + l[1] * u[2];
          a[1] -= l[0] * u[1] + l[1] * u[3];
          a[2] -= l[2] * u[0] + l[3] * u[2];
          a[3] -= l[2] * u[1] + l[3] * u[3];
        } else {
          for (int r = 0; r < 3; r++) {
            a[r * 3 + 0] -= l[r * 3 + 0] * u[0] + l[r * 3 + 1] * u[3] + l[r * 3 + 2] * u[6];
            a[r * 3 + 1] -= l[r * 3 + 0] * u[1] + l[r * 3 + 1] * u[4] + l[r * 3 + 2] * u[7];
            a[r * 3 + 2] -= l[r * 3 + 0] * u[2] + l[r * 3 + 1] * u[5] + l[r * 3 + 2] * u[8];
          }
        }
      }
    }
    /* D_i <- D_i^-1 (closed forms), singular pivots counted, not inverted */
    double* d = diag + (size_t)i * bb;
    if (b == 1) {
      const double v = d[0];
      if (fabs(v) > 1.0e-30) d[0] = 1.0 / v;
      else nsing++;
    } else if (b == 2) {
      const double det = d[0] * d[3] - d[1] * d[2];
      if (fabs(det) > 1.0e-30) {
        const double inv_det = 1.0 / det;
        const double t = d[0];
        d[0] = inv_det * d[3];
        d[1] = -inv_det * d[1];
        d[2] = -inv_det * d[2];
        d[3] = inv_det * t;
      } else nsing++;
    } else {
      const double det = d[0] * d[4] * d[8] + d[3] * d[7] * d[2] + d[6] * d[1] * d[5]
                       - d[0] * d[7] * d[5] - d[6] * d[4] * d[2] - d[3] * d[1] * d[8];
      if (fabs(det) > 1.0e-30) inv3(d);
      else nsing++;
    }
    if (nsing > 10) break; /* nmax_sing (:774) exceeded: the reference returns false */
    /* U_i <- D_i^-1 U_i */
    for (unsigned ij = diaind[i]; ij < rowptr[i + 1]; ij++) {
      double* u = off + (size_t)ij * bb;
      if (b == 1) {
        u[0] = u[0] * d[0];
      } else if (b == 2) {
        double t[4];
        for (int q = 0; q < 4; q++) t[q] = u[q];
        u[0] = d[0] * t[0] + d[1] * t[2];
        u[1] = d[0] * t[1] + d[1] * t[3];
        u[2] = d[2] * t[0] + d[3] * t[2];
        u[3] = d[2] * t[1] + d[3] * t[3];
      } else {
        double t[9];
        for (int q = 0; q < 9; q++) t[q] = u[q];
        for (int r = 0; r < 3; r++) {
          u[r * 3 + 0] = d[r * 3 + 0] * t[0] + d[r * 3 + 1] * t[3] + d[r * 3 + 2] * t[6];
          u[r * 3 + 1] = d[r * 3 + 0] * t[1] + d[r * 3 + 1] * t[4] + d[r * 3 + 2] * t[7];
          u[r * 3 + 2] = d[r * 3 + 0] * t[2] + d[r * 3 + 1] * t[5] + d[r * 3 + 2] * t[8];
        }
      }
    }
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) pos[colind[s]] = -1;
  }
  free(pos);
  return nsing;
}

void dfo_fwd(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
             const unsigned* diaind, const double* fdiag, const double* foff, double* v) {
  const unsigned bb = b * b;
  for (unsigned i = 0; i < N; i++) {
    double t[3] = {0, 0, 0};
    for (unsigned d = 0; d < b; d++) t[d] = v[i * b + d];
    for (unsigned s = rowptr[i]; s < diaind[i]; s++) {
      const double* m = foff + (size_t)s * bb;
      const double* xj = v + (size_t)colind[s] * b;
      if (b == 1) t[0] -= m[0] * xj[0];
      else if (b == 2) {
        t[0] -= m[0] * xj[0] + m[1] * xj[1];
        t[1] -= m[2] * xj[0] + m[3] * xj[1];
      } else {
        t[0] -= m[0] * xj[0] + m[1] * xj[1] + m[2] * xj[2];
        t[1] -= m[3] * xj[0] + m[4] * xj[1] + m[5] * xj[2];
        t[2] -= m[6] * xj[0] + m[7] * xj[1] + m[8] * xj[2];
      }
    }
    const double* d = fdiag + (size_t)i * bb;
    if (b == 1) v[i] = d[0] * t[0];
    else if (b == 2) {
      v[2 * i] = d[0] * t[0] + d[1] * t[1];
      v[2 * i + 1] = d[2] * t[0] + d[3] * t[1];
    } else {
      v[3 * i] = d[0] * t[0] + d[1] * t[1] + d[2] * t[2];
      v[3 * i + 1] = d[3] * t[0] + d[4] * t[1] + d[5] * t[2];
      v[3 * i + 2] = d[6] * t[0] + d[7] * t[1] + d[8] * t[2];
    }
  }
}

void dfo_bwd(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
             const unsigned* diaind, const double* foff, double* v) {
  const unsigned bb = b * b;
  for (unsigned ii = N; ii > 0; ii--) {
    const unsigned i = ii - 1;
    double t[3] = {0, 0, 0};
    for (unsigned d = 0; d < b; d++) t[d] = v[i * b + d];
    for (unsigned s = diaind[i]; s < rowptr[i + 1]; s++) {
      const double* m = foff + (size_t)s * bb;
      const double* xj = v + (size_t)colind[s] * b;
      if (b == 1) t[0] -= m[0] * xj[0];
      else if (b == 2) {
        t[0] -= m[0] * xj[0] + m[1] * xj[1];
        t[1] -= m[2] * xj[0] + m[3] * xj[1];
      } else {
        t[0] -= m[0] * xj[0] + m[1] * xj[1] + m[2] * xj[2];
        t[1] -= m[3] * xj[0] + m[4] * xj[1] + m[5] * xj[2];
        t[2] -= m[6] * xj[0] + m[7] * xj[1] + m[8] * xj[2];
      }
    }
    for (unsigned d = 0; d < b; d++) v[i * b + d] = t[d];
  }
}

/* --------------------------------------------------------------- Krylov */

static double vdot(size_t n, const double* a, const double* b) {
  double s = 0.0;
  for (size_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}
static void vaxpy(size_t n, double alpha, const double* x, double* y) { /* CLinearSystem::AXPY */
  if (alpha == 0) return;
  for (size_t i = 0; i < n; i++) y[i] += alpha * x[i];
}
static void vscal(size_t n, double alpha, double* x) {
  for (size_t i = 0; i < n; i++) x[i] *= alpha;
}
static void precond(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                    const unsigned* diaind, const double* fdiag, const double* foff, double* v) {
  dfo_fwd(N, b, rowptr, colind, diaind, fdiag, foff, v);
  dfo_bwd(N, b, rowptr, colind, diaind, foff, v);
}

int dfo_pcg(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
            const unsigned* diaind, const double* diag, const double* off, const double* fdiag,
            const double* foff, double* r, double* x, double tol, unsigned maxit,
            unsigned* iters, double* conv, double* hist) {
  return dfo_pcg_fill(N, b, rowptr, colind, diag, off, rowptr, colind, diaind, fdiag, foff, r, x, tol, maxit,
                      iters, conv, hist);
}

int dfo_pcg_fill(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind, const double* diag,
                 const double* off, const unsigned* frowptr, const unsigned* fcolind, const unsigned* fdiaind,
                 const double* fdiag, const double* foff, double* r, double* x, double tol, unsigned maxit,
                 unsigned* iters, double* conv, double* hist) {
  const size_t n = (size_t)N * b;
  double* p = (double*)calloc(n ? n : 1, sizeof(double));
  double* z = (double*)calloc(n ? n : 1, sizeof(double));
  vscal(n, 0.0, x);
  const double sq0 = vdot(n, r, r);
  if (sq0 < 1.0e-30) {
    *conv = 0.0; *iters = 0;
    free(p); free(z);
    return 1;
  }
  const double inv0 = 1.0 / sq0;
  memcpy(z, r, n * sizeof(double));
  precond(N, b, frowptr, fcolind, fdiaind, fdiag, foff, z);
  memcpy(p, z, n * sizeof(double));
  double rz = vdot(n, r, z);
  for (unsigned it = 0; it < maxit; it++) {
    dfo_spmv(N, b, rowptr, colind, diag, off, 1.0, p, 0.0, z);
    const double pap = vdot(n, p, z);
    const double alpha = rz / pap;
    vaxpy(n, -alpha, z, r);
    vaxpy(n, alpha, p, x);
    const double sq = vdot(n, r, r);
    if (hist) hist[it] = sqrt(sq * inv0);
    if (sq * inv0 < tol * tol) {
      *conv = sqrt(sq * inv0);
      *iters = it;
      free(p); free(z);
      return 1;
    }
    memcpy(z, r, n * sizeof(double));
    precond(N, b, frowptr, fcolind, fdiaind, fdiag, foff, z);
    const double rz_new = vdot(n, r, z);
    const double beta = rz_new / rz;
    rz = rz_new;
    vscal(n, beta, p);
    vaxpy(n, 1.0, z, p);
  }
  *conv = sqrt(vdot(n, r, r) * inv0);
  *iters = maxit;
  free(p); free(z);
  return 0;
}

/* LsSol::Solve_CG (src/ls/solver_ls_iter.cpp:31-97): no preconditioner.
   x = 0 (SCAL by 0); |r0|^2 < 1e-60 returns true with num_iter = 0 and
   conv_ratio = |r0|; the loop index is num_iter; at max_iter the loop ends
   with num_iter = max_iter, conv_ratio untouched and true returned. */
int dfo_cg(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind, const double* diag,
           const double* off, double* r, double* x, double tol, unsigned maxit, unsigned* iters, double* conv) {
  const size_t n = (size_t)N * b;
  double* p = (double*)calloc(n ? n : 1, sizeof(double));
  double* Ap = (double*)calloc(n ? n : 1, sizeof(double));
  vscal(n, 0.0, x);
  double sq = vdot(n, r, r);
  if (sq < 1.0e-60) {
    *iters = 0;
    *conv = sqrt(sq);
    free(p); free(Ap);
    return 1;
  }
  const double inv0 = 1.0 / sq;
  memcpy(p, r, n * sizeof(double));
  unsigned it;
  for (it = 0; it < maxit; it++) {
    dfo_spmv(N, b, rowptr, colind, diag, off, 1.0, p, 0.0, Ap);
    const double alpha = sq / vdot(n, p, Ap);
    vaxpy(n, alpha, p, x);
    vaxpy(n, -alpha, Ap, r);
    const double sq_new = vdot(n, r, r);
    if (sq_new * inv0 < tol * tol) {
      *conv = sqrt(sq_new * inv0);
      break;
    }
    const double beta = sq_new / sq;
    sq = sq_new;
    vscal(n, beta, p);
    vaxpy(n, 1.0, r, p);
  }
  if (it == maxit) *conv = tol;
  *iters = it;
  free(p); free(Ap);
  return 1;
}

int dfo_pbicgstab(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                  const unsigned* diaind, const double* diag, const double* off,
                  const double* fdiag, const double* foff, double* r, double* x, double tol,
                  unsigned maxit, unsigned* iters, double* conv) {
  const size_t n = (size_t)N * b;
  double* w = (double*)calloc(7 * (n ? n : 1), sizeof(double));
  double *s = w, *Ms = w + n, *AMs = w + 2 * n, *p = w + 3 * n, *Mp = w + 4 * n, *AMp = w + 5 * n,
         *r2 = w + 6 * n;
  const double sq0 = vdot(n, r, r);
  if (sq0 < 1.0e-60) {
    *conv = sqrt(sq0); *iters = 0;
    free(w);
    return 1;
  }
  const double inv0 = 1.0 / sq0;
  vscal(n, 0.0, x);
  memcpy(r2, r, n * sizeof(double));
  memcpy(p, r, n * sizeof(double));
  *iters = maxit;
  for (unsigned it = 1; it < maxit; it++) {
    memcpy(Mp, p, n * sizeof(double));
    precond(N, b, rowptr, colind, diaind, fdiag, foff, Mp);
    const double r_r2 = vdot(n, r, r2);
    dfo_spmv(N, b, rowptr, colind, diag, off, 1.0, Mp, 0.0, AMp);
    const double alpha = r_r2 / vdot(n, AMp, r2);
    memcpy(s, r, n * sizeof(double));
    vaxpy(n, -alpha, AMp, s);
    memcpy(Ms, s, n * sizeof(double));
    precond(N, b, rowptr, colind, diaind, fdiag, foff, Ms);
    dfo_spmv(N, b, rowptr, colind, diag, off, 1.0, Ms, 0.0, AMs);
    const double den = vdot(n, AMs, AMs);
    const double num = vdot(n, s, AMs);
    const double omega = num / den;
    vaxpy(n, alpha, Mp, x);
    vaxpy(n, omega, Ms, x);
    memcpy(r, s, n * sizeof(double));
    vaxpy(n, -omega, AMs, r);
    const double sq = vdot(n, r, r);
    if (sq * inv0 < tol * tol) {
      *conv = sqrt(sq * inv0);
      *iters = it;
      free(w);
      return 1;
    }
    const double tmp1 = vdot(n, r, r2);
    const double beta = tmp1 * alpha / (r_r2 * omega);
    vscal(n, beta, p);
    vaxpy(n, 1.0, r, p);
    vaxpy(n, -beta * omega, AMp, p);
  }
  *conv = tol; /* max_iter reached: the reference leaves conv_ratio at its input (the tolerance) */
  free(w);
  return 1; /* and returns true (src/ls/solver_ls_iter.cpp:327-407) */
}

/* ---------------------------------------------------------------- complex */

/* CZMatDia_BlkCrs::MatVec, b = 1 (src/matvec/zmatdia_blkcrs.cpp:737-801) */
void dfo_zspmv(unsigned N, const unsigned* rowptr, const unsigned* colind, const double* diag,
               const double* off, double alpha, const double* x, double beta, double* y) {
  for (unsigned i = 0; i < N; i++) {
    double re = 0, im = 0;
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
      const double* m = off + 2 * (size_t)s;
      const double* xj = x + 2 * (size_t)colind[s];
      re += alpha * (m[0] * xj[0] - m[1] * xj[1]);
      im += alpha * (m[0] * xj[1] + m[1] * xj[0]);
    }
    zc yi = zld(y + 2 * i);
    yi.re *= beta; yi.im *= beta;
    zc acc = {re, im};
    yi = zadd(yi, acc);
    zc ad = {alpha * diag[2 * i], alpha * diag[2 * i + 1]};
    yi = zadd(yi, zmul(ad, zld(x + 2 * i)));
    zst(y + 2 * i, yi);
  }
}

unsigned dfo_zilu0(unsigned N, const unsigned* rowptr, const unsigned* colind,
                   const unsigned* diaind, double* diag, double* off) {
  long* pos = (long*)malloc(sizeof(long) * (N ? N : 1));
  for (unsigned j = 0; j < N; j++) pos[j] = -1;
  unsigned nsmall = 0;
  for (unsigned i = 0; i < N; i++) {
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) pos[colind[s]] = (long)s;
    for (unsigned ik = rowptr[i]; ik < rowptr[i + 1]; ik++) {
      const unsigned k = colind[ik];
      if (k >= i) break;
      const zc ikv = zld(off + 2 * (size_t)ik);
      for (unsigned kj = diaind[k]; kj < rowptr[k + 1]; kj++) {
        const unsigned j = colind[kj];
        const zc kjv = zld(off + 2 * (size_t)kj);
        if (j != i) {
          if (pos[j] < 0) continue;
          double* a = off + 2 * (size_t)pos[j];
          zst(a, zsub(zld(a), zmul(ikv, kjv)));
        } else {
          zst(diag + 2 * i, zsub(zld(diag + 2 * i), zmul(ikv, kjv)));
        }
      }
    }
    const zc piv = zld(diag + 2 * i);
    if (piv.re * piv.re + piv.im * piv.im < 1.0e-20) nsmall++;
    const zc inv = zinv(1.0, piv);
    zst(diag + 2 * i, inv);
    for (unsigned ij = diaind[i]; ij < rowptr[i + 1]; ij++)
      zst(off + 2 * (size_t)ij, zmul(zld(off + 2 * (size_t)ij), inv));
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) pos[colind[s]] = -1;
  }
  free(pos);
  return nsmall;
}

void dfo_zfwdbwd(unsigned N, const unsigned* rowptr, const unsigned* colind,
                 const unsigned* diaind, const double* fdiag, const double* foff, double* v) {
  for (unsigned i = 0; i < N; i++) {
    zc t = zld(v + 2 * i);
    for (unsigned s = rowptr[i]; s < diaind[i]; s++)
      t = zsub(t, zmul(zld(foff + 2 * (size_t)s), zld(v + 2 * (size_t)colind[s])));
    zst(v + 2 * i, zmul(zld(fdiag + 2 * i), t));
  }
  for (unsigned ii = N; ii > 0; ii--) {
    const unsigned i = ii - 1;
    zc t = zld(v + 2 * i);
    for (unsigned s = diaind[i]; s < rowptr[i + 1]; s++)
      t = zsub(t, zmul(zld(foff + 2 * (size_t)s), zld(v + 2 * (size_t)colind[s])));
    zst(v + 2 * i, t);
  }
}

/* CZVector_Blk operator* (unconjugated, src/matvec/zvector_blk.cpp:39-59) */
static zc zdot(unsigned n, const double* a, const double* b) {
  double re = 0, im = 0;
  for (unsigned i = 0; i < n; i++) {
    const double d0 = a[2 * i], d1 = a[2 * i + 1], d2 = b[2 * i], d3 = b[2 * i + 1];
    re += d0 * d2 - d1 * d3;
    im += d0 * d3 + d1 * d2;
  }
  zc r = {re, im};
  return r;
}
/* InnerProduct (conjugated, :62-86), real part for (r, r) */
static double znorm2(unsigned n, const double* a) {
  double re = 0;
  for (unsigned i = 0; i < n; i++) re += a[2 * i] * a[2 * i] + a[2 * i + 1] * a[2 * i + 1];
  return re;
}
static zc zdiv(zc a, zc b) { /* operator/(Complex, Complex) */
  const double fact = 1.0 / (b.re * b.re + b.im * b.im);
  zc r = {(a.re * b.re + a.im * b.im) * fact, (-a.re * b.im + a.im * b.re) * fact};
  return r;
}
static void zaxpy(unsigned n, zc alpha, const double* x, double* y) {
  for (unsigned i = 0; i < n; i++) zst(y + 2 * i, zadd(zld(y + 2 * i), zmul(alpha, zld(x + 2 * i))));
}

int dfo_pcocg_fill(unsigned N, const unsigned* rowptr, const unsigned* colind, const double* diag,
                   const double* off, const unsigned* frowptr, const unsigned* fcolind, const unsigned* fdiaind,
                   const double* fdiag, const double* foff, double* r, double* x, double tol, unsigned maxit,
                   unsigned* iters, double* conv) {
  const size_t n2 = 2 * (size_t)N;
  double* p = (double*)calloc(n2 ? n2 : 1, sizeof(double));
  double* Ap = (double*)calloc(n2 ? n2 : 1, sizeof(double));
  double* w = (double*)calloc(n2 ? n2 : 1, sizeof(double));
  for (size_t i = 0; i < n2; i++) x[i] *= 0.0;
  const double sq0 = znorm2(N, r);
  if (sq0 < 1.0e-30) {
    *conv = 0.0; *iters = 0;
    free(p); free(Ap); free(w);
    return 1;
  }
  const double inv0 = 1.0 / sq0;
  memcpy(w, r, n2 * sizeof(double));
  dfo_zfwdbwd(N, frowptr, fcolind, fdiaind, fdiag, foff, w);
  memcpy(p, w, n2 * sizeof(double));
  zc rw = zdot(N, r, w);
  *iters = maxit;
  for (unsigned it = 1; it < maxit; it++) {
    dfo_zspmv(N, rowptr, colind, diag, off, 1.0, p, 0.0, Ap);
    const zc pap = zdot(N, p, Ap);
    const zc alpha = zdiv(rw, pap);
    zaxpy(N, alpha, p, x);
    const zc malpha = {-alpha.re, -alpha.im};
    zaxpy(N, malpha, Ap, r);
    const double ratio = sqrt(znorm2(N, r) * inv0);
    if (ratio < tol) {
      *conv = ratio;
      *iters = it;
      free(p); free(Ap); free(w);
      return 1;
    }
    memcpy(w, r, n2 * sizeof(double));
    dfo_zfwdbwd(N, frowptr, fcolind, fdiaind, fdiag, foff, w);
    const zc rw2 = zdot(N, r, w);
    const zc beta = zdiv(rw2, rw);
    rw = rw2;
    for (unsigned i = 0; i < N; i++) zst(p + 2 * i, zmul(zld(p + 2 * i), beta));
    const zc one = {1.0, 0.0};
    zaxpy(N, one, w, p);
  }
  *conv = tol; /* max_iter reached: conv_ratio keeps its input (the tolerance) */
  free(p); free(Ap); free(w);
  return 1; /* and Solve_PCOCG returns true (src/femls/zsolver_ls_iter.cpp:213-266) */
}

int dfo_pcocg(unsigned N, const unsigned* rowptr, const unsigned* colind, const unsigned* diaind,
              const double* diag, const double* off, const double* fdiag, const double* foff,
              double* r, double* x, double tol, unsigned maxit, unsigned* iters, double* conv) {
  return dfo_pcocg_fill(N, rowptr, colind, diag, off, rowptr, colind, diaind, fdiag, foff, r, x, tol, maxit, iters,
                        conv);
}

/* ------------------------------------------------ stored-matrix Newmark systems */

/* CMat_BlkCrs::SetBoundaryCondition_Row (src/matvec/mat_blkcrs.cpp:910-951):
   the rows of fixed DOFs zeroed in every block of the row (library layout:
   the diagonal block separate). */
void dfo_mat_zero_rows(unsigned N, unsigned b, const unsigned* rowptr, const int* flags, double* diag, double* off) {
  const unsigned bb = b * b;
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) {
      if (!flags[(size_t)i * b + d]) continue;
      for (unsigned c = 0; c < b; c++) diag[(size_t)i * bb + d * b + c] = 0.0;
      for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++)
        for (unsigned c = 0; c < b; c++) off[(size_t)s * bb + d * b + c] = 0.0;
    }
}

/* One stored-matrix block entry of CMat_BlkCrs::MatVec with alpha = -1 and
   beta = 1 (src/matvec/mat_blkcrs.cpp:955-1175): y += (alpha * m) * x term by
   term. */
static void nm_entry(unsigned b, const double* m, const double* x, double* y) {
  for (unsigned i = 0; i < b; i++)
    for (unsigned j = 0; j < b; j++) y[i] += (-1.0 * m[i * b + j]) * x[j];
}

/* MakeResidual of CLinearSystem_SaveDiaM_Newmark (scheme 1, :446-520) and
   CLinearSystem_SaveDiaM_NewmarkBeta (scheme 2, :706-794): the predictor
   t = u + v*(dt*(1-gamma)) or t = (u + v*dt) + a*((dt*dt)*(0.5-beta))
   (CNodeAry::AddValueFromNodeSegment adds val*alpha), r = force - B t in the
   reference's entry order - its stored matrix has the pattern of
   CMat_BlkCrs::SetPatternDia (:1267-1318): the diagonal block first when the
   row has a column below it, else last - then r = 0 at fixed DOFs and
   *norm = sqrt(r.r).  t is work space. */
void dfo_newmark_residual(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind, const double* diag,
                          const double* off, int scheme, double dt, double gamma, double beta, const double* force,
                          const double* u, const double* v, const double* a, const int* flags, double* t, double* r,
                          double* norm) {
  const size_t n = (size_t)N * b;
  const unsigned bb = b * b;
  const double c1 = scheme == 1 ? dt * (1 - gamma) : dt;
  const double c2 = dt * dt * (0.5 - beta);
  for (size_t k = 0; k < n; k++) {
    t[k] = u[k] + v[k] * c1;
    if (scheme == 2) t[k] = t[k] + a[k] * c2;
  }
  for (size_t k = 0; k < n; k++) r[k] = force[k];
  for (unsigned i = 0; i < N; i++) {
    const int dia_first = rowptr[i + 1] > rowptr[i] && colind[rowptr[i]] < i;
    double* y = r + (size_t)i * b;
    if (dia_first) nm_entry(b, diag + (size_t)i * bb, t + (size_t)i * b, y);
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) nm_entry(b, off + (size_t)s * bb, t + (size_t)colind[s] * b, y);
    if (!dia_first) nm_entry(b, diag + (size_t)i * bb, t + (size_t)i * b, y);
  }
  double s = 0.0;
  for (size_t k = 0; k < n; k++) {
    if (flags[k]) r[k] = 0.0;
    s += r[k] * r[k];
  }
  *norm = sqrt(s);
}

/* UpdateValueOfField of the two (:522-566, :796-877), x the solved update. */
void dfo_newmark_update(size_t n, int scheme, double dt, double gamma, double beta, const int* flags, double* x,
                        double* u, double* v, double* a) {
  for (size_t k = 0; k < n; k++) {
    if (scheme == 1) {
      const double velo0 = v[k];
      if (flags[k] == 0) {
        const double velo1 = x[k];
        u[k] += dt * (1 - gamma) * velo0 + dt * gamma * velo1;
      } else {
        x[k] = velo0;
      }
      v[k] = x[k];
    } else {
      const double velo0 = v[k], acc0 = a[k];
      if (flags[k] == 0) {
        const double acc1 = x[k];
        u[k] += dt * velo0 + dt * dt * (0.5 - beta) * acc0 + dt * dt * beta * acc1;
        v[k] += dt * (1 - gamma) * acc0 + gamma * dt * acc1;
      } else {
        x[k] = acc0;
      }
      a[k] = x[k];
    }
  }
}

/* ------------------------------------------------ complex ILU(k) */

/* CZMatDiaFrac_BlkCrs::SetValue_Initialize over a filled pattern (complex
   scalars as (re, im) pairs): A's entries at their slots, zero elsewhere. */
void dfo_ziluk_init(unsigned N, const unsigned* rowptr, const unsigned* colind, const double* diag,
                    const double* off, const unsigned* frowptr, const unsigned* fcolind, double* fdiag,
                    double* foff) {
  memcpy(fdiag, diag, sizeof(double) * 2 * N);
  memset(foff, 0, sizeof(double) * 2 * frowptr[N]);
  for (unsigned i = 0; i < N; i++) {
    unsigned t = frowptr[i];
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
      while (fcolind[t] != colind[s]) t++; /* A's row is a sorted subset of the factor's */
      foff[2 * (size_t)t] = off[2 * (size_t)s];
      foff[2 * (size_t)t + 1] = off[2 * (size_t)s + 1];
    }
  }
}

/* ------------------------------------------------ rectangular block matrices */

/* CMat_BlkCrs::MatVec, not transposed (src/matvec/mat_blkcrs.cpp:955-1175):
   per block row, y *= beta, then for every block and entry
   y += alpha * m * x (left to right); 1 x 1 blocks with beta == 0 start
   from y = 0 as the reference does. */
void dfo_rmat_spmv(unsigned nrow, unsigned brow, unsigned bcol, const unsigned* rowptr, const unsigned* colind,
                   const double* val, double alpha, const double* x, double beta, double* y) {
  const unsigned bb = brow * bcol;
  for (unsigned i = 0; i < nrow; i++) {
    double* yi = y + (size_t)i * brow;
    if (bb == 1 && beta == 0.0) yi[0] = 0.0;
    else
      for (unsigned r = 0; r < brow; r++) yi[r] *= beta;
    for (unsigned s = rowptr[i]; s < rowptr[i + 1]; s++) {
      const double* m = val + (size_t)s * bb;
      const double* xj = x + (size_t)colind[s] * bcol;
      if (brow == 1 && bcol > 1 && bcol <= 3) { /* the reference's unrolled 1 x 2 and 1 x 3 rows */
        double t = m[0] * xj[0] + m[1] * xj[1];
        if (bcol == 3) t = m[0] * xj[0] + m[1] * xj[1] + m[2] * xj[2];
        yi[0] += alpha * t;
      } else if (bcol == 1 && brow > 1 && brow <= 3) { /* 2 x 1 and 3 x 1: x scaled first */
        const double ax = xj[0] * alpha;
        for (unsigned r = 0; r < brow; r++) yi[r] += m[r] * ax;
      } else {
        for (unsigned r = 0; r < brow; r++)
          for (unsigned c = 0; c < bcol; c++) yi[r] += alpha * m[r * bcol + c] * xj[c];
      }
    }
  }
}
