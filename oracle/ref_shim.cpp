// C-ABI shim that drives the reference's own CPU implementation of the
// linear-solve path.  TEST INFRASTRUCTURE ONLY: it is the checker and the
// timed CPU baseline, never part of the product.  See ref_shim.h.
//
// Call order mirrored from the reference:
//   field level  : src/femeqn/eqnsys_scalar.cpp:213-359 (pattern -> BC -> ILU
//                  symbolic -> InitializeMarge -> element loop -> FinalizeMarge ->
//                  ILU numeric -> Solve_PCG), test_glut_lowlev/solid2d/main.cpp:203-223,
//                  test_glut/helmholtz2d/main.cpp:82-121 (complex COCG).
//   matrix level : LsSol::CLinearSystem::AddLinSysSeg/AddMat_Dia (src/ls/linearsystem.cpp),
//                  MatVec::CMatDiaFrac_BlkCrs (src/matvec/matdiafrac_blkcrs.cpp:227-287, :769).
#include "ref_shim.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>
#include <streambuf>
#include <vector>

#include "delfem/field.h"
#include "delfem/field_world.h"
#include "delfem/mesh3d.h"
#include "delfem/mesh_interface.h"
#include "delfem/mesher2d.h"
#include "delfem/femeqn/eqn_diffusion.h"
#include "delfem/femeqn/eqn_helmholtz.h"
#include "delfem/femeqn/eqn_linear_solid2d.h"
#include "delfem/femeqn/eqn_linear_solid3d.h"
#include "delfem/femeqn/eqn_poisson.h"
#include "delfem/femeqn/ker_emat_tri.h"
#include "delfem/femls/linearsystem_field.h"
#include "delfem/femls/linearsystem_fieldsave.h"
#include "delfem/femls/zlinearsystem.h"
#include "delfem/femls/zpreconditioner.h"
#include "delfem/femls/zsolver_ls_iter.h"
#include "delfem/ls/linearsystem.h"
#include "delfem/ls/preconditioner.h"
#include "delfem/ls/solver_ls_iter.h"
#include "delfem/matvec/bcflag_blk.h"
#include "delfem/matvec/mat_blkcrs.h"
#include "delfem/matvec/matdia_blkcrs.h"
#include "delfem/matvec/matdiafrac_blkcrs.h"
#include "delfem/matvec/vector_blk.h"
#include "delfem/matvec/zmatdia_blkcrs.h"
#include "delfem/matvec/zmatdiafrac_blkcrs.h"
#include "delfem/matvec/zvector_blk.h"

using namespace Fem::Field;

namespace {

// The reference prints progress text through std::cout on every assembly and
// factorisation; the shim keeps the caller's stdout clean.
struct NullBuf : std::streambuf {
  int overflow(int c) override { return c; }
};
struct Quiet {
  NullBuf nb;
  std::streambuf* old;
  Quiet() : old(std::cout.rdbuf(&nb)) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Structured meshes enter the reference through its own mesh interface
// (include/delfem/mesh_interface.h:58-75): id 1 = volume elements, id 2 =
// boundary elements, included in id 1.
class ArrayMesh : public Msh::IMesh {
 public:
  unsigned ndim = 2;
  std::vector<double> coord;
  Msh::MSH_TYPE vol_type = Msh::TRI, bnd_type = Msh::BAR;
  std::vector<int> vol, bnd;
  unsigned int GetDimention() const override { return ndim; }
  void GetInfo(unsigned int id_msh, unsigned int& id_cad_part, unsigned int& id_msh_before_ext,
               unsigned int& inum_ext, int& ilayer) const override {
    id_cad_part = id_msh;
    id_msh_before_ext = 0;
    inum_ext = 0;
    ilayer = 0;
  }
  void GetCoord(std::vector<double>& c) const override { c = coord; }
  Msh::MSH_TYPE GetConnectivity(unsigned int id_msh, std::vector<int>& lnods) const override {
    if (id_msh == 1) { lnods = vol; return vol_type; }
    lnods = bnd;
    return bnd_type;
  }
  std::vector<unsigned int> GetAry_ID() const override {
    std::vector<unsigned int> a(1, 1u);
    if (!bnd.empty()) a.push_back(2u);
    return a;
  }
  std::vector<unsigned int> GetIncludeElemIDAry(unsigned int id_msh) const override {
    std::vector<unsigned int> a;
    if (id_msh == 1 && !bnd.empty()) a.push_back(2u);
    return a;
  }
};

MatVec::CMatDia_BlkCrs* make_mat(unsigned N, unsigned b, const unsigned* rowptr,
                                 const unsigned* colind, const double* diag, const double* off) {
  MatVec::CMatDia_BlkCrs* m = new MatVec::CMatDia_BlkCrs(N, b);
  Com::CIndexedArray crs;
  crs.index.assign(rowptr, rowptr + N + 1);
  crs.array.assign(colind, colind + rowptr[N]);
  m->AddPattern(crs);
  m->SetZero();
  const unsigned bb = b * b;
  for (unsigned i = 0; i < N; i++) {
    std::memcpy(m->GetPtrValDia(i), diag + (size_t)i * bb, sizeof(double) * bb);
    unsigned n = 0;
    double* p = m->GetPtrValPSuP(i, n);
    if (n) std::memcpy(p, off + (size_t)rowptr[i] * bb, sizeof(double) * bb * n);
  }
  return m;
}

void read_mat(const MatVec::CMatDia_BlkCrs& m, unsigned b, double* diag, double* off) {
  const unsigned N = m.NBlkMatCol(), bb = b * b;
  size_t pos = 0;
  for (unsigned i = 0; i < N; i++) {
    if (diag) std::memcpy(diag + (size_t)i * bb, m.GetPtrValDia(i), sizeof(double) * bb);
    unsigned n = 0;
    const double* p = m.GetPtrValPSuP(i, n);
    if (off && n) std::memcpy(off + pos * bb, p, sizeof(double) * bb * n);
    pos += n;
  }
}

MatVec::CZMatDia_BlkCrs* make_zmat(unsigned N, const unsigned* rowptr, const unsigned* colind,
                                   const double* diag, const double* off) {
  MatVec::CZMatDia_BlkCrs* m = new MatVec::CZMatDia_BlkCrs(N, 1);
  Com::CIndexedArray crs;
  crs.index.assign(rowptr, rowptr + N + 1);
  crs.array.assign(colind, colind + rowptr[N]);
  m->AddPattern(crs);
  m->SetZero();
  for (unsigned i = 0; i < N; i++) {
    *m->GetPtrValDia(i) = Com::Complex(diag[2 * i], diag[2 * i + 1]);
    unsigned n = 0;
    Com::Complex* p = m->GetPtrValPSuP(i, n);
    for (unsigned k = 0; k < n; k++) {
      const size_t s = rowptr[i] + k;
      p[k] = Com::Complex(off[2 * s], off[2 * s + 1]);
    }
  }
  return m;
}

void read_zmat(const MatVec::CZMatDia_BlkCrs& m, double* diag, double* off) {
  const unsigned N = m.NBlkMatCol();
  size_t pos = 0;
  for (unsigned i = 0; i < N; i++) {
    const Com::Complex d = *m.GetPtrValDia(i);
    if (diag) { diag[2 * i] = d.Real(); diag[2 * i + 1] = d.Imag(); }
    unsigned n = 0;
    const Com::Complex* p = m.GetPtrValPSuP(i, n);
    for (unsigned k = 0; k < n; k++, pos++) {
      if (off) { off[2 * pos] = p[k].Real(); off[2 * pos + 1] = p[k].Imag(); }
    }
  }
}

}  // namespace

struct dfm_ref_sys {
  int kind = 0;
  unsigned b = 1;
  ArrayMesh mesh;
  CFieldWorld world;
  unsigned id_field = 0, id_bnd = 0, id_ea_vol = 0;
  Fem::Ls::CLinearSystem_Field ls;
  LsSol::CPreconditioner_ILU prec;
  Fem::Ls::CZLinearSystem zls;
  Fem::Ls::CZPreconditioner_ILU zprec;
  std::vector<double> rhs;  // residual right after FinalizeMarge (+ loads)
  bool assembled = false;

  bool complex_kind() const { return kind == DFM_REF_HELMHOLTZ2D; }
  MatVec::CMatDia_BlkCrs& mat() { return ls.m_ls.GetMatrix(0); }
  const MatVec::CMatDia_BlkCrs& mat() const { return ls.m_ls.GetMatrix(0); }
};

// Restatement of the element loop of AddLinearSystem_Poisson2D_P1
// (src/femeqn/eqn_poisson.cpp:49-125) with alpha scaled per element; it merges
// into the reference's own matrix/residual with the reference's Mearge/AddValue.
static void harness_poisson2d_coef(dfm_ref_sys* s, double alpha, double source, const double* coef) {
  const CField& fv = s->world.GetField(s->id_field);
  const CElemAry& ea = s->world.GetEA(s->id_ea_vol);
  const CElemAry::CElemSeg& es_va = fv.GetElemSeg(s->id_ea_vol, CORNER, true, s->world);
  const CElemAry::CElemSeg& es_co = fv.GetElemSeg(s->id_ea_vol, CORNER, false, s->world);
  MatVec::CMatDia_BlkCrs& mat_cc = s->ls.GetMatrix(s->id_field, CORNER, s->world);
  MatVec::CVector_Blk& res_c = s->ls.GetResidual(s->id_field, CORNER, s->world);
  const CNodeAry::CNodeSeg& ns_val = fv.GetNodeSeg(CORNER, true, s->world);
  const CNodeAry::CNodeSeg& ns_co = fv.GetNodeSeg(CORNER, false, s->world);
  for (unsigned ie = 0; ie < ea.Size(); ie++) {
    unsigned no[3];
    double co[3][2], val[3];
    es_co.GetNodes(ie, no);
    for (int k = 0; k < 3; k++) ns_co.GetValue(no[k], co[k]);
    es_va.GetNodes(ie, no);
    for (int k = 0; k < 3; k++) ns_val.GetValue(no[k], &val[k]);
    const double area = TriArea(co[0], co[1], co[2]);
    double dldx[3][2], cterm[3];
    TriDlDx(dldx, cterm, co[0], co[1], co[2]);
    const double a = alpha * coef[ie];
    double emat[3][3], eres[3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        emat[i][j] = a * area * (dldx[i][0] * dldx[j][0] + dldx[i][1] * dldx[j][1]);
    for (int i = 0; i < 3; i++) eres[i] = source * area * 0.33333333333333333;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) eres[i] -= emat[i][j] * val[j];
    mat_cc.Mearge(3, no, 3, no, 1, &emat[0][0]);
    for (int i = 0; i < 3; i++) res_c.AddValue(no[i], 0, eres[i]);
  }
}

// Restatement of AddLinSys_LinearSolid2D_Static_P1 (src/femeqn/eqn_linear_solid2d.cpp:505-598)
// with (lambda, myu) scaled per element.
static void harness_solid2d_coef(dfm_ref_sys* s, double lambda0, double myu0, double rho,
                                 double gx, double gy, const double* coef) {
  const CField& fd = s->world.GetField(s->id_field);
  const CElemAry& ea = s->world.GetEA(s->id_ea_vol);
  const CElemAry::CElemSeg& es_co = fd.GetElemSeg(s->id_ea_vol, CORNER, false, s->world);
  const CElemAry::CElemSeg& es_va = fd.GetElemSeg(s->id_ea_vol, CORNER, true, s->world);
  MatVec::CMatDia_BlkCrs& mat_cc = s->ls.GetMatrix(s->id_field, CORNER, s->world);
  MatVec::CVector_Blk& res_c = s->ls.GetResidual(s->id_field, CORNER, s->world);
  const CNodeAry::CNodeSeg& ns_disp = fd.GetNodeSeg(CORNER, true, s->world, VALUE);
  const CNodeAry::CNodeSeg& ns_co = fd.GetNodeSeg(CORNER, false, s->world, VALUE);
  for (unsigned ie = 0; ie < ea.Size(); ie++) {
    unsigned no[3];
    double co[3][2], disp[3][2];
    es_co.GetNodes(ie, no);
    for (int k = 0; k < 3; k++) ns_co.GetValue(no[k], co[k]);
    es_va.GetNodes(ie, no);
    for (int k = 0; k < 3; k++) ns_disp.GetValue(no[k], disp[k]);
    const double lambda = lambda0 * coef[ie], myu = myu0 * coef[ie];
    const double area = TriArea(co[0], co[1], co[2]);
    double dldx[3][2], zt[3];
    TriDlDx(dldx, zt, co[0], co[1], co[2]);
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
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        eres[i][0] -= emat[i][j][0][0] * disp[j][0] + emat[i][j][0][1] * disp[j][1];
        eres[i][1] -= emat[i][j][1][0] * disp[j][0] + emat[i][j][1][1] * disp[j][1];
      }
    mat_cc.Mearge(3, no, 3, no, 4, &emat[0][0][0][0]);
    for (int i = 0; i < 3; i++) {
      res_c.AddValue(no[i], 0, eres[i][0]);
      res_c.AddValue(no[i], 1, eres[i][1]);
    }
  }
}

extern "C" {

dfm_ref_sys* dfm_ref_create(int kind, int ndim, int nnode, const double* coord, int nnoel,
                            int nelem, const int* elem, int bnd_nnoel, int nbnd, const int* bnd) {
  if (kind < DFM_REF_POISSON2D || kind > DFM_REF_HELMHOLTZ2D) return nullptr;
  Quiet q;
  dfm_ref_sys* s = new dfm_ref_sys;
  s->kind = kind;
  s->mesh.ndim = ndim;
  s->mesh.coord.assign(coord, coord + (size_t)nnode * ndim);
  s->mesh.vol.assign(elem, elem + (size_t)nelem * nnoel);
  s->mesh.vol_type = (nnoel == 4) ? Msh::TET : Msh::TRI;
  if (nbnd > 0) {
    s->mesh.bnd.assign(bnd, bnd + (size_t)nbnd * bnd_nnoel);
    s->mesh.bnd_type = (bnd_nnoel == 2) ? Msh::BAR : Msh::TRI;
  }
  const unsigned id_base = s->world.AddMesh(s->mesh);
  const CIDConvEAMshCad conv = s->world.GetIDConverter(id_base);
  s->id_ea_vol = conv.GetIdEA_fromMsh(1);
  FIELD_TYPE ft = SCALAR;
  s->b = 1;
  if (kind == DFM_REF_SOLID2D) { ft = VECTOR2; s->b = 2; }
  if (kind == DFM_REF_SOLID3D) { ft = VECTOR3; s->b = 3; }
  if (kind == DFM_REF_HELMHOLTZ2D) ft = ZSCALAR;
  s->id_field = s->world.MakeField_FieldElemDim(id_base, ndim, ft, VALUE, CORNER);
  if (nbnd > 0) s->id_bnd = s->world.GetPartialField(s->id_field, conv.GetIdEA_fromMsh(2));
  if (s->complex_kind()) {
    s->zls.AddPattern_Field(s->id_field, s->world);
    s->zprec.SetFillInLevel(0);
    s->zprec.SetLinearSystem(s->zls);
  } else {
    s->ls.AddPattern_Field(s->id_field, s->world);
    if (s->id_bnd) s->ls.SetFixedBoundaryCondition_Field(s->id_bnd, s->world);
    s->prec.SetFillInLevel(0);
    s->prec.SetLinearSystem(s->ls.m_ls);
  }
  return s;
}

void dfm_ref_destroy(dfm_ref_sys* s) {
  Quiet q;
  delete s;
}

int dfm_ref_dims(const dfm_ref_sys* s, unsigned* N, unsigned* b, unsigned* ncrs) {
  if (s->complex_kind()) {
    const MatVec::CZMatDia_BlkCrs& m = s->zls.GetMatrix(0);
    *N = m.NBlkMatCol();
    *ncrs = m.NCrs();
  } else {
    *N = s->mat().NBlkMatCol();
    *ncrs = s->mat().NCrs();
  }
  *b = s->b;
  return 0;
}

int dfm_ref_pattern(const dfm_ref_sys* s, unsigned* rowptr, unsigned* colind) {
  unsigned N, b, ncrs;
  dfm_ref_dims(s, &N, &b, &ncrs);
  rowptr[0] = 0;
  for (unsigned i = 0; i < N; i++) {
    unsigned n = 0;
    const unsigned* p = s->complex_kind() ? s->zls.GetMatrix(0).GetPtrIndPSuP(i, n)
                                          : s->mat().GetPtrIndPSuP(i, n);
    for (unsigned k = 0; k < n; k++) colind[rowptr[i] + k] = p[k];
    rowptr[i + 1] = rowptr[i] + n;
  }
  return 0;
}

int dfm_ref_assemble(dfm_ref_sys* s, const double* p, const double* coef, const double* load,
                     double* res_norm, double* seconds) {
  Quiet q;
  unsigned N, b, ncrs;
  dfm_ref_dims(s, &N, &b, &ncrs);
  const double t0 = now_s();
  double res = 0.0;
  if (s->complex_kind()) {
    s->zls.InitializeMarge();
    Fem::Eqn::AddLinSys_Helmholtz(s->zls, p[0], s->world, s->id_field);
    if (s->id_bnd) Fem::Eqn::AddLinSys_SommerfeltRadiationBC(s->zls, p[0], s->world, s->id_bnd);
    MatVec::CZVector_Blk& r = s->zls.GetVector(-1, 0);
    if (load)
      for (unsigned i = 0; i < N; i++)
        r.SetValue(i, 0, r.GetValue(i, 0) + Com::Complex(load[2 * i], load[2 * i + 1]));
    res = s->zls.FinalizeMarge();
    s->rhs.resize(2 * (size_t)N);
    for (unsigned i = 0; i < N; i++) {
      s->rhs[2 * i] = r.GetValue(i, 0).Real();
      s->rhs[2 * i + 1] = r.GetValue(i, 0).Imag();
    }
  } else {
    s->ls.InitializeMarge();
    switch (s->kind) {
      case DFM_REF_POISSON2D:
        if (coef) harness_poisson2d_coef(s, p[0], p[1], coef);
        else Fem::Eqn::AddLinSys_Poisson(s->ls, p[0], p[1], s->world, s->id_field);
        break;
      case DFM_REF_SOLID2D:
        if (coef) harness_solid2d_coef(s, p[0], p[1], p[2], p[3], p[4], coef);
        else Fem::Eqn::AddLinSys_LinearSolid2D_Static(s->ls, p[0], p[1], p[2], p[3], p[4], s->world, s->id_field);
        break;
      case DFM_REF_SOLID3D:
        Fem::Eqn::AddLinSys_LinearSolid3D_Static(s->ls, p[0], p[1], p[2], p[3], p[4], p[5], s->world, s->id_field);
        break;
    }
    MatVec::CVector_Blk& r = s->ls.m_ls.GetVector(-1, 0);
    if (load)
      for (unsigned i = 0; i < N; i++)
        for (unsigned d = 0; d < b; d++) r.AddValue(i, d, load[(size_t)i * b + d]);
    res = s->ls.FinalizeMarge();
    s->rhs.resize((size_t)N * b);
    for (unsigned i = 0; i < N; i++)
      for (unsigned d = 0; d < b; d++) s->rhs[(size_t)i * b + d] = r.GetValue(i, d);
  }
  const double t1 = now_s();
  if (res_norm) *res_norm = res;
  if (seconds) *seconds = t1 - t0;
  s->assembled = true;
  return 0;
}

int dfm_ref_get_system(const dfm_ref_sys* s, double* diag, double* off, double* rhs) {
  if (!s->assembled) return 1;
  if (s->complex_kind()) read_zmat(s->zls.GetMatrix(0), diag, off);
  else read_mat(s->mat(), s->b, diag, off);
  if (rhs) std::memcpy(rhs, s->rhs.data(), sizeof(double) * s->rhs.size());
  return 0;
}

int dfm_ref_get_bcflag(const dfm_ref_sys* s, int* flags) {
  if (s->complex_kind()) return 1;
  unsigned N, b, ncrs;
  dfm_ref_dims(s, &N, &b, &ncrs);
  // const_cast: CLinearSystem exposes the flags only through a non-const getter.
  MatVec::CBCFlag& f = const_cast<dfm_ref_sys*>(s)->ls.m_ls.GetBCFlag(0);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) flags[(size_t)i * b + d] = f.GetBCFlag(i, d);
  return 0;
}

int dfm_ref_ilu(dfm_ref_sys* s, double* seconds) {
  if (!s->assembled) return 1;
  Quiet q;
  const double t0 = now_s();
  bool ok = true;
  if (s->complex_kind()) ok = s->zprec.SetValue(s->zls);
  else ok = s->prec.SetValue(s->ls.m_ls);
  if (seconds) *seconds = now_s() - t0;
  return ok ? 0 : 1;
}

int dfm_ref_get_ilu(const dfm_ref_sys* s, double* diag, double* off) {
  if (!s->assembled) return 1;
  Quiet q;
  if (s->complex_kind()) {
    MatVec::CZMatDiaFrac_BlkCrs f(0, s->zls.GetMatrix(0));
    f.SetValue_Initialize(s->zls.GetMatrix(0));
    f.DoILUDecomp();
    read_zmat(f, diag, off);
    return 0;
  }
  MatVec::CMatDiaFrac_BlkCrs f(0, s->mat());
  f.SetValue_Initialize(s->mat());
  const bool ok = f.DoILUDecomp();
  read_mat(f, s->b, diag, off);
  return ok ? 0 : 1;
}

int dfm_ref_solve(dfm_ref_sys* s, int method, double tol, unsigned maxit, unsigned* iters,
                  double* conv, double* x, double* seconds) {
  if (!s->assembled) return 1;
  Quiet q;
  unsigned N, b, ncrs;
  dfm_ref_dims(s, &N, &b, &ncrs);
  double c = tol;
  unsigned it = maxit;
  bool ok = false;
  double t0 = 0, t1 = 0;
  if (s->complex_kind()) {
    MatVec::CZVector_Blk& r = s->zls.GetVector(-1, 0);
    for (unsigned i = 0; i < N; i++) r.SetValue(i, 0, Com::Complex(s->rhs[2 * i], s->rhs[2 * i + 1]));
    t0 = now_s();
    ok = Fem::Ls::Solve_PCOCG(c, it, s->zls, s->zprec);
    t1 = now_s();
    MatVec::CZVector_Blk& u = s->zls.GetVector(-2, 0);
    for (unsigned i = 0; i < N; i++) {
      x[2 * i] = u.GetValue(i, 0).Real();
      x[2 * i + 1] = u.GetValue(i, 0).Imag();
    }
  } else {
    MatVec::CVector_Blk& r = s->ls.m_ls.GetVector(-1, 0);
    for (unsigned i = 0; i < N; i++)
      for (unsigned d = 0; d < b; d++) r.SetValue(i, d, s->rhs[(size_t)i * b + d]);
    LsSol::CLinearSystemPreconditioner lsp(s->ls.m_ls, s->prec);
    t0 = now_s();
    if (method == DFM_REF_PBICGSTAB) ok = LsSol::Solve_PBiCGSTAB(c, it, lsp);
    else ok = LsSol::Solve_PCG(c, it, lsp);
    t1 = now_s();
    MatVec::CVector_Blk& u = s->ls.m_ls.GetVector(-2, 0);
    for (unsigned i = 0; i < N; i++)
      for (unsigned d = 0; d < b; d++) x[(size_t)i * b + d] = u.GetValue(i, d);
  }
  *iters = it;
  *conv = c;
  if (seconds) *seconds = t1 - t0;
  return ok ? 0 : 3;
}

int dfm_ref_mat_spmv(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                     const double* diag, const double* off, double alpha, const double* x,
                     double beta, double* y) {
  Quiet q;
  MatVec::CMatDia_BlkCrs* m = make_mat(N, b, rowptr, colind, diag, off);
  MatVec::CVector_Blk vx(N, b), vy(N, b);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) {
      vx.SetValue(i, d, x[(size_t)i * b + d]);
      vy.SetValue(i, d, y[(size_t)i * b + d]);
    }
  m->MatVec(alpha, vx, beta, vy);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) y[(size_t)i * b + d] = vy.GetValue(i, d);
  delete m;
  return 0;
}

int dfm_ref_mat_ilu0(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                     const double* diag, const double* off, double* fdiag, double* foff) {
  Quiet q;
  MatVec::CMatDia_BlkCrs* m = make_mat(N, b, rowptr, colind, diag, off);
  MatVec::CMatDiaFrac_BlkCrs f(0, *m);
  f.SetValue_Initialize(*m);
  const bool ok = f.DoILUDecomp();
  read_mat(f, b, fdiag, foff);
  delete m;
  return ok ? 0 : 1;
}

int dfm_ref_mat_precond(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                        const double* fdiag, const double* foff, double* vec) {
  Quiet q;
  MatVec::CMatDia_BlkCrs* m = make_mat(N, b, rowptr, colind, fdiag, foff);
  // A factor object whose values are the given factor: build the ILU(0) pattern
  // (and m_DiaInd) from m, then overwrite the copied values.
  MatVec::CMatDiaFrac_BlkCrs f(0, *m);
  f.SetValue_Initialize(*m);
  MatVec::CVector_Blk v(N, b);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) v.SetValue(i, d, vec[(size_t)i * b + d]);
  f.ForwardSubstitution(v);
  f.BackwardSubstitution(v);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) vec[(size_t)i * b + d] = v.GetValue(i, d);
  delete m;
  return 0;
}

int dfm_ref_mat_iluk(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                     const double* diag, const double* off, int lev, unsigned cap, unsigned* frowptr,
                     unsigned* fcolind, double* fdiag, double* foff, unsigned* fncrs) {
  return dfm_ref_mat_iluk_rows(N, b, rowptr, colind, diag, off, lev, 0, nullptr, cap, frowptr, fcolind, fdiag, foff,
                               fncrs);
}

// With rows: the preconditioner's SetFillBlk path (src/ls/preconditioner.cpp:
// 91, 140-142): CMatDiaFrac_BlkCrs(0, A), AddFracPtn(lev, aBlkFill), and the
// pattern finalised as SetValue does (MakePatternFinalize).
int dfm_ref_mat_iluk_rows(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                          const double* diag, const double* off, int lev, unsigned nrows, const unsigned* rows,
                          unsigned cap, unsigned* frowptr, unsigned* fcolind, double* fdiag, double* foff,
                          unsigned* fncrs) {
  Quiet q;
  MatVec::CMatDia_BlkCrs* m = make_mat(N, b, rowptr, colind, diag, off);
  MatVec::CMatDiaFrac_BlkCrs f(nrows ? 0 : lev, *m);
  if (nrows) {
    const std::vector<unsigned int> blk(rows, rows + nrows);
    f.AddFracPtn(lev, blk);
    f.MakePatternFinalize();
  }
  *fncrs = f.NCrs();
  if (!frowptr || f.NCrs() > cap) {
    delete m;
    return 2;
  }
  frowptr[0] = 0;
  for (unsigned i = 0; i < N; i++) {
    unsigned n = 0;
    const unsigned* c = f.GetPtrIndPSuP(i, n);
    if (n) std::memcpy(fcolind + frowptr[i], c, sizeof(unsigned) * n);
    frowptr[i + 1] = frowptr[i] + n;
  }
  f.SetValue_Initialize(*m);
  const bool ok = f.DoILUDecomp();
  read_mat(f, b, fdiag, foff);
  delete m;
  return ok ? 0 : 1;
}

int dfm_ref_mat_solve(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                      const double* diag, const double* off, const double* rhs, int method,
                      double tol, unsigned maxit, unsigned* iters, double* conv, double* x,
                      double* t_ilu, double* t_solve) {
  return dfm_ref_mat_solve_lev(N, b, rowptr, colind, diag, off, rhs, method, tol, maxit, 0, iters, conv, x,
                               t_ilu, t_solve);
}

int dfm_ref_mat_solve_lev(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                          const double* diag, const double* off, const double* rhs, int method,
                          double tol, unsigned maxit, int lev, unsigned* iters, double* conv, double* x,
                          double* t_ilu, double* t_solve) {
  Quiet q;
  LsSol::CLinearSystem ls;
  ls.AddLinSysSeg(N, b);
  Com::CIndexedArray crs;
  crs.index.assign(rowptr, rowptr + N + 1);
  crs.array.assign(colind, colind + rowptr[N]);
  ls.AddMat_Dia(0, crs);
  ls.InitializeMarge();
  MatVec::CMatDia_BlkCrs& m = ls.GetMatrix(0);
  const unsigned bb = b * b;
  for (unsigned i = 0; i < N; i++) {
    std::memcpy(m.GetPtrValDia(i), diag + (size_t)i * bb, sizeof(double) * bb);
    unsigned n = 0;
    double* p = m.GetPtrValPSuP(i, n);
    if (n) std::memcpy(p, off + (size_t)rowptr[i] * bb, sizeof(double) * bb * n);
  }
  MatVec::CVector_Blk& r = ls.GetVector(-1, 0);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) r.SetValue(i, d, rhs[(size_t)i * b + d]);
  LsSol::CPreconditioner_ILU prec;
  prec.SetFillInLevel(lev);
  prec.SetLinearSystem(ls);
  double t0 = now_s();
  const bool ilu_ok = prec.SetValue(ls);
  double t1 = now_s();
  if (t_ilu) *t_ilu = t1 - t0;
  if (!ilu_ok) return 1;
  LsSol::CLinearSystemPreconditioner lsp(ls, prec);
  double c = tol;
  unsigned it = maxit;
  t0 = now_s();
  bool ok = (method == DFM_REF_PBICGSTAB) ? LsSol::Solve_PBiCGSTAB(c, it, lsp)
            : (method == DFM_REF_CG)        ? LsSol::Solve_CG(c, it, ls)
                                            : LsSol::Solve_PCG(c, it, lsp);
  t1 = now_s();
  if (t_solve) *t_solve = t1 - t0;
  MatVec::CVector_Blk& u = ls.GetVector(-2, 0);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) x[(size_t)i * b + d] = u.GetValue(i, d);
  *iters = it;
  *conv = c;
  return ok ? 0 : 3;
}

int dfm_ref_zmat_spmv(unsigned N, const unsigned* rowptr, const unsigned* colind,
                      const double* diag, const double* off, double alpha, const double* x,
                      double beta, double* y) {
  Quiet q;
  MatVec::CZMatDia_BlkCrs* m = make_zmat(N, rowptr, colind, diag, off);
  MatVec::CZVector_Blk vx(N, 1), vy(N, 1);
  for (unsigned i = 0; i < N; i++) {
    vx.SetValue(i, 0, Com::Complex(x[2 * i], x[2 * i + 1]));
    vy.SetValue(i, 0, Com::Complex(y[2 * i], y[2 * i + 1]));
  }
  m->MatVec(alpha, vx, beta, vy);
  for (unsigned i = 0; i < N; i++) {
    y[2 * i] = vy.GetValue(i, 0).Real();
    y[2 * i + 1] = vy.GetValue(i, 0).Imag();
  }
  delete m;
  return 0;
}

int dfm_ref_zmat_ilu0(unsigned N, const unsigned* rowptr, const unsigned* colind,
                      const double* diag, const double* off, double* fdiag, double* foff) {
  Quiet q;
  MatVec::CZMatDia_BlkCrs* m = make_zmat(N, rowptr, colind, diag, off);
  MatVec::CZMatDiaFrac_BlkCrs f(0, *m);
  f.SetValue_Initialize(*m);
  f.DoILUDecomp();
  read_zmat(f, fdiag, foff);
  delete m;
  return 0;
}

int dfm_ref_zmat_read(const char* path, unsigned cap, unsigned* N, unsigned* ncrs, unsigned* rowptr,
                      unsigned* colind, double* diag, double* off) {
  Quiet q;
  MatVec::CZMatDia_BlkCrs m{std::string(path)};
  *N = m.NBlkMatCol();
  *ncrs = m.NCrs();
  if (!rowptr || m.NCrs() > cap) return 2;
  rowptr[0] = 0;
  for (unsigned i = 0; i < *N; i++) {
    unsigned n = 0;
    const unsigned* c = m.GetPtrIndPSuP(i, n);
    if (n) std::memcpy(colind + rowptr[i], c, sizeof(unsigned) * n);
    rowptr[i + 1] = rowptr[i] + n;
  }
  read_zmat(m, diag, off);
  return 0;
}

// CLinearSystem_Save's boundary matrix built the reference's way: the pattern
// of CMat_BlkCrs::SetPatternBoundary over K, the entries filled with K's
// values (what the element routines merge into both), the two masks of
// FinalizeMarge, then MakeResidual's product r = force - B u.  B is returned
// row by row in the reference's own entry order (the diagonal block first).
int dfm_ref_boundary_residual(unsigned N, unsigned b, const unsigned* rowptr, const unsigned* colind,
                              const double* diag, const double* off, const int* flags, const double* force,
                              const double* u, unsigned cap, unsigned* brow, unsigned* bcol, double* bval,
                              unsigned* bncrs, double* r) {
  Quiet q;
  MatVec::CMatDia_BlkCrs* K = make_mat(N, b, rowptr, colind, diag, off);
  MatVec::CBCFlag bc(N, b);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++)
      if (flags[(size_t)i * b + d]) bc.SetBC(i, d);
  MatVec::CMat_BlkCrs B(N, b, N, b);
  B.SetPatternBoundary(*K, bc, bc);
  B.SetZero();  // allocates the values (CLinearSystem_Save::InitializeMarge does the same)
  *bncrs = B.NCrs();
  const unsigned bb = b * b;
  for (unsigned i = 0; i < N; i++) {
    unsigned n = 0;
    const unsigned* cols = B.GetPtrIndPSuP(i, n);
    double* vals = B.GetPtrValPSuP(i, n);
    for (unsigned k = 0; k < n; k++) {
      const unsigned j = cols[k];
      const double* src = nullptr;
      if (j == i) src = K->GetPtrValDia(i);
      else {
        unsigned nk = 0;
        const unsigned* kc = K->GetPtrIndPSuP(i, nk);
        const double* kv = K->GetPtrValPSuP(i, nk);
        for (unsigned t = 0; t < nk; t++)
          if (kc[t] == j) src = kv + (size_t)t * bb;
      }
      std::memcpy(vals + (size_t)k * bb, src, sizeof(double) * bb);
    }
  }
  B.SetBoundaryConditionInverse_Colum(bc);
  B.SetBoundaryCondition_Row(bc);
  MatVec::CVector_Blk vu(N, b), vr(N, b);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) {
      vu.SetValue(i, d, u[(size_t)i * b + d]);
      vr.SetValue(i, d, force[(size_t)i * b + d]);
    }
  B.MatVec(-1.0, vu, 1.0, vr, true);
  for (unsigned i = 0; i < N; i++)
    for (unsigned d = 0; d < b; d++) r[(size_t)i * b + d] = vr.GetValue(i, d);
  if (brow && B.NCrs() <= cap) {
    brow[0] = 0;
    for (unsigned i = 0; i < N; i++) {
      unsigned n = 0;
      const unsigned* cols = B.GetPtrIndPSuP(i, n);
      const double* vals = B.GetPtrValPSuP(i, n);
      for (unsigned k = 0; k < n; k++) {
        bcol[brow[i] + k] = cols[k];
        std::memcpy(bval + (size_t)(brow[i] + k) * bb, vals + (size_t)k * bb, sizeof(double) * bb);
      }
      brow[i + 1] = brow[i] + n;
    }
  }
  delete K;
  return 0;
}

// The reference's GiD readers, read back through their public accessors.
int dfm_ref_gid_read(const char* path, int want2d, unsigned cap_node, unsigned cap_elem, unsigned* nnode,
                     unsigned* nelem, int* nnoel, double* coord, int* elem) {
  Quiet q;
  if (want2d) {
    Msh::CMesher2D m;
    if (!m.ReadFromFile_GiDMsh(path)) return 1;
    const std::vector<Com::CVector2D>& v = m.GetVectorAry();
    const std::vector<Msh::CTriAry2D>& ta = m.GetTriArySet();
    *nnode = (unsigned)v.size();
    *nnoel = 3;
    *nelem = ta.empty() ? 0u : (unsigned)ta[0].m_aTri.size();
    if (!coord || *nnode > cap_node || *nelem > cap_elem) return 2;
    for (unsigned i = 0; i < *nnode; i++) { coord[2 * i] = v[i].x; coord[2 * i + 1] = v[i].y; }
    for (unsigned e = 0; e < *nelem; e++)
      for (int k = 0; k < 3; k++) elem[3 * e + k] = (int)ta[0].m_aTri[e].v[k];
    return 0;
  }
  Msh::CMesh3D m;
  if (!m.ReadFromFile_GiDMsh(path)) return 1;
  const auto& v = m.GetVectorAry();
  *nnode = (unsigned)v.size();
  const bool hex = !m.GetHexArySet().empty();
  *nnoel = hex ? 8 : 4;
  *nelem = hex ? (unsigned)m.GetHexArySet()[0].m_aHex.size()
               : (m.GetTetArySet().empty() ? 0u : (unsigned)m.GetTetArySet()[0].m_aTet.size());
  if (!coord || *nnode > cap_node || *nelem > cap_elem) return 2;
  for (unsigned i = 0; i < *nnode; i++) { coord[3 * i] = v[i].x; coord[3 * i + 1] = v[i].y; coord[3 * i + 2] = v[i].z; }
  for (unsigned e = 0; e < *nelem; e++)
    for (int k = 0; k < *nnoel; k++)
      elem[(size_t)*nnoel * e + k] =
          hex ? (int)m.GetHexArySet()[0].m_aHex[e].v[k] : (int)m.GetTetArySet()[0].m_aTet[e].v[k];
  return 0;
}


// The boundary facets the reference's GiD readers derive and store: 3-D
// (CMesh3D), the colour-coded triangle arrays; 2-D (CMesher2D), the bar arrays
// (chains of outer bars) and the vertices at their ends.  Facets come out
// grouped, group by group in the readers' order, with each group's array id;
// 2-D vertices with their node and id, and each chain's id_se as indices into
// the vertex list.
int dfm_ref_gid_boundary(const char* path, int want2d, unsigned cap_facet, unsigned cap_group, unsigned cap_vertex,
                         unsigned* nfacet, unsigned* ngroup, unsigned* nvertex, unsigned* facet, unsigned* group_ptr,
                         unsigned* group_id, unsigned* vertex, unsigned* vertex_id, unsigned* group_ends) {
  Quiet q;
  std::vector<unsigned> f, gp(1, 0), gid, vx, vid, ge;
  if (want2d) {
    Msh::CMesher2D m;
    if (!m.ReadFromFile_GiDMsh(path)) return 1;
    for (const Msh::SVertex& v : m.GetVertexAry()) {
      vx.push_back(v.v);
      vid.push_back(v.id);
    }
    for (const Msh::CBarAry& a : m.GetBarArySet()) {
      for (const Msh::SBar& b : a.m_aBar) {
        f.push_back(b.v[0]);
        f.push_back(b.v[1]);
      }
      gp.push_back((unsigned)(f.size() / 2));
      gid.push_back(a.id);
      for (int k = 0; k < 2; k++) {
        unsigned idx = ~0u;
        for (size_t i = 0; i < vid.size(); i++)
          if (vid[i] == a.id_se[k]) idx = (unsigned)i;
        ge.push_back(idx);
      }
    }
  } else {
    Msh::CMesh3D m;
    if (!m.ReadFromFile_GiDMsh(path)) return 1;
    for (const Msh::CTriAry3D& a : m.GetTriArySet()) {
      for (const Msh::STri3D& t : a.m_aTri)
        for (int k = 0; k < 3; k++) f.push_back(t.v[k]);
      gp.push_back((unsigned)(f.size() / 3));
      gid.push_back(a.id);
    }
  }
  *nfacet = gp.back();
  *ngroup = (unsigned)gid.size();
  *nvertex = (unsigned)vx.size();
  if (!facet || *nfacet > cap_facet || *ngroup > cap_group || *nvertex > cap_vertex) return 2;
  std::copy(f.begin(), f.end(), facet);
  std::copy(gp.begin(), gp.end(), group_ptr);
  std::copy(gid.begin(), gid.end(), group_id);
  std::copy(vx.begin(), vx.end(), vertex);
  std::copy(vid.begin(), vid.end(), vertex_id);
  std::copy(ge.begin(), ge.end(), group_ends);
  return 0;
}

// The stored-matrix Newmark systems through the reference's own classes
// (src/femls/linearsystem_fieldsave.cpp:367-880).  Scheme 1:
// CLinearSystem_SaveDiaM_Newmark + AddLinSys_Diffusion (scalar field with
// velocity; p = rho, alpha, source).  Scheme 2: CLinearSystem_SaveDiaM_NewmarkBeta
// + AddLinSys_LinearSolid2D_NonStatic_Save_NewmarkBeta (2-D displacement with
// velocity and acceleration; p = lambda, myu, rho, gx, gy).  P1 triangles;
// the boundary bars fix every DOF of their nodes.
int dfm_ref_newmark(int scheme, int nnode, const double* coord, int nelem, const int* elem, int nbnd,
                    const int* bnd, const double* p, double dt, double gamma, double beta, double* u, double* v,
                    double* a, double* x, double* bdiag, double* boff, double* force, int* flags, double* r,
                    double* norm) {
  if (scheme != 1 && scheme != 2) return 1;
  Quiet q;
  ArrayMesh mesh;
  mesh.ndim = 2;
  mesh.coord.assign(coord, coord + (size_t)nnode * 2);
  mesh.vol.assign(elem, elem + (size_t)nelem * 3);
  mesh.bnd.assign(bnd, bnd + (size_t)nbnd * 2);
  CFieldWorld world;
  const unsigned id_base = world.AddMesh(mesh);
  const CIDConvEAMshCad conv = world.GetIDConverter(id_base);
  const unsigned b = scheme == 1 ? 1 : 2;
  const int fdt = scheme == 1 ? (VALUE | VELOCITY) : (VALUE | VELOCITY | ACCELERATION);
  const unsigned id_field = world.MakeField_FieldElemDim(id_base, 2, scheme == 1 ? SCALAR : VECTOR2, fdt, CORNER);
  const unsigned id_bnd = world.GetPartialField(id_field, conv.GetIdEA_fromMsh(2));
  {  // the field's current state
    CField& f = world.GetField(id_field);
    CNodeAry::CNodeSeg& nu = f.GetNodeSeg(CORNER, true, world, VALUE);
    CNodeAry::CNodeSeg& nv = f.GetNodeSeg(CORNER, true, world, VELOCITY);
    for (int i = 0; i < nnode; i++)
      for (unsigned d = 0; d < b; d++) {
        nu.SetValue(i, d, u[(size_t)i * b + d]);
        nv.SetValue(i, d, v[(size_t)i * b + d]);
      }
    if (scheme == 2) {
      CNodeAry::CNodeSeg& na = f.GetNodeSeg(CORNER, true, world, ACCELERATION);
      for (int i = 0; i < nnode; i++)
        for (unsigned d = 0; d < b; d++) na.SetValue(i, d, a[(size_t)i * b + d]);
    }
  }
  Fem::Ls::CLinearSystem_SaveDiaM_Newmark ls1;
  Fem::Ls::CLinearSystem_SaveDiaM_NewmarkBeta ls2;
  Fem::Ls::CLinearSystem_Save& ls = scheme == 1 ? static_cast<Fem::Ls::CLinearSystem_Save&>(ls1)
                                                : static_cast<Fem::Ls::CLinearSystem_Save&>(ls2);
  ls.AddPattern_Field(id_field, world);
  ls.SetFixedBoundaryCondition_Field(id_bnd, world);
  if (scheme == 1) ls1.SetNewmarkParameter(gamma, dt);
  else ls2.SetNewmarkParameter(beta, gamma, dt);
  ls.InitializeMarge();
  if (scheme == 1) Fem::Eqn::AddLinSys_Diffusion(ls1, p[0], p[1], p[2], world, id_field);
  else Fem::Eqn::AddLinSys_LinearSolid2D_NonStatic_Save_NewmarkBeta(ls2, p[0], p[1], p[2], p[3], p[4], world, id_field);
  ls.FinalizeMarge();
  const unsigned bb = b * b;
  {  // the stored matrix in the library's layout: diagonal block apart, the rest in column order
    MatVec::CMat_BlkCrs& B = ls.GetMatrix_Boundary(id_field, CORNER, id_field, CORNER, world);
    size_t pos = 0;
    for (int i = 0; i < nnode; i++) {
      unsigned np = 0;
      const unsigned* ind = B.GetPtrIndPSuP(i, np);
      unsigned nv = 0;
      const double* val = B.GetPtrValPSuP(i, nv);
      for (unsigned k = 0; k < np; k++) {
        double* dst = (ind[k] == (unsigned)i) ? bdiag + (size_t)i * bb : boff + (pos++) * bb;
        std::memcpy(dst, val + (size_t)k * bb, sizeof(double) * bb);
      }
    }
    MatVec::CVector_Blk& F = ls.GetForce(id_field, CORNER, world);
    MatVec::CBCFlag& bc = ls.m_ls.GetBCFlag(0);
    for (int i = 0; i < nnode; i++)
      for (unsigned d = 0; d < b; d++) {
        force[(size_t)i * b + d] = F.GetValue(i, d);
        flags[(size_t)i * b + d] = bc.GetBCFlag(i, d);
      }
  }
  *norm = ls.MakeResidual(world);
  {
    MatVec::CVector_Blk& R = ls.m_ls.GetVector(-1, 0);
    MatVec::CVector_Blk& U = ls.m_ls.GetVector(-2, 0);
    for (int i = 0; i < nnode; i++)
      for (unsigned d = 0; d < b; d++) {
        r[(size_t)i * b + d] = R.GetValue(i, d);
        U.SetValue(i, d, x[(size_t)i * b + d]);  // the solved update
      }
  }
  ls.UpdateValueOfField(id_field, world, scheme == 1 ? VELOCITY : ACCELERATION);
  {
    CField& f = world.GetField(id_field);
    CNodeAry::CNodeSeg& nu = f.GetNodeSeg(CORNER, true, world, VALUE);
    CNodeAry::CNodeSeg& nv = f.GetNodeSeg(CORNER, true, world, VELOCITY);
    MatVec::CVector_Blk& U = ls.m_ls.GetVector(-2, 0);
    std::vector<double> t(b);
    for (int i = 0; i < nnode; i++) {
      nu.GetValue(i, t.data());
      for (unsigned d = 0; d < b; d++) u[(size_t)i * b + d] = t[d];
      nv.GetValue(i, t.data());
      for (unsigned d = 0; d < b; d++) v[(size_t)i * b + d] = t[d];
      for (unsigned d = 0; d < b; d++) x[(size_t)i * b + d] = U.GetValue(i, d);
    }
    if (scheme == 2) {
      CNodeAry::CNodeSeg& na = f.GetNodeSeg(CORNER, true, world, ACCELERATION);
      for (int i = 0; i < nnode; i++) {
        na.GetValue(i, t.data());
        for (unsigned d = 0; d < b; d++) a[(size_t)i * b + d] = t[d];
      }
    }
  }
  return 0;
}


// CZMatDiaFrac_BlkCrs(lev, A) + SetValue_Initialize + DoILUDecomp
// (src/matvec/zmatdiafrac_blkcrs.cpp:77-107, :263-441): the complex ILU(k)
// pattern and factor, as dfm_ref_mat_iluk for real matrices.
int dfm_ref_zmat_iluk(unsigned N, const unsigned* rowptr, const unsigned* colind, const double* diag,
                      const double* off, int lev, unsigned cap, unsigned* frowptr, unsigned* fcolind, double* fdiag,
                      double* foff, unsigned* fncrs) {
  Quiet q;
  MatVec::CZMatDia_BlkCrs* m = make_zmat(N, rowptr, colind, diag, off);
  MatVec::CZMatDiaFrac_BlkCrs f(lev, *m);
  *fncrs = f.NCrs();
  if (!frowptr || f.NCrs() > cap) {
    delete m;
    return 2;
  }
  frowptr[0] = 0;
  for (unsigned i = 0; i < N; i++) {
    unsigned n = 0;
    const unsigned* c = f.GetPtrIndPSuP(i, n);
    if (n) std::memcpy(fcolind + frowptr[i], c, sizeof(unsigned) * n);
    frowptr[i + 1] = frowptr[i] + n;
  }
  f.SetValue_Initialize(*m);
  f.DoILUDecomp();
  read_zmat(f, fdiag, foff);
  delete m;
  return 0;
}

// The field-level system's preconditioner at fill level lev
// (CPreconditioner_ILU / CZPreconditioner_ILU SetFillInLevel + SetLinearSystem);
// the next dfm_ref_ilu factors it.
int dfm_ref_set_fill(dfm_ref_sys* s, int lev) {
  Quiet q;
  if (s->complex_kind()) {
    s->zprec.SetFillInLevel((unsigned)lev);
    s->zprec.SetLinearSystem(s->zls);
  } else {
    s->prec.Clear();
    s->prec.SetFillInLevel(lev);
    s->prec.SetLinearSystem(s->ls.m_ls);
  }
  return 0;
}


// CMat_BlkCrs(nrow, brow, ncol, bcol) with the given pattern and values, then
// MatVec(alpha, x, beta, y) (src/matvec/mat_blkcrs.cpp:955-1175).
int dfm_ref_rmat_spmv(unsigned nrow, unsigned ncol, unsigned brow, unsigned bcol, const unsigned* rowptr,
                      const unsigned* colind, const double* val, double alpha, const double* x, double beta,
                      double* y) {
  Quiet q;
  MatVec::CMat_BlkCrs m(nrow, brow, ncol, bcol);
  Com::CIndexedArray crs;
  crs.index.assign(rowptr, rowptr + nrow + 1);
  crs.array.assign(colind, colind + rowptr[nrow]);
  m.AddPattern(crs);
  m.SetZero();
  const unsigned bb = brow * bcol;
  for (unsigned i = 0; i < nrow; i++) {
    unsigned np = 0;
    double* p = m.GetPtrValPSuP(i, np);
    if (np) std::memcpy(p, val + (size_t)rowptr[i] * bb, sizeof(double) * bb * np);
  }
  MatVec::CVector_Blk vx(ncol, bcol), vy(nrow, brow);
  for (unsigned j = 0; j < ncol; j++)
    for (unsigned c = 0; c < bcol; c++) vx.SetValue(j, c, x[(size_t)j * bcol + c]);
  for (unsigned i = 0; i < nrow; i++)
    for (unsigned r = 0; r < brow; r++) vy.SetValue(i, r, y[(size_t)i * brow + r]);
  m.MatVec(alpha, vx, beta, vy, true);
  for (unsigned i = 0; i < nrow; i++)
    for (unsigned r = 0; r < brow; r++) y[(size_t)i * brow + r] = vy.GetValue(i, r);
  return 0;
}

}  // extern "C"
