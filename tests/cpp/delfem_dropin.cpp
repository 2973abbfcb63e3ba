// A DelFEM program that switches its linear solve to the B200 library through
// include/dfm_b200_delfem.hpp.  Test infrastructure: it is compiled against
// DelFEM's own headers and linked with the reference library built from its
// sources (oracle/Makefile, target `dropin`), so the field world, the pattern,
// the element assembly (Fem::Eqn::AddLinSys_*), the Dirichlet elimination
// (FinalizeMarge) and UpdateValueOfField are the reference's code; only the
// preconditioner and the solver change.
//
//   delfem_dropin poisson N     2-D Poisson -lap u = 1 on an N x N grid of P1 triangles, u = 0 on the boundary
//   delfem_dropin solid3d NX NY NZ   3-D linear elasticity of a box (Kuhn tetrahedra), x = 0 face clamped,
//                                    unit body force in -z
//   delfem_dropin twoseg N M L0 L1 [lev]   a linear system of two segments built at the matrix level
//                                    (LsSol::CLinearSystem::AddLinSysSeg / AddMat_Dia / AddMat_NonDia):
//                                    an N x N grid of L0 x L0 blocks and a chain of M nodes of L1 x L1
//                                    blocks, coupled both ways; symmetric positive definite
//   [lev]                       optional: ILU fill-in level (SetFillInLevel), default 0
//   [rev|rand]                  optional trailing argument: a block ordering (CPreconditioner_ILU::SetOrdering),
//                               the rows reversed or shuffled (one-segment problems)
//   [fill]                      optional trailing argument: CPreconditioner_ILU::SetFillBlk with every 9th
//                               block row of the first segment's middle fifth (unlimited fill through them)
//
// Every run builds the problem from scratch, solves, calls the reference's
// UpdateValueOfField and reads the field back (the segments' update vectors
// for twoseg).  Runs:
//   ref_pcg, ref_bicg, ref_cg  the reference's LsSol solvers with LsSol::CPreconditioner_ILU
//   gpu_pcg, gpu_bicg, gpu_cg  dfm_delfem::Solve_*_GPU over dfm_delfem::CLinearSystemGPU
//   ref_over_gpu               the reference's LsSol::Solve_PCG driving CLinearSystemGPU step by step
//   glue_gpu_prec              the reference's CLinearSystemPreconditioner glue with
//                              dfm_delfem::CPreconditioner_ILU_GPU as its LsSol::CPreconditioner
// and prints one JSON object: per run ok, iterations, conv and the field values.
#include <algorithm>
#include <cmath>
#include <random>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <utility>
#include <iostream>
#include <memory>
#include <streambuf>
#include <string>
#include <vector>

#include "delfem/field.h"
#include "delfem/field_world.h"
#include "delfem/femeqn/eqn_linear_solid3d.h"
#include "delfem/femeqn/eqn_poisson.h"
#include "delfem/femls/linearsystem_field.h"
#include "delfem/ls/linearsystem.h"
#include "delfem/ls/preconditioner.h"
#include "delfem/ls/solver_ls_iter.h"
#include "delfem/matvec/mat_blkcrs.h"
#include "delfem/matvec/matdia_blkcrs.h"
#include "delfem/matvec/vector_blk.h"
#include "delfem/mesh_interface.h"
#include "dfm_b200_delfem.hpp"

using namespace Fem::Field;

namespace {

// the reference prints progress text on std::cout; the JSON goes to stdout by printf
struct Quiet {
  struct Null : std::streambuf {
    int overflow(int c) override { return c; }
  } nb;
  std::streambuf* old;
  Quiet() : old(std::cout.rdbuf(&nb)) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

// A structured mesh through the reference's mesh interface: id 1 the volume
// elements, id 2 the Dirichlet boundary (included in id 1).
class GridMesh : public Msh::IMesh {
 public:
  unsigned ndim = 2;
  std::vector<double> coord;
  Msh::MSH_TYPE vol_type = Msh::TRI, bnd_type = Msh::BAR;
  std::vector<int> vol, bnd;
  unsigned int GetDimention() const override { return ndim; }
  void GetInfo(unsigned int id_msh, unsigned int& id_cad_part, unsigned int& id_msh_before_ext, unsigned int& inum_ext,
               int& ilayer) const override {
    id_cad_part = id_msh;
    id_msh_before_ext = 0;
    inum_ext = 0;
    ilayer = 0;
  }
  void GetCoord(std::vector<double>& c) const override { c = coord; }
  Msh::MSH_TYPE GetConnectivity(unsigned int id_msh, std::vector<int>& lnods) const override {
    if (id_msh == 1) {
      lnods = vol;
      return vol_type;
    }
    lnods = bnd;
    return bnd_type;
  }
  std::vector<unsigned int> GetAry_ID() const override { return {1u, 2u}; }
  std::vector<unsigned int> GetIncludeElemIDAry(unsigned int id_msh) const override {
    return id_msh == 1 ? std::vector<unsigned int>{2u} : std::vector<unsigned int>{};
  }
};

GridMesh poisson_mesh(int n) {
  GridMesh m;
  const int s = n + 1;
  for (int j = 0; j < s; j++)
    for (int i = 0; i < s; i++) {
      m.coord.push_back((double)i / n);
      m.coord.push_back((double)j / n);
    }
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      const int p = i + j * s;
      const int t[6] = {p, p + 1, p + s + 1, p, p + s + 1, p + s};
      m.vol.insert(m.vol.end(), t, t + 6);
    }
  for (int i = 0; i < n; i++) {  // the four sides as bars
    const int e[8] = {i, i + 1, n * s + i, n * s + i + 1, i * s, (i + 1) * s, i * s + n, (i + 1) * s + n};
    m.bnd.insert(m.bnd.end(), e, e + 8);
  }
  return m;
}

// n = (nx+1)(ny+1)(nz+1) nodes, x fastest; each hex split into 6 tetrahedra
// around its v0-v6 diagonal; the x = 0 face as triangles
GridMesh solid_mesh(int nx, int ny, int nz) {
  GridMesh m;
  m.ndim = 3;
  m.vol_type = Msh::TET;
  m.bnd_type = Msh::TRI;
  const double lx = 1.0, ly = 0.2, lz = 0.2;
  auto id = [&](int i, int j, int k) { return i + (nx + 1) * (j + (ny + 1) * k); };
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        m.coord.push_back(lx * i / nx);
        m.coord.push_back(ly * j / ny);
        m.coord.push_back(lz * k / nz);
      }
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const int v[8] = {id(i, j, k),         id(i + 1, j, k),         id(i + 1, j + 1, k),     id(i, j + 1, k),
                          id(i, j, k + 1),     id(i + 1, j, k + 1),     id(i + 1, j + 1, k + 1), id(i, j + 1, k + 1)};
        const int tets[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
        for (auto& t : tets) {
          int e[4] = {v[t[0]], v[t[1]], v[t[2]], v[t[3]]};
          const double* c0 = &m.coord[3 * e[0]];
          double a[3][3];
          for (int q = 0; q < 3; q++)
            for (int d = 0; d < 3; d++) a[q][d] = m.coord[3 * e[q + 1] + d] - c0[d];
          const double vol = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                             a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                             a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
          if (vol < 0) std::swap(e[1], e[2]);  // positively oriented
          m.vol.insert(m.vol.end(), e, e + 4);
        }
      }
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      const int a = id(0, j, k), b = id(0, j + 1, k), c = id(0, j + 1, k + 1), d = id(0, j, k + 1);
      const int t[6] = {a, b, c, a, c, d};
      m.bnd.insert(m.bnd.end(), t, t + 6);
    }
  return m;
}

// One fresh linear system to solve: the solver-side CLinearSystem, its
// assembly, and the solution after the solve.
struct Sys {
  virtual ~Sys() {}
  virtual LsSol::CLinearSystem& lin() = 0;
  virtual void assemble() = 0;
  virtual std::vector<double> result() = 0;
};

// One fresh DelFEM problem: field world, field, boundary, linear system.
struct Problem : Sys {
  std::string kind;
  GridMesh mesh;
  CFieldWorld world;
  unsigned id_field = 0, id_bnd = 0;
  Fem::Ls::CLinearSystem_Field ls;

  Problem(const std::string& k, const GridMesh& m) : kind(k), mesh(m) {
    Quiet q;
    const unsigned id_base = world.AddMesh(mesh);
    const CIDConvEAMshCad conv = world.GetIDConverter(id_base);
    id_field = world.MakeField_FieldElemDim(id_base, mesh.ndim, kind == "poisson" ? SCALAR : VECTOR3, VALUE, CORNER);
    id_bnd = world.GetPartialField(id_field, conv.GetIdEA_fromMsh(2));
    ls.AddPattern_Field(id_field, world);
    ls.SetFixedBoundaryCondition_Field(id_bnd, world);
  }
  void assemble() override {
    Quiet q;
    ls.InitializeMarge();
    if (kind == "poisson") {
      Fem::Eqn::AddLinSys_Poisson(ls, 1.0, 1.0, world, id_field);
    } else {
      const double nu = 0.3, lam = nu / ((1 + nu) * (1 - 2 * nu)), myu = 1.0 / (2 * (1 + nu));
      Fem::Eqn::AddLinSys_LinearSolid3D_Static(ls, lam, myu, 1.0, 0.0, 0.0, -1.0, world, id_field);
    }
    ls.FinalizeMarge();
  }
  LsSol::CLinearSystem& lin() override { return ls.m_ls; }
  std::vector<double> result() override {
    {
      Quiet q;
      ls.UpdateValueOfField(id_field, world, VALUE);
    }
    return field();
  }
  std::vector<double> field() const {
    const CField& f = world.GetField(id_field);
    const CNodeAry::CNodeSeg& ns = f.GetNodeSeg(CORNER, true, world, VALUE);
    const unsigned len = ns.Length();
    std::vector<double> out((size_t)ns.Size() * len);
    for (unsigned i = 0; i < ns.Size(); i++) ns.GetValue(i, &out[(size_t)i * len]);
    return out;
  }
};

// Two segments at the matrix level: segment 0 an n x n grid (4 neighbours) of
// L0 x L0 blocks, segment 1 a chain of m nodes of L1 x L1 blocks, node k of the
// chain coupled to two grid nodes; couplings C (rows in segment 1) and C^T.
struct TwoSeg : Sys {
  unsigned n, m, L0, L1, N0;
  LsSol::CLinearSystem ls;
  std::vector<std::vector<unsigned>> grid, chain, cpl, cplT;

  TwoSeg(unsigned n_, unsigned m_, unsigned l0, unsigned l1) : n(n_), m(m_), L0(l0), L1(l1), N0(n_ * n_) {
    grid.resize(N0);
    for (unsigned j = 0; j < n; j++)
      for (unsigned i = 0; i < n; i++) {
        auto& g = grid[i + j * n];
        if (j > 0) g.push_back(i + (j - 1) * n);
        if (i > 0) g.push_back(i - 1 + j * n);
        if (i + 1 < n) g.push_back(i + 1 + j * n);
        if (j + 1 < n) g.push_back(i + (j + 1) * n);
      }
    chain.resize(m);
    cpl.resize(m);
    cplT.resize(N0);
    for (unsigned k = 0; k < m; k++) {
      if (k > 0) chain[k].push_back(k - 1);
      if (k + 1 < m) chain[k].push_back(k + 1);
      unsigned a = (3 * k) % N0, b = (7 * k + 1) % N0;
      if (a > b) std::swap(a, b);
      cpl[k].push_back(a);
      if (b != a) cpl[k].push_back(b);
      for (unsigned c : cpl[k]) cplT[c].push_back(k);
    }
    Quiet q;
    ls.AddLinSysSeg(N0, L0);
    ls.AddLinSysSeg(m, L1);
    ls.AddMat_Dia(0, crs(grid));
    ls.AddMat_Dia(1, crs(chain));
    ls.AddMat_NonDia(1, 0, crs(cpl));
    ls.AddMat_NonDia(0, 1, crs(cplT));
  }
  static Com::CIndexedArray crs(const std::vector<std::vector<unsigned>>& rows) {
    Com::CIndexedArray a;
    a.index.assign(1, 0);
    for (const auto& r : rows) {
      a.array.insert(a.array.end(), r.begin(), r.end());
      a.index.push_back((unsigned)a.array.size());
    }
    return a;
  }
  // symmetric coupling block values: entry (r, c) of C's block (k, g)
  static double cval(unsigned k, unsigned g, unsigned r, unsigned c) { return -0.1 - 0.01 * ((k + 2 * g + r + 3 * c) % 5); }
  LsSol::CLinearSystem& lin() override { return ls; }
  void assemble() override {
    Quiet q;
    ls.InitializeMarge();
    MatVec::CMatDia_BlkCrs& A0 = ls.GetMatrix(0);
    MatVec::CMatDia_BlkCrs& A1 = ls.GetMatrix(1);
    for (unsigned p = 0; p < N0; p++) {
      double* d = A0.GetPtrValDia(p);
      for (unsigned r = 0; r < L0; r++)
        for (unsigned c = 0; c < L0; c++) d[r * L0 + c] = (r == c ? 4.0 + 0.5 * L0 : 0.0) + 0.1;
      unsigned np = 0;
      double* o = A0.GetPtrValPSuP(p, np);
      for (unsigned t = 0; t < np * L0 * L0; t++) o[t] = ((t % (L0 * L0)) % (L0 + 1) == 0 ? -1.0 : 0.0) - 0.05;
    }
    for (unsigned k = 0; k < m; k++) {
      double* d = A1.GetPtrValDia(k);
      for (unsigned r = 0; r < L1; r++)
        for (unsigned c = 0; c < L1; c++) d[r * L1 + c] = (r == c ? 2.2 + 0.4 * L0 + 0.2 * L1 : 0.0) + 0.1;
      unsigned np = 0;
      double* o = A1.GetPtrValPSuP(k, np);
      for (unsigned t = 0; t < np * L1 * L1; t++) o[t] = ((t % (L1 * L1)) % (L1 + 1) == 0 ? -1.0 : 0.0) - 0.05;
    }
    {  // C: rows in the chain, columns in the grid; C^T: the transpose, block by block
      MatVec::CMat_BlkCrs& C = ls.GetMatrix(1, 0);
      MatVec::CMat_BlkCrs& CT = ls.GetMatrix(0, 1);
      for (unsigned k = 0; k < m; k++) {
        unsigned np = 0;
        double* o = C.GetPtrValPSuP(k, np);
        for (unsigned t = 0; t < np; t++)
          for (unsigned r = 0; r < L1; r++)
            for (unsigned c = 0; c < L0; c++) o[(t * L1 + r) * L0 + c] = cval(k, cpl[k][t], r, c);
      }
      for (unsigned g = 0; g < N0; g++) {
        unsigned np = 0;
        double* o = CT.GetPtrValPSuP(g, np);
        for (unsigned t = 0; t < np; t++)
          for (unsigned r = 0; r < L0; r++)
            for (unsigned c = 0; c < L1; c++) o[(t * L0 + r) * L1 + c] = cval(cplT[g][t], g, c, r);
      }
    }
    for (unsigned s = 0; s < 2; s++) {
      MatVec::CVector_Blk& f = ls.GetVector(-1, s);
      const unsigned L = s ? L1 : L0;
      for (unsigned i = 0; i < f.NBlk(); i++)
        for (unsigned d = 0; d < L; d++) f.SetValue(i, d, std::sin(0.37 * i + 1.3 * d + 0.5 * s) + 0.2);
    }
    ls.FinalizeMarge();
  }
  std::vector<double> result() override {
    std::vector<double> x;
    for (unsigned s = 0; s < 2; s++) {
      const MatVec::CVector_Blk& u = ls.GetVector(-2, s);
      const unsigned L = s ? L1 : L0;
      for (unsigned i = 0; i < u.NBlk(); i++)
        for (unsigned d = 0; d < L; d++) x.push_back(u.GetValue(i, d));
    }
    return x;
  }
};

struct Run {
  std::string name;
  bool ok = false;
  unsigned it = 0;
  double conv = 0.0;
  std::vector<double> x;
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s poisson N [lev] | solid3d NX NY NZ [lev] | twoseg N M L0 L1 [lev]\n", argv[0]);
    return 2;
  }
  std::string ordk;      // block ordering for SetOrdering
  bool fillblk = false;  // SetFillBlk
  while (argc > 3) {
    const std::string a = argv[argc - 1];
    if (a == "rev" || a == "rand") ordk = a;
    else if (a == "fill") fillblk = true;
    else break;
    argc--;
  }
  const std::string kind = argv[1];
  GridMesh mesh;
  int lev = 0;
  std::function<std::unique_ptr<Sys>()> make;
  if (kind == "poisson") {
    mesh = poisson_mesh(std::atoi(argv[2]));
    if (argc > 3) lev = std::atoi(argv[3]);
    make = [&]() { return std::unique_ptr<Sys>(new Problem(kind, mesh)); };
  } else if (kind == "solid3d" && argc >= 5) {
    mesh = solid_mesh(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]));
    if (argc > 5) lev = std::atoi(argv[5]);
    make = [&]() { return std::unique_ptr<Sys>(new Problem(kind, mesh)); };
  } else if (kind == "twoseg" && argc >= 6) {
    const unsigned n = std::atoi(argv[2]), m = std::atoi(argv[3]), l0 = std::atoi(argv[4]), l1 = std::atoi(argv[5]);
    if (argc > 6) lev = std::atoi(argv[6]);
    make = [=]() { return std::unique_ptr<Sys>(new TwoSeg(n, m, l0, l1)); };
  } else {
    return 2;
  }
  const double tol = 1e-10;
  const unsigned maxit = 5000;
  // aind[new] = old: the rows reversed, or shuffled with a fixed seed
  auto ordering = [&](Sys& P) {
    std::vector<int> a;
    if (ordk.empty()) return a;
    const unsigned n = P.lin().GetMatrix(0).NBlkMatCol();
    for (unsigned i = 0; i < n; i++) a.push_back(ordk == "rev" ? (int)(n - 1 - i) : (int)i);
    if (ordk == "rand") std::shuffle(a.begin(), a.end(), std::mt19937(7));
    return a;
  };
  // SetFillBlk list: every 9th block row of the first segment's middle fifth
  auto fill_rows = [&](Sys& P) {
    std::vector<unsigned int> a;
    if (!fillblk) return a;
    const unsigned n = P.lin().GetMatrix(0).NBlkMatCol();
    for (unsigned i = 2 * n / 5; i < 3 * n / 5; i += 9) a.push_back(i);
    return a;
  };
  std::vector<Run> runs;
  try {
    dfm_lsol::Context ctx(0);
    // the reference's path: LsSol::CPreconditioner_ILU + LsSol solvers
    auto ref_run = [&](const char* name, int method) {
      std::unique_ptr<Sys> P = make();
      Run r;
      r.name = name;
      r.conv = tol;
      r.it = maxit;
      Quiet q;
      LsSol::CPreconditioner_ILU prec;
      if (lev) prec.SetFillInLevel(lev);
      prec.SetOrdering(ordering(*P));
      prec.SetFillBlk(fill_rows(*P));
      prec.SetLinearSystem(P->lin());
      P->assemble();
      prec.SetValue(P->lin());
      LsSol::CLinearSystemPreconditioner lsp(P->lin(), prec);
      if (method == 0) r.ok = LsSol::Solve_PCG(r.conv, r.it, lsp);
      else if (method == 1) r.ok = LsSol::Solve_PBiCGSTAB(r.conv, r.it, lsp);
      else r.ok = LsSol::Solve_CG(r.conv, r.it, P->lin());
      r.x = P->result();
      runs.push_back(r);
    };
    // the drop-in: only the preconditioner, the interface object and the solver change
    auto gpu_run = [&](const char* name, int method) {
      std::unique_ptr<Sys> P = make();
      Run r;
      r.name = name;
      r.conv = tol;
      r.it = maxit;
      dfm_delfem::CPreconditioner_ILU_GPU prec(ctx);
      prec.SetFillInLevel(lev);
      prec.SetOrdering(ordering(*P));
      prec.SetFillBlk(fill_rows(*P));
      prec.SetLinearSystem(P->lin());
      P->assemble();
      if (!prec.SetValue(P->lin())) throw dfm_lsol::Error(DFM_SINGULAR_PIVOT, name);
      {
        dfm_delfem::CLinearSystemGPU lsp(P->lin(), prec);
        if (method == 0) r.ok = dfm_delfem::Solve_PCG_GPU(r.conv, r.it, lsp);
        else if (method == 1) r.ok = dfm_delfem::Solve_PBiCGSTAB_GPU(r.conv, r.it, lsp);
        else if (method == 2) r.ok = dfm_delfem::Solve_CG_GPU(r.conv, r.it, lsp);
        else {  // the reference's own solver, one device operation per step
          Quiet q;
          r.ok = LsSol::Solve_PCG(r.conv, r.it, lsp);
          lsp.SyncToHost();
        }
      }
      r.x = P->result();
      runs.push_back(r);
    };
    ref_run("ref_pcg", 0);
    ref_run("ref_bicg", 1);
    ref_run("ref_cg", 2);
    gpu_run("gpu_pcg", 0);
    gpu_run("gpu_bicg", 1);
    gpu_run("gpu_cg", 2);
    gpu_run("ref_over_gpu", 3);
    {  // the reference's glue class with the device preconditioner as its LsSol::CPreconditioner
      std::unique_ptr<Sys> P = make();
      Run r;
      r.name = "glue_gpu_prec";
      r.conv = tol;
      r.it = maxit;
      dfm_delfem::CPreconditioner_ILU_GPU prec(ctx);
      prec.SetFillInLevel(lev);
      prec.SetOrdering(ordering(*P));
      prec.SetFillBlk(fill_rows(*P));
      LsSol::CPreconditioner& base = prec;
      base.SetLinearSystem(P->lin());
      P->assemble();
      base.SetValue(P->lin());
      LsSol::CLinearSystemPreconditioner lsp(P->lin(), base);
      {
        Quiet q;
        r.ok = LsSol::Solve_PCG(r.conv, r.it, lsp);
      }
      r.x = P->result();
      runs.push_back(r);
    }
  } catch (const dfm_lsol::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  std::printf("{");
  for (size_t k = 0; k < runs.size(); k++) {
    const Run& r = runs[k];
    std::printf("%s\"%s\": {\"ok\": %s, \"iters\": %u, \"conv\": %.17g, \"x\": [", k ? ", " : "", r.name.c_str(),
                r.ok ? "true" : "false", r.it, r.conv);
    for (size_t i = 0; i < r.x.size(); i++) std::printf("%s%.17g", i ? ", " : "", r.x[i]);
    std::printf("]}");
  }
  std::printf("}\n");
  return 0;
}
