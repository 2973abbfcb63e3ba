// dfm_b200_delfem.hpp - the B200 solve path behind DelFEM's own solver
// interfaces.  Header-only; compile with DelFEM's include directory on the
// path (it includes the reference's headers) and link libdfm_b200.so.
//
// What replaces what (a DelFEM program changes these names only):
//
//   LsSol::CPreconditioner_ILU       -> dfm_delfem::CPreconditioner_ILU_GPU
//       a LsSol::CPreconditioner (include/delfem/ls/preconditioner.h:46-53):
//       SetLinearSystem (pattern + ILU(k) symbolic, level sets),
//       SetValue (values + numeric ILU on the device), SolvePrecond;
//       SetFillInLevel as in include/delfem/ls/preconditioner.h:72.
//   LsSol::CLinearSystemPreconditioner -> dfm_delfem::CLinearSystemGPU
//       a LsSol::ILinearSystemPreconditioner_Sol and LsSol::ILinearSystem_Sol
//       (include/delfem/ls/linearsystem_interface_solver.h:39-82) over the
//       CLinearSystem's matrix and vectors mirrored on the device: handles
//       -1 (residual) and -2 (update) plus the solver's temporaries.
//   LsSol::Solve_PCG / Solve_PBiCGSTAB / Solve_CG
//                                    -> dfm_delfem::Solve_PCG_GPU /
//                                       Solve_PBiCGSTAB_GPU / Solve_CG_GPU
//       same signature and in/out conventions (include/delfem/ls/
//       solver_ls_iter.h:35-45): the whole iteration runs on the device
//       (captured CUDA graphs, scalars on the device), then -1 and -2 are
//       written back into the CLinearSystem, so the reference's own
//       CLinearSystem_Field::UpdateValueOfField (src/femls/
//       linearsystem_field.cpp:715-793) reads the solution unchanged.
//
// The usual sequence of a DelFEM equation system (src/femeqn/eqnsys_scalar.cpp:
// 213-359) then reads
//
//   dfm_lsol::Context ctx(0);
//   dfm_delfem::CPreconditioner_ILU_GPU prec(ctx);
//   prec.SetLinearSystem(ls.m_ls);          // after AddPattern_Field / BCs
//   ls.InitializeMarge(); ...AddLinSys_*...; ls.FinalizeMarge();
//   prec.SetValue(ls.m_ls);
//   dfm_delfem::CLinearSystemGPU lsp(ls.m_ls, prec);
//   double conv = 1e-10; unsigned it = 1000;
//   dfm_delfem::Solve_PCG_GPU(conv, it, lsp);
//   ls.UpdateValueOfField(id_field, world, Fem::Field::VALUE);
//
// CLinearSystemGPU is also a complete implementation of the reference's
// interface, so the reference's own LsSol::Solve_PCG(conv, it, lsp) runs on
// it too, one device operation per step; call SyncToHost() (or let lsp go out
// of scope) before reading -1 / -2 on the host after such a solve.
//
// Scope: one linear-system segment with fixed b x b blocks, b in {1, 2, 3}
// (the CMatDia_BlkCrs of a single field).  Errors other than the reference's
// boolean results throw dfm_lsol::Error.
#ifndef DFM_B200_DELFEM_HPP
#define DFM_B200_DELFEM_HPP

#include <memory>
#include <vector>

#include "delfem/ls/linearsystem.h"
#include "delfem/ls/linearsystem_interface_solver.h"
#include "delfem/ls/preconditioner.h"
#include "delfem/matvec/matdia_blkcrs.h"
#include "delfem/matvec/vector_blk.h"
#include "dfm_b200.h"
#include "dfm_b200_lsol.hpp"

namespace dfm_delfem {

using dfm_lsol::check;
using dfm_lsol::Context;
using dfm_lsol::DeviceVector;
using dfm_lsol::Error;

namespace detail {
// The single segment's matrix as the device library takes it.
inline const MatVec::CMatDia_BlkCrs& segment_matrix(const LsSol::CLinearSystem& ls) {
  if (ls.GetNLinSysSeg() != 1 || !ls.IsMatrix(0, 0)) throw Error(DFM_ERR_UNSUPPORTED, "one segment expected");
  const MatVec::CMatDia_BlkCrs& m = ls.GetMatrix(0);
  if (m.LenBlkCol() < 1 || m.LenBlkCol() > 3) throw Error(DFM_ERR_UNSUPPORTED, "block size");
  return m;
}
// Contiguous values of a fixed-length CVector_Blk.
inline double* values(MatVec::CVector_Blk& v) { return v.NBlk() ? v.GetValuePtr(0) : nullptr; }
inline const double* values(const MatVec::CVector_Blk& v) { return v.NBlk() ? v.GetValuePtr(0) : nullptr; }
}  // namespace detail

// LsSol::CPreconditioner_ILU on the device: ILU(0), or ILU(k) after
// SetFillInLevel(k), in the natural ordering.  It also owns the device copy of
// the system matrix, which CLinearSystemGPU multiplies with.
class CPreconditioner_ILU_GPU : public LsSol::CPreconditioner {
 public:
  explicit CPreconditioner_ILU_GPU(Context& ctx) : ctx_(&ctx) {}
  CPreconditioner_ILU_GPU(Context& ctx, const LsSol::CLinearSystem& ls, unsigned int nlev = 0) : ctx_(&ctx) {
    SetFillInLevel((int)nlev);
    SetLinearSystem(ls);
  }
  ~CPreconditioner_ILU_GPU() override { Clear(); }
  CPreconditioner_ILU_GPU(const CPreconditioner_ILU_GPU&) = delete;
  CPreconditioner_ILU_GPU& operator=(const CPreconditioner_ILU_GPU&) = delete;

  void Clear() {
    if (ilu_) dfm_ilu_destroy(ilu_);
    if (mat_) dfm_mat_destroy(mat_);
    ilu_ = nullptr;
    mat_ = nullptr;
    tmp_r_.reset();
    tmp_z_.reset();
  }
  // the fill-in level of the next SetLinearSystem (-1: no limit); one
  // segment, so ilss0 must be -1 or 0
  void SetFillInLevel(int lev, int ilss0 = -1) {
    if (ilss0 != -1 && ilss0 != 0) throw Error(DFM_ERR_UNSUPPORTED, "SetFillInLevel");
    if (lev < -1) throw Error(DFM_ERR_INVALID, "SetFillInLevel");
    lev_ = lev;
  }
  // pattern of the system matrix on the device, fill pattern and level sets
  void SetLinearSystem(const LsSol::CLinearSystem& ls) override {
    Clear();
    const MatVec::CMatDia_BlkCrs& m = detail::segment_matrix(ls);
    nblk_ = m.NBlkMatCol();
    len_ = (unsigned)m.LenBlkCol();
    std::vector<unsigned> rp(nblk_ + 1, 0), ci;
    ci.reserve(m.NCrs());
    for (unsigned i = 0; i < nblk_; i++) {
      unsigned np = 0;
      const unsigned* p = m.GetPtrIndPSuP(i, np);
      rp[i + 1] = rp[i] + np;
      ci.insert(ci.end(), p, p + np);
    }
    check(dfm_mat_create(ctx_->get(), nblk_, len_, DFM_REAL, rp.data(), ci.data(), &mat_), "SetLinearSystem");
    check(dfm_ilu_create_fill(mat_, lev_, &ilu_), "SetLinearSystem");
  }
  // the system's current values to the device and the numeric factorisation;
  // false when more than 10 pivots were singular (the reference's result)
  bool SetValue(const LsSol::CLinearSystem& ls) override {
    if (!mat_) throw Error(DFM_ERR_INVALID, "SetValue before SetLinearSystem");
    const MatVec::CMatDia_BlkCrs& m = detail::segment_matrix(ls);
    if (m.NBlkMatCol() != nblk_ || (unsigned)m.LenBlkCol() != len_) throw Error(DFM_ERR_INVALID, "SetValue");
    unsigned np = 0;
    const double* off = m.NCrs() ? m.GetPtrValPSuP(0, np) : nullptr;  // row-ordered, contiguous
    const double* dia = nblk_ ? m.GetPtrValDia(0) : nullptr;
    check(dfm_mat_set_values(mat_, dia, off, DFM_HOST), "SetValue");
    unsigned ns = 0;
    return check(dfm_ilu_factor(ilu_, mat_, &ns), "SetValue", DFM_SINGULAR_PIVOT) == DFM_OK;
  }
  // {iv} := (LU)^-1 {iv} on the CLinearSystem's host vector (copied to the
  // device and back); solvers over CLinearSystemGPU apply it on the device
  bool SolvePrecond(LsSol::CLinearSystem& ls, unsigned int iv) override {
    MatVec::CVector_Blk& v = ls.GetVector((int)iv, 0);
    const size_t n = VectorSize();
    if (!tmp_r_) {
      tmp_r_.reset(new DeviceVector(*ctx_, n));
      tmp_z_.reset(new DeviceVector(*ctx_, n));
    }
    tmp_r_->upload(detail::values(v));
    ApplyDevice(tmp_r_->data(), tmp_z_->data());
    tmp_z_->download(detail::values(v));
    return true;
  }
  // z := (LU)^-1 r on device arrays (r != z)
  void ApplyDevice(const double* r, double* z) { check(dfm_ilu_apply(ilu_, r, z), "SolvePrecond"); }

  dfm_mat matrix() const { return mat_; }
  dfm_ilu ilu() const { return ilu_; }
  Context& context() const { return *ctx_; }
  size_t VectorSize() const { return (size_t)nblk_ * len_; }

 private:
  Context* ctx_;
  dfm_mat mat_ = nullptr;
  dfm_ilu ilu_ = nullptr;
  int lev_ = 0;
  unsigned nblk_ = 0, len_ = 1;
  std::unique_ptr<DeviceVector> tmp_r_, tmp_z_;
};

// The reference's solver interface over device vectors: handle -1 is the
// CLinearSystem's residual, -2 its update, 0.. the solver's temporaries.
// -1 and -2 are read from the CLinearSystem at construction and written back
// by SyncToHost(), by the Solve_*_GPU functions on exit and by the destructor.
class CLinearSystemGPU : public LsSol::ILinearSystemPreconditioner_Sol, public LsSol::ILinearSystem_Sol {
 public:
  CLinearSystemGPU(LsSol::CLinearSystem& ls, CPreconditioner_ILU_GPU& prec)
      : ls_(&ls), prec_(&prec), n_(prec.VectorSize()), r_(prec.context(), n_), u_(prec.context(), n_) {
    if (!prec.matrix()) throw Error(DFM_ERR_INVALID, "preconditioner without SetLinearSystem");
    const MatVec::CMatDia_BlkCrs& m = detail::segment_matrix(ls);
    if ((size_t)m.NBlkMatCol() * (unsigned)m.LenBlkCol() != n_) throw Error(DFM_ERR_INVALID, "CLinearSystemGPU");
    SyncFromHost();
  }
  ~CLinearSystemGPU() {
    try {
      SyncToHost();
    } catch (...) {
    }
  }
  CLinearSystemGPU(const CLinearSystemGPU&) = delete;
  CLinearSystemGPU& operator=(const CLinearSystemGPU&) = delete;

  // the CLinearSystem's residual (-1) and update (-2) to / from the device
  void SyncFromHost() {
    r_.upload(detail::values(ls_->GetVector(-1, 0)));
    u_.upload(detail::values(ls_->GetVector(-2, 0)));
  }
  void SyncToHost() {
    r_.download(detail::values(ls_->GetVector(-1, 0)));
    u_.download(detail::values(ls_->GetVector(-2, 0)));
  }

  unsigned int GetTmpVectorArySize() const override { return (unsigned)tmp_.size(); }
  bool ReSizeTmpVecSolver(unsigned int size_new) override {
    while (tmp_.size() > size_new) tmp_.pop_back();
    while (tmp_.size() < size_new) tmp_.emplace_back(new DeviceVector(prec_->context(), n_));
    return true;
  }
  double DOT(int iv1, int iv2) override {
    double d = 0.0;
    check(dfm_vec_dot(ctx(), n_, vec(iv1), vec(iv2), &d), "DOT");
    return d;
  }
  bool COPY(int iv1, int iv2) override {
    if (iv1 == iv2) return true;
    check(dfm_vec_copy(ctx(), n_, vec(iv1), vec(iv2)), "COPY");
    return true;
  }
  bool SCAL(double alpha, int iv1) override {
    check(dfm_vec_scal(ctx(), n_, alpha, vec(iv1)), "SCAL");
    return true;
  }
  bool AXPY(double alpha, int iv1, int iv2) override {
    if (alpha == 0.0) return true;  // CLinearSystem::AXPY returns at once
    if (iv1 == iv2) return false;   // not implemented in the reference either
    check(dfm_vec_axpy(ctx(), n_, alpha, vec(iv1), vec(iv2)), "AXPY");
    return true;
  }
  bool MATVEC(double alpha, int iv1, double beta, int iv2) override {
    if (alpha == 0.0) return SCAL(beta, iv2);  // as CLinearSystem::MATVEC
    if (iv1 == iv2) return false;
    check(dfm_spmv(prec_->matrix(), alpha, vec(iv1), beta, vec(iv2)), "MATVEC");
    return true;
  }
  bool SolvePrecond(int iv) override {
    if (!z_) z_.reset(new DeviceVector(prec_->context(), n_));
    prec_->ApplyDevice(vec(iv), z_->data());
    check(dfm_vec_copy(ctx(), n_, z_->data(), vec(iv)), "SolvePrecond");
    return true;
  }

  // device array behind a handle
  double* vec(int iv) {
    if (iv == -1) return r_.data();
    if (iv == -2) return u_.data();
    if (iv < 0 || (size_t)iv >= tmp_.size()) throw Error(DFM_ERR_INVALID, "vector handle");
    return tmp_[(size_t)iv]->data();
  }
  CPreconditioner_ILU_GPU& preconditioner() const { return *prec_; }

 private:
  dfm_ctx ctx() const { return prec_->context().get(); }
  LsSol::CLinearSystem* ls_;
  CPreconditioner_ILU_GPU* prec_;
  size_t n_;
  DeviceVector r_, u_;
  std::vector<std::unique_ptr<DeviceVector>> tmp_;
  std::unique_ptr<DeviceVector> z_;
};

namespace detail {
template <class I>
inline CLinearSystemGPU& gpu_system(I& lsp, const char* who) {
  CLinearSystemGPU* g = dynamic_cast<CLinearSystemGPU*>(&lsp);
  if (!g) throw Error(DFM_ERR_UNSUPPORTED, std::string(who) + ": the linear system is not a CLinearSystemGPU");
  return *g;
}
// runs one device solve with the reference's in/out conventions, then writes
// -1 and -2 back into the CLinearSystem
template <class Fn>
inline bool run(CLinearSystemGPU& g, Fn fn, double& conv_ratio, unsigned int& iteration, bool true_at_maxit) {
  bool ok = false;
  try {
    ok = dfm_lsol::detail::solve(fn, conv_ratio, iteration, true_at_maxit);
  } catch (...) {
    try {
      g.SyncToHost();
    } catch (...) {
    }
    throw;
  }
  g.SyncToHost();
  return ok;
}
}  // namespace detail

// LsSol::Solve_PCG(conv_ratio, iteration, lsp): ILU-preconditioned CG on the
// device; iteration is the 0-based index of the converged iteration, false at
// max_iter with conv_ratio = |r|/|r0|.
inline bool Solve_PCG_GPU(double& conv_ratio, unsigned int& iteration, LsSol::ILinearSystemPreconditioner_Sol& lsp) {
  CLinearSystemGPU& g = detail::gpu_system(lsp, "Solve_PCG_GPU");
  CPreconditioner_ILU_GPU& M = g.preconditioner();
  return detail::run(g, [&](double t, unsigned m, unsigned* it, double* cv) {
    return dfm_solve_pcg(M.matrix(), M.ilu(), g.vec(-1), g.vec(-2), t, m, it, cv);
  }, conv_ratio, iteration, false);
}

// LsSol::Solve_PBiCGSTAB(conv_ratio, num_iter, lsp): 1-based count; at
// max_iter true with conv_ratio left at the tolerance.
inline bool Solve_PBiCGSTAB_GPU(double& conv_ratio, unsigned int& num_iter,
                                LsSol::ILinearSystemPreconditioner_Sol& lsp) {
  CLinearSystemGPU& g = detail::gpu_system(lsp, "Solve_PBiCGSTAB_GPU");
  CPreconditioner_ILU_GPU& M = g.preconditioner();
  return detail::run(g, [&](double t, unsigned m, unsigned* it, double* cv) {
    return dfm_solve_pbicgstab(M.matrix(), M.ilu(), g.vec(-1), g.vec(-2), t, m, it, cv);
  }, conv_ratio, num_iter, true);
}

// LsSol::Solve_CG(conv_ratio, num_iter, ls): no preconditioner (the
// CLinearSystemGPU's matrix only); at max_iter true with conv_ratio left at
// the tolerance.
inline bool Solve_CG_GPU(double& conv_ratio, unsigned int& num_iter, LsSol::ILinearSystem_Sol& ls) {
  CLinearSystemGPU& g = detail::gpu_system(ls, "Solve_CG_GPU");
  CPreconditioner_ILU_GPU& M = g.preconditioner();
  return detail::run(g, [&](double t, unsigned m, unsigned* it, double* cv) {
    return dfm_solve_cg(M.matrix(), g.vec(-1), g.vec(-2), t, m, it, cv);
  }, conv_ratio, num_iter, true);
}

}  // namespace dfm_delfem

#endif
