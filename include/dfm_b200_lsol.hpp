// dfm_b200_lsol.hpp - header-only C++ adapters over the C ABI (dfm_b200.h)
// that mirror the reference's solver-side classes and functions, so code
// written against them switches by changing the namespace:
//
//   MatVec::CMatDia_BlkCrs                 -> dfm_lsol::CMatDia_BlkCrs
//       (include/delfem/matvec/matdia_blkcrs.h:44-118)
//   LsSol::CPreconditioner_ILU             -> dfm_lsol::CPreconditioner_ILU
//       (include/delfem/ls/preconditioner.h:54-108: SetFillInLevel,
//        SetLinearSystem, SetValue, SolvePrecond; one segment, no ordering)
//   LsSol::Solve_PCG / Solve_PBiCGSTAB     -> dfm_lsol::Solve_PCG / Solve_PBiCGSTAB
//       (include/delfem/ls/solver_ls_iter.h:35-45)
//   Fem::Ls::Solve_PCOCG                   -> dfm_lsol::Solve_PCOCG
//       (include/delfem/femls/zsolver_ls_iter.h:53-54)
//
// The solver functions keep the reference's in/out argument convention:
// conv_ratio holds the tolerance on entry and the achieved ratio on exit,
// iteration holds max_iter on entry and the count on exit (0-based index for
// PCG, 1-based for PBiCGSTAB / PCOCG), and the return value is the
// reference's: PCG returns false at max_iter, PBiCGSTAB and PCOCG return true
// there (and leave conv_ratio at the tolerance).  Vectors live on the device
// (DeviceVector); r holds the right-hand side on entry and the residual on
// exit, x receives the solution from a zero start.  Errors other than
// non-convergence throw dfm_lsol::Error.
//
// Only the C ABI is used: a program needs this header, dfm_b200.h and
// libdfm_b200.so, not the CUDA toolkit.
#ifndef DFM_B200_LSOL_HPP
#define DFM_B200_LSOL_HPP

#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dfm_b200.h"

namespace dfm_lsol {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& where)
      : std::runtime_error(where + ": " + dfm_status_string(c)), code(c) {}
};

inline int check(int rc, const char* where, int allow = DFM_OK) {
  if (rc != DFM_OK && rc != allow) throw Error(rc, where);
  return rc;
}

// One device and its stream.
class Context {
 public:
  explicit Context(int device = 0) { check(dfm_ctx_create(device, &h_), "dfm_ctx_create"); }
  ~Context() { dfm_ctx_destroy(h_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  dfm_ctx get() const { return h_; }

 private:
  dfm_ctx h_ = nullptr;
};

// A device array of doubles (the reference's CVector_Blk storage on the GPU).
class DeviceVector {
 public:
  DeviceVector(Context& c, size_t n) : c_(&c), n_(n) {
    check(dfm_buf_alloc(c.get(), n * sizeof(double), &p_), "dfm_buf_alloc");
    check(dfm_buf_zero(c.get(), p_, n * sizeof(double)), "dfm_buf_zero");
  }
  ~DeviceVector() {
    if (p_) dfm_buf_free(c_->get(), p_);
  }
  DeviceVector(const DeviceVector&) = delete;
  DeviceVector& operator=(const DeviceVector&) = delete;
  DeviceVector(DeviceVector&& o) noexcept : c_(o.c_), p_(o.p_), n_(o.n_) { o.p_ = nullptr; }
  double* data() { return static_cast<double*>(p_); }
  const double* data() const { return static_cast<const double*>(p_); }
  size_t size() const { return n_; }
  void upload(const double* h) { check(dfm_buf_copy(c_->get(), p_, h, n_ * sizeof(double), DFM_H2D), "upload"); }
  void download(double* h) const {
    check(dfm_buf_copy(c_->get(), h, p_, n_ * sizeof(double), DFM_D2H), "download");
  }
  void copy_from(const DeviceVector& o) {
    check(dfm_buf_copy(c_->get(), p_, o.p_, n_ * sizeof(double), DFM_D2D), "copy");
  }
  void set_zero() { check(dfm_buf_zero(c_->get(), p_, n_ * sizeof(double)), "set_zero"); }

 private:
  Context* c_;
  void* p_ = nullptr;
  size_t n_ = 0;
};

// MatVec::CMatDia_BlkCrs / CZMatDia_BlkCrs (complex: len = 1, is_complex).
class CMatDia_BlkCrs {
 public:
  CMatDia_BlkCrs(Context& c, unsigned nblk, unsigned len, const unsigned* rowptr, const unsigned* colind,
                 bool is_complex = false)
      : c_(&c), nblk_(nblk), len_(len), cplx_(is_complex) {
    check(dfm_mat_create(c.get(), nblk, len, is_complex ? DFM_COMPLEX : DFM_REAL, rowptr, colind, &h_),
          "dfm_mat_create");
    unsigned n, b, ncrs;
    int vt;
    check(dfm_mat_info(h_, &n, &b, &ncrs, &vt), "dfm_mat_info");
    ncrs_ = ncrs;
  }
  // From a reference matrix through its public accessors (NBlkMatCol,
  // LenBlkCol, GetPtrIndPSuP, GetPtrValPSuP, GetPtrValDia): pattern and values.
  template <class RefMat>
  static CMatDia_BlkCrs FromReference(Context& c, const RefMat& m) {
    const unsigned n = m.NBlkMatCol(), len = m.LenBlkCol();
    std::vector<unsigned> rp(n + 1, 0), ci;
    for (unsigned i = 0; i < n; i++) {
      unsigned np = 0;
      const unsigned* p = m.GetPtrIndPSuP(i, np);
      rp[i + 1] = rp[i] + np;
      ci.insert(ci.end(), p, p + np);
    }
    CMatDia_BlkCrs A(c, n, len, rp.data(), ci.data());
    A.SetValueFromReference(m);
    return A;
  }
  // MatVec::CZMatDia_BlkCrs(const std::string& file_path): a complex matrix
  // from the reference's text format (dfm_zmat_read_text).
  static CMatDia_BlkCrs FromTextFile(Context& c, const std::string& path) {
    unsigned n = 0, ncrs = 0;
    check(dfm_zmat_read_text(path.c_str(), &n, &ncrs, nullptr, nullptr, nullptr, nullptr), "FromTextFile");
    std::vector<unsigned> rp(n + 1), ci(ncrs);
    std::vector<double> d(2 * (size_t)n), o(2 * (size_t)ncrs);
    check(dfm_zmat_read_text(path.c_str(), &n, &ncrs, rp.data(), ci.data(), d.data(), o.data()), "FromTextFile");
    CMatDia_BlkCrs A(c, n, 1, rp.data(), ci.data(), true);
    A.SetValue(d.data(), o.data());
    return A;
  }
  template <class RefMat>
  void SetValueFromReference(const RefMat& m) {
    const size_t bb = (size_t)len_ * len_;
    std::vector<double> d((size_t)nblk_ * bb), o((size_t)ncrs_ * bb);
    size_t k = 0;
    for (unsigned i = 0; i < nblk_; i++) {
      const double* pd = m.GetPtrValDia(i);
      for (size_t q = 0; q < bb; q++) d[i * bb + q] = pd[q];
      unsigned np = 0;
      const double* po = m.GetPtrValPSuP(i, np);
      for (size_t q = 0; q < np * bb; q++) o[k + q] = po[q];
      k += np * bb;
    }
    SetValue(d.data(), o.data());
  }
  ~CMatDia_BlkCrs() { dfm_mat_destroy(h_); }
  CMatDia_BlkCrs(const CMatDia_BlkCrs&) = delete;
  CMatDia_BlkCrs& operator=(const CMatDia_BlkCrs&) = delete;
  CMatDia_BlkCrs(CMatDia_BlkCrs&& o) noexcept
      : c_(o.c_), h_(o.h_), nblk_(o.nblk_), len_(o.len_), ncrs_(o.ncrs_), cplx_(o.cplx_) {
    o.h_ = nullptr;
  }

  unsigned NBlkMatCol() const { return nblk_; }
  unsigned LenBlkCol() const { return len_; }
  unsigned NCrs() const { return ncrs_; }
  bool IsComplex() const { return cplx_; }
  size_t VectorSize() const { return (size_t)nblk_ * (cplx_ ? 2 : len_); }
  // CMatDia_BlkCrs::SetZero
  void SetZero() { check(dfm_mat_set_zero(h_), "SetZero"); }
  // host arrays in the reference layout (diag[nblk*len*len], off[ncrs*len*len])
  void SetValue(const double* diag, const double* off) {
    check(dfm_mat_set_values(h_, diag, off, DFM_HOST), "SetValue");
  }
  // {y} := alpha [A] {x} + beta {y}  (CMatDia_BlkCrs::MatVec)
  void MatVec(double alpha, const DeviceVector& x, double beta, DeviceVector& y) const {
    check(dfm_spmv(h_, alpha, x.data(), beta, y.data()), "MatVec");
  }
  dfm_mat get() const { return h_; }
  Context& context() const { return *c_; }

 private:
  Context* c_;
  dfm_mat h_ = nullptr;
  unsigned nblk_ = 0, len_ = 1, ncrs_ = 0;
  bool cplx_ = false;
};

// LsSol::CPreconditioner_ILU with the natural ordering: ILU(0), or ILU(k)
// after SetFillInLevel(k).
class CPreconditioner_ILU {
 public:
  CPreconditioner_ILU() = default;
  explicit CPreconditioner_ILU(const CMatDia_BlkCrs& A) { SetLinearSystem(A); }
  ~CPreconditioner_ILU() { Clear(); }
  CPreconditioner_ILU(const CPreconditioner_ILU&) = delete;
  CPreconditioner_ILU& operator=(const CPreconditioner_ILU&) = delete;
  void Clear() {
    if (h_) dfm_ilu_destroy(h_);
    h_ = nullptr;
  }
  // SetFillInLevel(lev, ilss): ILU(lev) from the next SetLinearSystem on
  // (-1: no limit).  A single-segment system: ilss must be -1 or 0.
  void SetFillInLevel(int lev, int ilss = -1) {
    if (ilss != -1 && ilss != 0) throw Error(DFM_ERR_UNSUPPORTED, "SetFillInLevel");
    if (lev < -1) throw Error(DFM_ERR_INVALID, "SetFillInLevel");
    lev_ = lev;
  }
  // SetFillBlk(aBlk): block rows whose fill has no level limit from the next
  // SetLinearSystem on (AddFracPtn(lev, aBlkFill)); empty: none
  void SetFillBlk(const std::vector<unsigned int>& aBlk) { blk_ = aBlk; }
  // fill pattern (ILU(lev)) and level sets of the sweeps
  void SetLinearSystem(const CMatDia_BlkCrs& A) {
    Clear();
    check(dfm_ilu_create_fill_rows(A.get(), lev_, blk_.data(), blk_.size(), A.NBlkMatCol(), &h_), "SetLinearSystem");
  }
  // numeric factorization; false when more than 10 pivots were singular
  bool SetValue(const CMatDia_BlkCrs& A) {
    unsigned ns = 0;
    return check(dfm_ilu_factor(h_, A.get(), &ns), "SetValue", DFM_SINGULAR_PIVOT) == DFM_OK;
  }
  // {z} := (LU)^-1 {r}
  bool SolvePrecond(const DeviceVector& r, DeviceVector& z) {
    check(dfm_ilu_apply(h_, r.data(), z.data()), "SolvePrecond");
    return true;
  }
  dfm_ilu get() const { return h_; }

 private:
  dfm_ilu h_ = nullptr;
  int lev_ = 0;
  std::vector<unsigned int> blk_;
};

// Fem::Ls::CLinearSystem_Save::MakeResidual: {r} := {force} - [B]{u} with B
// the stored boundary matrix (dfm_boundary_matrix); returns |r|.
inline double MakeResidual(const CMatDia_BlkCrs& B, const DeviceVector& force, const DeviceVector& u,
                           DeviceVector& r) {
  r.copy_from(force);
  B.MatVec(-1.0, u, 1.0, r);
  std::vector<double> h(B.VectorSize());
  r.download(h.data());
  double s = 0.0;
  for (double v : h) s += v * v;
  return std::sqrt(s);
}

namespace detail {
template <class Fn>
inline bool solve(Fn fn, double& conv_ratio, unsigned int& iteration, bool true_at_maxit) {
  const double tol = conv_ratio;
  const unsigned maxit = iteration;
  unsigned it = 0;
  double conv = 0.0;
  const int rc = check(fn(tol, maxit, &it, &conv), "solve", DFM_NOT_CONVERGED);
  iteration = it;
  if (rc == DFM_NOT_CONVERGED) {
    if (true_at_maxit) return true;  // the reference keeps conv_ratio at the tolerance here
    conv_ratio = conv;
    return false;
  }
  conv_ratio = conv;
  return true;
}
}  // namespace detail

// LsSol::Solve_PCG(conv_ratio, iteration, lsp)
inline bool Solve_PCG(double& conv_ratio, unsigned int& iteration, CMatDia_BlkCrs& A, CPreconditioner_ILU& M,
                      DeviceVector& r, DeviceVector& x) {
  return detail::solve([&](double t, unsigned m, unsigned* it, double* cv) {
    return dfm_solve_pcg(A.get(), M.get(), r.data(), x.data(), t, m, it, cv);
  }, conv_ratio, iteration, false);
}

// LsSol::Solve_PBiCGSTAB(conv_ratio, num_iter, lsp)
inline bool Solve_PBiCGSTAB(double& conv_ratio, unsigned int& num_iter, CMatDia_BlkCrs& A, CPreconditioner_ILU& M,
                            DeviceVector& r, DeviceVector& x) {
  return detail::solve([&](double t, unsigned m, unsigned* it, double* cv) {
    return dfm_solve_pbicgstab(A.get(), M.get(), r.data(), x.data(), t, m, it, cv);
  }, conv_ratio, num_iter, true);
}

// Fem::Ls::Solve_PCOCG(conv_ratio, iteration, ls, prec)
inline bool Solve_PCOCG(double& conv_ratio, unsigned int& iteration, CMatDia_BlkCrs& A, CPreconditioner_ILU& M,
                        DeviceVector& r, DeviceVector& x) {
  return detail::solve([&](double t, unsigned m, unsigned* it, double* cv) {
    return dfm_solve_pcocg(A.get(), M.get(), r.data(), x.data(), t, m, it, cv);
  }, conv_ratio, iteration, true);
}

}  // namespace dfm_lsol

#endif
