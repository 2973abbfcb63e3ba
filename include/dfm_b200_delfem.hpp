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
// Scope: fixed b x b blocks, b in {1, 2, 3}, in one segment (the
// CMatDia_BlkCrs of a single field) or in several (a combined field, bubble
// DOFs: CLinearSystem::AddLinSysSeg with couplings GetMatrix(i, j)); several
// segments are joined into one device matrix (detail::Layout) and take ILU(0).
// Errors other than the reference's boolean results throw dfm_lsol::Error.
#ifndef DFM_B200_DELFEM_HPP
#define DFM_B200_DELFEM_HPP

#include <algorithm>
#include <memory>
#include <utility>
#include <vector>

#include "delfem/ls/linearsystem.h"
#include "delfem/ls/linearsystem_interface_solver.h"
#include "delfem/ls/preconditioner.h"
#include "delfem/ls/solver_ls_iter.h"
#include "delfem/matvec/mat_blkcrs.h"
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
// Contiguous values of a fixed-length CVector_Blk.
inline double* values(MatVec::CVector_Blk& v) { return v.NBlk() ? v.GetValuePtr(0) : nullptr; }
inline const double* values(const MatVec::CVector_Blk& v) { return v.NBlk() ? v.GetValuePtr(0) : nullptr; }

// The segments of a CLinearSystem (src/ls/linearsystem.cpp: AddLinSysSeg,
// AddMat_Dia, AddMat_NonDia) joined into one square matrix for the device:
// segment i's rows follow segment i-1's, its diagonal matrix GetMatrix(i)
// and its couplings GetMatrix(i, j) (CMat_BlkCrs, rows in segment i, columns
// in segment j) become one block row each.  Segments of one block length b
// keep b x b blocks; segments of different lengths are joined one row per
// DOF (b = 1).  Either way the joined vector is the segments' vectors one
// after the other, and the joined pattern is the union of the segments'
// patterns, so ILU(0) of the joined matrix is the reference's segment-wise
// block ILU(0) (src/ls/preconditioner.cpp:57-335: the same incomplete
// factorization on the same block pattern, summed in another order).
struct Layout {
  unsigned nseg = 0;
  std::vector<unsigned> nblk, len;
  std::vector<size_t> dof0;  // first joined vector entry of each segment
  unsigned b = 1, N = 0;     // joined block size and block rows
  bool scalar = false;       // segments of different lengths: one row per DOF
  size_t ndof = 0;
  std::vector<unsigned> rowptr, colind;

  void build(const LsSol::CLinearSystem& ls) {
    nseg = ls.GetNLinSysSeg();
    if (nseg == 0) throw Error(DFM_ERR_INVALID, "a linear system without segments");
    nblk.assign(nseg, 0);
    len.assign(nseg, 0);
    dof0.assign(nseg + 1, 0);
    for (unsigned i = 0; i < nseg; i++) {
      if (!ls.IsMatrix(i, i)) throw Error(DFM_ERR_UNSUPPORTED, "a segment without its diagonal matrix");
      const MatVec::CMatDia_BlkCrs& m = ls.GetMatrix(i);
      if (m.LenBlkCol() < 1 || m.LenBlkCol() > 3) throw Error(DFM_ERR_UNSUPPORTED, "block size");
      nblk[i] = m.NBlkMatCol();
      len[i] = (unsigned)m.LenBlkCol();
      dof0[i + 1] = dof0[i] + (size_t)nblk[i] * len[i];
    }
    ndof = dof0[nseg];
    scalar = false;
    for (unsigned i = 1; i < nseg; i++) scalar |= len[i] != len[0];
    b = scalar ? 1u : len[0];
    N = (unsigned)(ndof / b);
    std::vector<double> d, o;
    walk(ls, false, d, o);
  }

  // pattern (always) and values (with_values) of the joined matrix, row by row
  // in ascending columns; the pattern pass reads no values (a CLinearSystem
  // has none before its first InitializeMarge)
  void walk(const LsSol::CLinearSystem& ls, bool with_values, std::vector<double>& diag, std::vector<double>& off) {
    std::vector<unsigned>& rp = rowptr;
    std::vector<unsigned>& ci = colind;
    const size_t bb = (size_t)b * b;
    if (!with_values) {
      rp.assign(N + 1, 0);
      ci.clear();
    } else {
      diag.assign((size_t)N * bb, 0.0);
      off.assign(colind.size() * bb, 0.0);
    }
    size_t k = 0;  // off-diagonal slot
    auto put = [&](unsigned col, const double* v) {
      if (!with_values) ci.push_back(col);
      else std::copy(v, v + bb, off.begin() + k * bb);
      k++;
    };
    unsigned row = 0;
    for (unsigned i = 0; i < nseg; i++) {
      const MatVec::CMatDia_BlkCrs& A = ls.GetMatrix(i);
      const unsigned Li = len[i];
      for (unsigned p = 0; p < nblk[i]; p++) {
        unsigned nd = 0, nv = 0;
        const unsigned* dcol = A.GetPtrIndPSuP(p, nd);
        const double* dval = A.GetPtrValPSuP(p, nv);
        const double* dia = A.GetPtrValDia(p);
        for (unsigned d = 0; d < (scalar ? Li : 1u); d++) {
          // one joined row: block row p of segment i, or its DOF d
          for (unsigned j = 0; j < nseg; j++) {
            if (j == i) {
              bool dia_done = false;
              auto put_dia = [&]() {  // the rest of the diagonal block (scalar rows only)
                for (unsigned e = 0; e < Li; e++)
                  if (e != d) {
                    const double v = with_values ? dia[d * Li + e] : 0.0;
                    put((unsigned)(dof0[i] + (size_t)p * Li + e), &v);
                  }
                dia_done = true;
              };
              for (unsigned t = 0; t < nd; t++) {
                const unsigned c = dcol[t];
                if (scalar && !dia_done && c > p) put_dia();
                if (!scalar) {
                  put((unsigned)(dof0[i] / b + c), dval + (size_t)t * bb);
                } else {
                  for (unsigned e = 0; e < Li; e++) {
                    const double v = with_values ? dval[(size_t)t * Li * Li + d * Li + e] : 0.0;
                    put((unsigned)(dof0[i] + (size_t)c * Li + e), &v);
                  }
                }
              }
              if (scalar && !dia_done) put_dia();
            } else if (ls.IsMatrix(i, j)) {
              const MatVec::CMat_BlkCrs& C = ls.GetMatrix(i, j);
              const unsigned Lj = len[j];
              unsigned nc = 0, ncv = 0;
              const unsigned* ccol = C.GetPtrIndPSuP(p, nc);
              const double* cval = C.GetPtrValPSuP(p, ncv);
              for (unsigned t = 0; t < nc; t++) {
                if (!scalar) {
                  put((unsigned)(dof0[j] / b + ccol[t]), cval + (size_t)t * bb);
                } else {
                  for (unsigned e = 0; e < Lj; e++) {
                    const double v = with_values ? cval[(size_t)t * Li * Lj + d * Lj + e] : 0.0;
                    put((unsigned)(dof0[j] + (size_t)ccol[t] * Lj + e), &v);
                  }
                }
              }
            }
          }
          if (with_values) {
            if (!scalar) std::copy(dia, dia + bb, diag.begin() + (size_t)row * bb);
            else diag[row] = dia[d * Li + d];
          }
          row++;
          if (!with_values) rp[row] = (unsigned)k;
        }
      }
    }
  }

  // the CLinearSystem's vector iv, segments one after the other
  void gather(const LsSol::CLinearSystem& ls, int iv, double* out) const {
    for (unsigned i = 0; i < nseg; i++) {
      const double* v = values(ls.GetVector(iv, i));
      if (v) std::copy(v, v + (dof0[i + 1] - dof0[i]), out + dof0[i]);
    }
  }
  void scatter(LsSol::CLinearSystem& ls, int iv, const double* in) const {
    for (unsigned i = 0; i < nseg; i++) {
      double* v = values(ls.GetVector(iv, i));
      if (v) std::copy(in + dof0[i], in + dof0[i + 1], v);
    }
  }
};
}  // namespace detail

// LsSol::CPreconditioner_ILU on the device: ILU(0), or ILU(k) after
// SetFillInLevel(k), in the natural ordering.  It also owns the device copy of
// the system matrix, which CLinearSystemGPU multiplies with.  A system of
// several segments is factored as one joined matrix (segments one after the
// other; one row per DOF when their block lengths differ): ILU(k) of the
// joined matrix is the reference's segment-wise block ILU(k)
// (src/ls/preconditioner.cpp:57-335) when every segment pair has the same
// level, since both are the incomplete factorisation on the same fill pattern.
class CPreconditioner_ILU_GPU : public LsSol::CPreconditioner {
 public:
  explicit CPreconditioner_ILU_GPU(Context& ctx) : ctx_(&ctx) {}
  CPreconditioner_ILU_GPU(Context& ctx, const LsSol::CLinearSystem& ls, unsigned int nlev = 0) : ctx_(&ctx) {
    SetFillInLevel((int)nlev);
    SetLinearSystem(ls);
  }
  ~CPreconditioner_ILU_GPU() override { release(); }
  CPreconditioner_ILU_GPU(const CPreconditioner_ILU_GPU&) = delete;
  CPreconditioner_ILU_GPU& operator=(const CPreconditioner_ILU_GPU&) = delete;

  // the device objects, the fill-level requests and the ordering (as the
  // reference's Clear, src/ls/preconditioner.cpp:31-52)
  void Clear() {
    release();
    lev_in_.clear();
    order_.clear();
  }
  // CPreconditioner_ILU::SetOrdering (include/delfem/ls/preconditioner.h:93-97):
  // for the next SetLinearSystem, factor the system with its block rows and
  // columns renumbered, aind[new] = old (COrdering_Blk); empty: off.  As the
  // reference's ordered path (src/ls/preconditioner.cpp:60-82, 224-229,
  // 305-311) it is ILU(0) of one segment, whatever the fill level.
  void SetOrdering(const std::vector<int>& aind) { order_ = aind; }
  bool ordered() const { return !order_.empty(); }
  // a fill-in level request for the next SetLinearSystem (-1: no limit), for
  // every segment pair (ilss0 == -1) or the pairs of segment ilss0; requests
  // apply in order, later ones over earlier ones (the reference's alev table)
  void SetFillInLevel(int lev, int ilss0 = -1) {
    if (lev < -1 || ilss0 < -1) throw Error(DFM_ERR_INVALID, "SetFillInLevel");
    lev_in_.emplace_back(lev, ilss0);
  }
  // CPreconditioner_ILU::SetFillBlk (include/delfem/ls/preconditioner.h:80):
  // block rows of the first segment whose fill has no level limit at the next
  // SetLinearSystem (the reference passes the list to that segment's diagonal
  // matrix, AddFracPtn(lev, aBlkFill), src/ls/preconditioner.cpp:140-142);
  // Clear keeps it, as the reference's does, and an ordering ignores it
  void SetFillBlk(const std::vector<unsigned int>& aBlk) { fill_blk_ = aBlk; }
  // pattern of the (joined) system matrix on the device, fill pattern and
  // level sets
  void SetLinearSystem(const LsSol::CLinearSystem& ls) override {
    release();
    lay_.build(ls);
    lev_ = fill_level(lay_.nseg);
    check(dfm_mat_create(ctx_->get(), lay_.N, lay_.b, DFM_REAL, lay_.rowptr.data(), lay_.colind.data(), &mat_),
          "SetLinearSystem");
    if (ordered()) {
      make_ordered();
      check(dfm_ilu_create(pmat_, &ilu_), "SetLinearSystem");
    } else if (!fill_blk_.empty()) {
      // the listed block rows as rows of the joined matrix (every DOF row of
      // the block when the join is one row per DOF); the flags act within the
      // first segment's rows
      const unsigned L = lay_.scalar ? lay_.len[0] : 1u;
      std::vector<unsigned> rows;
      rows.reserve(fill_blk_.size() * L);
      for (unsigned r : fill_blk_) {
        if (r >= lay_.nblk[0]) throw Error(DFM_ERR_INVALID, "SetFillBlk: block row out of range");
        for (unsigned d = 0; d < L; d++) rows.push_back(r * L + d);
      }
      check(dfm_ilu_create_fill_rows(mat_, lev_, rows.data(), rows.size(), lay_.nblk[0] * L, &ilu_),
            "SetLinearSystem");
    } else {
      check(dfm_ilu_create_fill(mat_, lev_, &ilu_), "SetLinearSystem");
    }
  }
  // the fill level of every segment pair after the requests; different levels
  // for different pairs are not supported
  int fill_level(unsigned nseg) const {
    std::vector<int> alev((size_t)nseg * nseg, 0);
    for (const auto& r : lev_in_) {
      if (r.second == -1) {
        std::fill(alev.begin(), alev.end(), r.first);
        continue;
      }
      if ((unsigned)r.second >= nseg) throw Error(DFM_ERR_INVALID, "SetFillInLevel: segment index");
      for (unsigned i = 0; i < nseg; i++) alev[(size_t)i * nseg + r.second] = alev[(size_t)r.second * nseg + i] = r.first;
    }
    for (int v : alev)
      if (v != alev[0]) throw Error(DFM_ERR_UNSUPPORTED, "different fill-in levels for different segment pairs");
    return alev.empty() ? 0 : alev[0];
  }
  // the system's current values to the device and the numeric factorisation;
  // false when more than 10 pivots were singular (the reference's result)
  bool SetValue(const LsSol::CLinearSystem& ls) override {
    if (!mat_) throw Error(DFM_ERR_INVALID, "SetValue before SetLinearSystem");
    if (ls.GetNLinSysSeg() != lay_.nseg) throw Error(DFM_ERR_INVALID, "SetValue");
    for (unsigned i = 0; i < lay_.nseg; i++)
      if (ls.GetMatrix(i).NBlkMatCol() != lay_.nblk[i] || (unsigned)ls.GetMatrix(i).LenBlkCol() != lay_.len[i])
        throw Error(DFM_ERR_INVALID, "SetValue");
    if (lay_.nseg == 1) {  // one segment: the reference's arrays are the library's layout
      const MatVec::CMatDia_BlkCrs& m = ls.GetMatrix(0);
      unsigned np = 0;
      const double* off = m.NCrs() ? m.GetPtrValPSuP(0, np) : nullptr;  // row-ordered, contiguous
      const double* dia = lay_.N ? m.GetPtrValDia(0) : nullptr;
      check(dfm_mat_set_values(mat_, dia, off, DFM_HOST), "SetValue");
      if (ordered()) {  // the renumbered matrix: block i of row i' from block n2o(i) of row n2o(i')
        const size_t bb = (size_t)lay_.b * lay_.b;
        std::vector<double> pd((size_t)lay_.N * bb), po(psrc_.size() * bb);
        for (unsigned i = 0; i < lay_.N; i++) std::copy(dia + n2o_[i] * bb, dia + (n2o_[i] + 1) * bb, pd.begin() + i * bb);
        for (size_t t = 0; t < psrc_.size(); t++)
          std::copy(off + psrc_[t] * bb, off + (psrc_[t] + 1) * bb, po.begin() + t * bb);
        check(dfm_mat_set_values(pmat_, pd.data(), po.data(), DFM_HOST), "SetValue");
      }
    } else {
      std::vector<double> d, o;
      lay_.walk(ls, true, d, o);
      check(dfm_mat_set_values(mat_, d.data(), o.data(), DFM_HOST), "SetValue");
    }
    unsigned ns = 0;
    return check(dfm_ilu_factor(ilu_, ordered() ? pmat_ : mat_, &ns), "SetValue", DFM_SINGULAR_PIVOT) == DFM_OK;
  }
  // {iv} := (LU)^-1 {iv} on the CLinearSystem's host vectors (copied to the
  // device and back); solvers over CLinearSystemGPU apply it on the device
  bool SolvePrecond(LsSol::CLinearSystem& ls, unsigned int iv) override {
    const size_t n = VectorSize();
    if (!tmp_r_) {
      tmp_r_.reset(new DeviceVector(*ctx_, n));
      tmp_z_.reset(new DeviceVector(*ctx_, n));
    }
    std::vector<double> h(n);
    lay_.gather(ls, (int)iv, h.data());
    tmp_r_->upload(h.data());
    ApplyDevice(tmp_r_->data(), tmp_z_->data());
    tmp_z_->download(h.data());
    lay_.scatter(ls, (int)iv, h.data());
    return true;
  }
  // z := (LU)^-1 r on device arrays (r != z); with an ordering the vector is
  // renumbered in (OrderingVector_OldToNew), swept, and renumbered back
  void ApplyDevice(const double* r, double* z) {
    if (!ordered()) {
      check(dfm_ilu_apply(ilu_, r, z), "SolvePrecond");
      return;
    }
    if (!tmp_o1_) {
      tmp_o1_.reset(new DeviceVector(*ctx_, lay_.ndof));
      tmp_o2_.reset(new DeviceVector(*ctx_, lay_.ndof));
    }
    check(dfm_vec_gather(ctx_->get(), lay_.N, lay_.b, static_cast<const unsigned*>(d_n2o_), r, tmp_o1_->data()),
          "SolvePrecond");
    check(dfm_ilu_apply(ilu_, tmp_o1_->data(), tmp_o2_->data()), "SolvePrecond");
    check(dfm_vec_gather(ctx_->get(), lay_.N, lay_.b, static_cast<const unsigned*>(d_o2n_), tmp_o2_->data(), z),
          "SolvePrecond");
  }

  dfm_mat matrix() const { return mat_; }
  dfm_ilu ilu() const { return ilu_; }
  Context& context() const { return *ctx_; }
  size_t VectorSize() const { return lay_.ndof; }
  const detail::Layout& layout() const { return lay_; }

 private:
  void release() {
    if (ilu_) dfm_ilu_destroy(ilu_);
    if (mat_) dfm_mat_destroy(mat_);
    if (pmat_) dfm_mat_destroy(pmat_);
    if (d_n2o_) dfm_buf_free(ctx_->get(), d_n2o_);
    if (d_o2n_) dfm_buf_free(ctx_->get(), d_o2n_);
    ilu_ = nullptr;
    mat_ = pmat_ = nullptr;
    d_n2o_ = d_o2n_ = nullptr;
    tmp_r_.reset();
    tmp_z_.reset();
    tmp_o1_.reset();
    tmp_o2_.reset();
  }
  // the renumbered pattern (row i = old row n2o[i], columns renumbered and
  // sorted), where each of its blocks comes from, and the maps on the device
  void make_ordered() {
    if (lay_.nseg != 1) throw Error(DFM_ERR_UNSUPPORTED, "SetOrdering with several segments");
    const unsigned N = lay_.N;
    if (order_.size() != N) throw Error(DFM_ERR_INVALID, "SetOrdering: one entry per block row");
    n2o_.assign(N, 0);
    std::vector<unsigned> o2n(N, ~0u);
    for (unsigned i = 0; i < N; i++) {
      const int v = order_[i];
      if (v < 0 || (unsigned)v >= N || o2n[v] != ~0u) throw Error(DFM_ERR_INVALID, "SetOrdering: not a permutation");
      n2o_[i] = (unsigned)v;
      o2n[v] = i;
    }
    std::vector<unsigned> prow(N + 1, 0), pcol;
    psrc_.clear();
    std::vector<std::pair<unsigned, unsigned>> row;
    for (unsigned i = 0; i < N; i++) {
      const unsigned o = n2o_[i];
      row.clear();
      for (unsigned t = lay_.rowptr[o]; t < lay_.rowptr[o + 1]; t++) row.emplace_back(o2n[lay_.colind[t]], t);
      std::sort(row.begin(), row.end());
      for (const auto& e : row) {
        pcol.push_back(e.first);
        psrc_.push_back(e.second);
      }
      prow[i + 1] = (unsigned)pcol.size();
    }
    check(dfm_mat_create(ctx_->get(), N, lay_.b, DFM_REAL, prow.data(), pcol.data(), &pmat_), "SetOrdering");
    for (void** d : {&d_n2o_, &d_o2n_}) check(dfm_buf_alloc(ctx_->get(), sizeof(unsigned) * std::max(N, 1u), d), "SetOrdering");
    check(dfm_buf_copy(ctx_->get(), d_n2o_, n2o_.data(), sizeof(unsigned) * N, DFM_H2D), "SetOrdering");
    check(dfm_buf_copy(ctx_->get(), d_o2n_, o2n.data(), sizeof(unsigned) * N, DFM_H2D), "SetOrdering");
  }

  Context* ctx_;
  dfm_mat mat_ = nullptr;
  dfm_ilu ilu_ = nullptr;
  std::vector<std::pair<int, int>> lev_in_;
  std::vector<unsigned int> fill_blk_;  // SetFillBlk: block rows of segment 0 with unlimited fill
  int lev_ = 0;
  std::vector<int> order_;             // SetOrdering: new -> old block row (empty: off)
  dfm_mat pmat_ = nullptr;             // the renumbered matrix the ordered ILU(0) factors
  std::vector<unsigned> n2o_, psrc_;   // new -> old row; source slot of each renumbered block
  void* d_n2o_ = nullptr;              // device copies of new -> old and old -> new
  void* d_o2n_ = nullptr;
  detail::Layout lay_;
  std::unique_ptr<DeviceVector> tmp_r_, tmp_z_, tmp_o1_, tmp_o2_;
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
    const detail::Layout& L = prec.layout();
    if (ls.GetNLinSysSeg() != L.nseg) throw Error(DFM_ERR_INVALID, "CLinearSystemGPU");
    for (unsigned i = 0; i < L.nseg; i++)
      if ((size_t)ls.GetVector(-1, i).NBlk() * L.len[i] != L.dof0[i + 1] - L.dof0[i])
        throw Error(DFM_ERR_INVALID, "CLinearSystemGPU");
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
    std::vector<double> h(n_);
    prec_->layout().gather(*ls_, -1, h.data());
    r_.upload(h.data());
    prec_->layout().gather(*ls_, -2, h.data());
    u_.upload(h.data());
  }
  void SyncToHost() {
    std::vector<double> h(n_);
    r_.download(h.data());
    prec_->layout().scatter(*ls_, -1, h.data());
    u_.download(h.data());
    prec_->layout().scatter(*ls_, -2, h.data());
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
  if (M.ordered()) {  // the reference's own driver over the device operations (renumbering in SolvePrecond)
    const bool ok = LsSol::Solve_PCG(conv_ratio, iteration, g);
    g.SyncToHost();
    return ok;
  }
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
  if (M.ordered()) {
    const bool ok = LsSol::Solve_PBiCGSTAB(conv_ratio, num_iter, g);
    g.SyncToHost();
    return ok;
  }
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
