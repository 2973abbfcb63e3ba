// ILU(0) on the device: numeric factorisation and the two triangular sweeps,
// scheduled by the level sets of the reference's natural ordering.
//
// Reference: CMatDiaFrac_BlkCrs (src/matvec/matdiafrac_blkcrs.cpp):
//   DoILUDecomp :769-1102  row i -= L_ik (D^-1 U)_kj over the pattern, k ascending;
//                          D_i <- D_i^-1 (closed forms); U_i <- D_i^-1 U_i
//   ForwardSubstitution :332-503   y_i = D_i^-1 (r_i - sum_{j<i} L_ij y_j)
//   BackwardSubstitution :505-663  z_i = y_i - sum_{j>i} (D^-1 U)_ij z_j
// complex twin: CZMatDiaFrac_BlkCrs (src/matvec/zmatdiafrac_blkcrs.cpp:116-261).
//
// Scheduling.  Rows are processed in level order (order_f / order_b: rows
// sorted by level, ascending row inside a level).  Two sweep schedules:
//  * sync-free (mode 1): a persistent, co-resident grid; worker w takes level-
//    order positions w, w+W, ...; a row waits only for the rows it reads, by
//    polling their outputs, which start out as a NaN sentinel.  Because every
//    dependency sits at an earlier position, and a worker's earlier positions
//    are all smaller, every wait ends (induction on the position).
//  * one CTA with level barriers (mode 2): for long dependency chains with few
//    rows per level the whole sweep runs on one SM with __syncthreads between
//    levels, so a level costs a CTA barrier instead of a trip through L2.
// The factorisation uses the sync-free schedule with per-row completion epochs
// and reproduces the reference's arithmetic exactly (no FMA contraction).
#include <algorithm>

#include "dfm_internal.h"

namespace dfm {

// ------------------------------------------------------------------ waits
DFM_DEVINL int ld_status(const DevStatus* st) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(&st->code) : "memory");
  return v;
}

// Back-off between polls (ns) of a sync-free sweep; 0 spins without sleeping.
// Thousands of waiting lanes polling L2 back to back starve the stores that
// would release them, so waiting lanes sleep briefly between polls.
__constant__ unsigned c_poll_sleep_ns = 0;

template <typename T>
DFM_DEVINL T poll_value(const T* p, DevStatus* st, uint64_t wait_ns, int where) {
  T v = ld_relaxed(p);
  if (!Sent<T>::is(v)) return v;
  SpinGuard g(wait_ns);
  const unsigned nap = c_poll_sleep_ns;
  for (;;) {
    if (nap) __nanosleep(nap);
    v = ld_relaxed(p);
    if (!Sent<T>::is(v)) return v;
    if (g.expired() || ((g.n & 1023u) == 0 && ld_status(st) != 0)) {
      raise_error(st, DFM_WAIT_TIMEOUT, where);
      return v;
    }
  }
}

// The K consecutive values of one row (a b x b block's operand, or re/im):
// all K are read before any is checked and the missing ones are re-read
// together, so a row costs one L2 round trip per pass, not one per value.
template <int K, typename T>
DFM_DEVINL void poll_values(const T* p, T* v, DevStatus* st, uint64_t wait_ns, int where) {
#pragma unroll
  for (int c = 0; c < K; c++) v[c] = ld_relaxed(p + c);
  auto missing = [&]() {
    bool m = false;
#pragma unroll
    for (int c = 0; c < K; c++) m |= Sent<T>::is(v[c]);
    return m;
  };
  if (!missing()) return;
  SpinGuard g(wait_ns);
  const unsigned nap = c_poll_sleep_ns;
  for (;;) {
    if (nap) __nanosleep(nap);
#pragma unroll
    for (int c = 0; c < K; c++)
      if (Sent<T>::is(v[c])) v[c] = ld_relaxed(p + c);
    if (!missing()) return;
    if (g.expired() || ((g.n & 1023u) == 0 && ld_status(st) != 0)) {
      raise_error(st, DFM_WAIT_TIMEOUT, where);
      return;
    }
  }
}

DFM_DEVINL void wait_epoch(const unsigned* flag, unsigned epoch, DevStatus* st, uint64_t wait_ns, int where) {
  if (ld_acquire_u32(flag) == epoch) return;
  SpinGuard g(wait_ns);
  for (;;) {
    if (ld_acquire_u32(flag) == epoch) return;
    if (g.expired() || ((g.n & 1023u) == 0 && ld_status(st) != 0)) {
      raise_error(st, DFM_WAIT_TIMEOUT, where);
      return;
    }
  }
}

// --------------------------------------------------- numeric factorisation
DFM_DEVINL long find_slot(const unsigned* colind, unsigned s0, unsigned s1, unsigned j) {
  while (s0 < s1) {  // strictly ascending columns
    const unsigned m = (s0 + s1) >> 1;
    const unsigned c = __ldg(colind + m);
    if (c == j) return (long)m;
    if (c < j) s0 = m + 1; else s1 = m;
  }
  return -1;
}

// D <- D^-1 with the reference's closed forms; returns false if singular.
template <int B>
DFM_DEVINL bool invert_pivot(double* d);
template <>
DFM_DEVINL bool invert_pivot<1>(double* d) {
  const double v = d[0];
  if (fabs(v) > 1.0e-30) { d[0] = __ddiv_rn(1.0, v); return true; }
  return false;
}
template <>
DFM_DEVINL bool invert_pivot<2>(double* d) {
  const double det = sub_rn(mul_rn(d[0], d[3]), mul_rn(d[1], d[2]));
  if (!(fabs(det) > 1.0e-30)) return false;
  const double inv = __ddiv_rn(1.0, det);
  const double t = d[0];
  d[0] = mul_rn(inv, d[3]);
  d[1] = mul_rn(-inv, d[1]);
  d[2] = mul_rn(-inv, d[2]);
  d[3] = mul_rn(inv, t);
  return true;
}
DFM_DEVINL double det3(const double* a) {
  double v = mul_rn(mul_rn(a[0], a[4]), a[8]);
  v = add_rn(v, mul_rn(mul_rn(a[3], a[7]), a[2]));
  v = add_rn(v, mul_rn(mul_rn(a[6], a[1]), a[5]));
  v = sub_rn(v, mul_rn(mul_rn(a[0], a[7]), a[5]));
  v = sub_rn(v, mul_rn(mul_rn(a[6], a[4]), a[2]));
  v = sub_rn(v, mul_rn(mul_rn(a[3], a[1]), a[8]));
  return v;
}
template <>
DFM_DEVINL bool invert_pivot<3>(double* a) {
  const double det = det3(a);
  if (!(fabs(det) > 1.0e-30)) return false;
  const double inv = __ddiv_rn(1.0, det);
  double t[9];
#pragma unroll
  for (int q = 0; q < 9; q++) t[q] = a[q];
  a[0] = mul_rn(inv, sub_rn(mul_rn(t[4], t[8]), mul_rn(t[5], t[7])));
  a[1] = mul_rn(inv, sub_rn(mul_rn(t[2], t[7]), mul_rn(t[1], t[8])));
  a[2] = mul_rn(inv, sub_rn(mul_rn(t[1], t[5]), mul_rn(t[2], t[4])));
  a[3] = mul_rn(inv, sub_rn(mul_rn(t[5], t[6]), mul_rn(t[3], t[8])));
  a[4] = mul_rn(inv, sub_rn(mul_rn(t[0], t[8]), mul_rn(t[2], t[6])));
  a[5] = mul_rn(inv, sub_rn(mul_rn(t[2], t[3]), mul_rn(t[0], t[5])));
  a[6] = mul_rn(inv, sub_rn(mul_rn(t[3], t[7]), mul_rn(t[4], t[6])));
  a[7] = mul_rn(inv, sub_rn(mul_rn(t[1], t[6]), mul_rn(t[0], t[7])));
  a[8] = mul_rn(inv, sub_rn(mul_rn(t[0], t[4]), mul_rn(t[1], t[3])));
  return true;
}

// One warp per row.  Values are read/written with .cg (L2) accesses: another
// SM may have finished a row whose bytes share an L1 line this SM cached.
template <int B>
__global__ void __launch_bounds__(256)
k_ilu0_factor(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
              const unsigned* __restrict__ diaind, const unsigned* __restrict__ order, double* fdiag,
              double* foff, unsigned* flags, unsigned epoch, DevStatus* st, uint64_t wait_ns) {
  constexpr int BB = B * B;
  const int lane = threadIdx.x & 31;
  const unsigned w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nw = (gridDim.x * blockDim.x) >> 5;
  for (unsigned p = w0; p < N; p += nw) {
    const unsigned i = __ldg(order + p);
    const unsigned s0 = __ldg(rowptr + i), s1 = __ldg(rowptr + i + 1), di = __ldg(diaind + i);
    for (unsigned ik = s0; ik < di; ik++) {
      const unsigned k = __ldg(colind + ik);
      wait_epoch(flags + k, epoch, st, wait_ns, 1);  // every lane acquires row k
      __syncwarp();
      const unsigned u0 = __ldg(diaind + k), u1 = __ldg(rowptr + k + 1);
      const unsigned nq = (u1 - u0) * BB;
      for (unsigned q = lane; q < nq; q += 32) {
        const unsigned kj = u0 + q / BB;
        const int e = q % BB, r = e / B, c = e % B;
        const unsigned j = __ldg(colind + kj);
        double* tgt;
        if (j == i) tgt = fdiag + (size_t)i * BB + e;
        else {
          const long t = find_slot(colind, s0, s1, j);
          if (t < 0) continue;  // no fill-in in ILU(0)
          tgt = foff + (size_t)t * BB + e;
        }
        const double* l = foff + (size_t)ik * BB + r * B;
        const double* u = foff + (size_t)kj * BB + c;
        double acc = mul_rn(__ldcg(l), __ldcg(u));
#pragma unroll
        for (int m = 1; m < B; m++) acc = add_rn(acc, mul_rn(__ldcg(l + m), __ldcg(u + m * B)));
        __stcg(tgt, sub_rn(__ldcg(tgt), acc));
      }
      __syncwarp();
    }
    __shared__ double s_d[8][BB];
    double* d = s_d[threadIdx.x >> 5];
    if (lane < BB) d[lane] = __ldcg(fdiag + (size_t)i * BB + lane);
    __syncwarp();
    if (lane == 0) {
      if (!invert_pivot<B>(d)) atomicAdd(&st->nsing, 1u);
    }
    __syncwarp();
    if (lane < BB) __stcg(fdiag + (size_t)i * BB + lane, d[lane]);
    for (unsigned ij = di + lane; ij < s1; ij += 32) {
      double* u = foff + (size_t)ij * BB;
      double t[BB];
#pragma unroll
      for (int q = 0; q < BB; q++) t[q] = __ldcg(u + q);
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int c = 0; c < B; c++) {
          double v = mul_rn(d[r * B], t[c]);
#pragma unroll
          for (int m = 1; m < B; m++) v = add_rn(v, mul_rn(d[r * B + m], t[m * B + c]));
          __stcg(u + r * B + c, v);
        }
    }
    __syncwarp();
    __threadfence();
    if (lane == 0) st_release_u32(flags + i, epoch);
  }
}

// complex b = 1 (CZMatDiaFrac_BlkCrs::DoILUDecomp)
DFM_DEVINL double2 zmul_rn(double2 a, double2 b) {
  return make_double2(sub_rn(mul_rn(a.x, b.x), mul_rn(a.y, b.y)), add_rn(mul_rn(a.x, b.y), mul_rn(a.y, b.x)));
}
__global__ void __launch_bounds__(256)
k_zilu0_factor(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
               const unsigned* __restrict__ diaind, const unsigned* __restrict__ order, double2* fdiag,
               double2* foff, unsigned* flags, unsigned epoch, DevStatus* st, uint64_t wait_ns) {
  const int lane = threadIdx.x & 31;
  const unsigned w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nw = (gridDim.x * blockDim.x) >> 5;
  for (unsigned p = w0; p < N; p += nw) {
    const unsigned i = __ldg(order + p);
    const unsigned s0 = __ldg(rowptr + i), s1 = __ldg(rowptr + i + 1), di = __ldg(diaind + i);
    for (unsigned ik = s0; ik < di; ik++) {
      const unsigned k = __ldg(colind + ik);
      wait_epoch(flags + k, epoch, st, wait_ns, 2);
      __syncwarp();
      const double2 ikv = __ldcg(foff + ik);
      const unsigned u0 = __ldg(diaind + k), u1 = __ldg(rowptr + k + 1);
      for (unsigned kj = u0 + lane; kj < u1; kj += 32) {
        const unsigned j = __ldg(colind + kj);
        double2* tgt;
        if (j == i) tgt = fdiag + i;
        else {
          const long t = find_slot(colind, s0, s1, j);
          if (t < 0) continue;
          tgt = foff + t;
        }
        const double2 pr = zmul_rn(ikv, __ldcg(foff + kj));
        const double2 a = __ldcg(tgt);
        __stcg(tgt, make_double2(sub_rn(a.x, pr.x), sub_rn(a.y, pr.y)));
      }
      __syncwarp();
    }
    __shared__ double2 s_inv[8];
    if (lane == 0) {
      const double2 piv = __ldcg(fdiag + i);
      const double n2 = add_rn(mul_rn(piv.x, piv.x), mul_rn(piv.y, piv.y));
      if (n2 < 1.0e-20) atomicAdd(&st->nsing, 1u);  // the reference stops for a key press here
      const double fact = __ddiv_rn(1.0, n2);
      const double2 inv = make_double2(mul_rn(fact, piv.x), mul_rn(-fact, piv.y));
      __stcg(fdiag + i, inv);
      s_inv[threadIdx.x >> 5] = inv;
    }
    __syncwarp();
    const double2 inv = s_inv[threadIdx.x >> 5];
    for (unsigned ij = di + lane; ij < s1; ij += 32) __stcg(foff + ij, zmul_rn(__ldcg(foff + ij), inv));
    __syncwarp();
    __threadfence();
    if (lane == 0) st_release_u32(flags + i, epoch);
  }
}

// ------------------------------------------------------------ sweep helpers
// Convergence guard run at the top of the forward sweep inside a Krylov
// iteration: every block reduces the (r, r) partials of the previous kernel
// and returns early once |r|^2/|r0|^2 < tol^2 (block 0 records the result).
DFM_DEVINL bool converged_guard(KrylovScalars* sc, const double* rr_part, int nparts) {
  if (!sc) return false;
  if (block_flag(&sc->done)) return true;
  if (!rr_part) return false;  // solver checks convergence elsewhere
  const double rr = reduce_partials(rr_part, nparts);
  if (rr * sc->inv0 < sc->tol2) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      sc->conv = sqrt(rr * sc->inv0);
      sc->conv_it = sc->it;
      sc->done = sc->conv_code;
    }
    return true;
  }
  return false;
}

// Real b x b block row: acc_r = sum_c m[r*B+c] * v[c]
template <int B, typename TV, typename TX>
DFM_DEVINL void block_mv(double* acc, const TV* m, const TX* v) {
#pragma unroll
  for (int r = 0; r < B; r++)
#pragma unroll
    for (int c = 0; c < B; c++) acc[r] += (double)m[r * B + c] * (double)v[c];
}

// ------------------------------------------------------- sync-free sweeps
// FWD: out_i = D_i^-1 (in_i - sum_{L} m * out_j);  BWD: out_i = in_i - sum_{U} m * out_j.
// DOT (BWD only): partial of rdot . out, for the Krylov (r, z).
template <int B, int LPR, typename TV, typename TX, bool FWD, bool DOT>
__global__ void __launch_bounds__(256)
k_sweep_syncfree(unsigned N, const unsigned* __restrict__ order, const unsigned* __restrict__ rowptr,
                 const unsigned* __restrict__ colind, const unsigned* __restrict__ diaind,
                 const double* __restrict__ fdiag, const TV* __restrict__ foff, const TX* __restrict__ in,
                 TX* out, const TX* __restrict__ rdot, double* part, KrylovScalars* sc,
                 const double* rr_part, int rr_nparts, DevStatus* st, uint64_t wait_ns) {
  if (FWD) {
    if (converged_guard(sc, rr_part, rr_nparts)) return;
  } else if (sc && block_flag(&sc->done)) {
    return;
  }
  constexpr int BB = B * B;
  const int lane = threadIdx.x % LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  const unsigned g0 = (blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const unsigned ng = gridDim.x * blockDim.x / LPR;
  double dacc = 0.0;
  for (unsigned p = g0; p < N; p += ng) {
    const unsigned i = __ldg(order + p);
    unsigned s0, s1;
    if (FWD) { s0 = __ldg(rowptr + i); s1 = __ldg(diaind + i); }
    else { s0 = __ldg(diaind + i); s1 = __ldg(rowptr + i + 1); }
    double acc[B];
#pragma unroll
    for (int r = 0; r < B; r++) acc[r] = 0.0;
    for (unsigned s = s0 + lane; s < s1; s += LPR) {
      const unsigned col = __ldg(colind + s);
      TV mv[BB];
#pragma unroll
      for (int e = 0; e < BB; e++) mv[e] = __ldcs(foff + (size_t)s * BB + e);
      TX xv[B];
      poll_values<B>(out + (size_t)col * B, xv, st, wait_ns, FWD ? 3 : 4);
      block_mv<B>(acc, mv, xv);
    }
#pragma unroll
    for (int r = 0; r < B; r++)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
    if (lane == 0) {
      double t[B];
#pragma unroll
      for (int r = 0; r < B; r++) t[r] = (double)in[(size_t)i * B + r] - acc[r];
      double o[B];
      if (FWD) {
        const double* d = fdiag + (size_t)i * BB;
#pragma unroll
        for (int r = 0; r < B; r++) {
          o[r] = 0.0;
#pragma unroll
          for (int c = 0; c < B; c++) o[r] += d[r * B + c] * t[c];
        }
      } else {
#pragma unroll
        for (int r = 0; r < B; r++) o[r] = t[r];
      }
#pragma unroll
      for (int r = 0; r < B; r++) {
        const TX v = (TX)o[r];
        st_relaxed(out + (size_t)i * B + r, v);
        if (DOT) dacc += (double)rdot[(size_t)i * B + r] * (double)v;
      }
    }
  }
  if (DOT) block_partial<256>(dacc, part);
}

// complex b = 1
template <int LPR, bool FWD, bool DOT, typename TV = double2>
__global__ void __launch_bounds__(256)
k_zsweep_syncfree(unsigned N, const unsigned* __restrict__ order, const unsigned* __restrict__ rowptr,
                  const unsigned* __restrict__ colind, const unsigned* __restrict__ diaind,
                  const double2* __restrict__ fdiag, const TV* __restrict__ foff,
                  const double2* __restrict__ in, double2* out, const double2* __restrict__ rdot, double* part,
                  KrylovScalars* sc, const double* rr_part, int rr_nparts, DevStatus* st, uint64_t wait_ns) {
  if (FWD) {
    if (converged_guard(sc, rr_part, rr_nparts)) return;
  } else if (sc && block_flag(&sc->done)) {
    return;
  }
  const int lane = threadIdx.x % LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  const unsigned g0 = (blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const unsigned ng = gridDim.x * blockDim.x / LPR;
  double dre = 0.0, dim = 0.0;
  double* o64 = reinterpret_cast<double*>(out);
  for (unsigned p = g0; p < N; p += ng) {
    const unsigned i = __ldg(order + p);
    unsigned s0, s1;
    if (FWD) { s0 = __ldg(rowptr + i); s1 = __ldg(diaind + i); }
    else { s0 = __ldg(diaind + i); s1 = __ldg(rowptr + i + 1); }
    double re = 0.0, im = 0.0;
    for (unsigned s = s0 + lane; s < s1; s += LPR) {
      const unsigned col = __ldg(colind + s);
      const TV mv = __ldcs(foff + s);
      const double2 m = make_double2((double)mv.x, (double)mv.y);
      double xz[2];
      poll_values<2>(o64 + 2 * (size_t)col, xz, st, wait_ns, FWD ? 5 : 6);
      const double xr = xz[0], xi = xz[1];
      re += m.x * xr - m.y * xi;
      im += m.x * xi + m.y * xr;
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      re += __shfl_xor_sync(gmask, re, o);
      im += __shfl_xor_sync(gmask, im, o);
    }
    if (lane == 0) {
      const double2 v_in = in[i];
      double tr = v_in.x - re, ti = v_in.y - im;
      if (FWD) {
        const double2 d = fdiag[i];
        const double a = d.x * tr - d.y * ti, b = d.x * ti + d.y * tr;
        tr = a; ti = b;
      }
      st_relaxed(o64 + 2 * (size_t)i, tr);
      st_relaxed(o64 + 2 * (size_t)i + 1, ti);
      if (DOT) {  // unconjugated r^T z
        const double2 rv = rdot[i];
        dre += rv.x * tr - rv.y * ti;
        dim += rv.x * ti + rv.y * tr;
      }
    }
  }
  if (DOT) {
    block_partial<256>(dre, part);
    block_partial<256>(dim, part + kMaxBlocks);
  }
}

// ------------------------------------------------- single-CTA level sweeps
template <int B, int LPR, typename TV, typename TX, bool FWD, bool DOT>
__global__ void __launch_bounds__(1024)
k_sweep_cta(unsigned nlev, const unsigned* __restrict__ lvl, const unsigned* __restrict__ order,
            const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
            const unsigned* __restrict__ diaind, const double* __restrict__ fdiag, const TV* __restrict__ foff,
            const TX* __restrict__ in, TX* out, const TX* __restrict__ rdot, double* part, KrylovScalars* sc,
            const double* rr_part, int rr_nparts) {
  if (FWD) {
    if (converged_guard(sc, rr_part, rr_nparts)) return;
  } else if (sc && block_flag(&sc->done)) {
    return;
  }
  constexpr int BB = B * B;
  const int lane = threadIdx.x % LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  const unsigned g = threadIdx.x / LPR, ng = blockDim.x / LPR;
  double dacc = 0.0;
  for (unsigned l = 0; l < nlev; l++) {
    const unsigned p0 = __ldg(lvl + l), p1 = __ldg(lvl + l + 1);
    for (unsigned pb = p0; pb < p1; pb += ng) {
      const unsigned p = pb + g;
      const bool valid = p < p1;
      unsigned i = 0, s0 = 0, s1 = 0;
      if (valid) {
        i = __ldg(order + p);
        if (FWD) { s0 = __ldg(rowptr + i); s1 = __ldg(diaind + i); }
        else { s0 = __ldg(diaind + i); s1 = __ldg(rowptr + i + 1); }
      }
      double acc[B];
#pragma unroll
      for (int r = 0; r < B; r++) acc[r] = 0.0;
      for (unsigned s = s0 + lane; s < s1; s += LPR) {
        const unsigned col = __ldg(colind + s);
        TV mv[BB];
#pragma unroll
        for (int e = 0; e < BB; e++) mv[e] = __ldg(foff + (size_t)s * BB + e);
        TX xv[B];
#pragma unroll
        for (int c = 0; c < B; c++) xv[c] = out[(size_t)col * B + c];
        block_mv<B>(acc, mv, xv);
      }
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
      if (valid && lane == 0) {
        double t[B];
#pragma unroll
        for (int r = 0; r < B; r++) t[r] = (double)in[(size_t)i * B + r] - acc[r];
#pragma unroll
        for (int r = 0; r < B; r++) {
          double o = t[r];
          if (FWD) {
            const double* d = fdiag + (size_t)i * BB + r * B;
            o = 0.0;
#pragma unroll
            for (int c = 0; c < B; c++) o += d[c] * t[c];
          }
          const TX v = (TX)o;
          out[(size_t)i * B + r] = v;
          if (DOT) dacc += (double)rdot[(size_t)i * B + r] * (double)v;
        }
      }
    }
    __syncthreads();
  }
  if (DOT) block_partial<1024>(dacc, part);
}

template <int LPR, bool FWD, bool DOT, typename TV = double2>
__global__ void __launch_bounds__(1024)
k_zsweep_cta(unsigned nlev, const unsigned* __restrict__ lvl, const unsigned* __restrict__ order,
             const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
             const unsigned* __restrict__ diaind, const double2* __restrict__ fdiag,
             const TV* __restrict__ foff, const double2* __restrict__ in, double2* out,
             const double2* __restrict__ rdot, double* part, KrylovScalars* sc, const double* rr_part,
             int rr_nparts) {
  if (FWD) {
    if (converged_guard(sc, rr_part, rr_nparts)) return;
  } else if (sc && block_flag(&sc->done)) {
    return;
  }
  const int lane = threadIdx.x % LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  const unsigned g = threadIdx.x / LPR, ng = blockDim.x / LPR;
  double dre = 0.0, dim = 0.0;
  for (unsigned l = 0; l < nlev; l++) {
    const unsigned p0 = __ldg(lvl + l), p1 = __ldg(lvl + l + 1);
    for (unsigned pb = p0; pb < p1; pb += ng) {
      const unsigned p = pb + g;
      const bool valid = p < p1;
      unsigned i = 0, s0 = 0, s1 = 0;
      if (valid) {
        i = __ldg(order + p);
        if (FWD) { s0 = __ldg(rowptr + i); s1 = __ldg(diaind + i); }
        else { s0 = __ldg(diaind + i); s1 = __ldg(rowptr + i + 1); }
      }
      double re = 0.0, im = 0.0;
      for (unsigned s = s0 + lane; s < s1; s += LPR) {
        const TV mv = __ldg(foff + s);
        const double2 m = make_double2((double)mv.x, (double)mv.y);
        const double2 xv = out[__ldg(colind + s)];
        re += m.x * xv.x - m.y * xv.y;
        im += m.x * xv.y + m.y * xv.x;
      }
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) {
        re += __shfl_xor_sync(gmask, re, o);
        im += __shfl_xor_sync(gmask, im, o);
      }
      if (valid && lane == 0) {
        const double2 v_in = in[i];
        double tr = v_in.x - re, ti = v_in.y - im;
        if (FWD) {
          const double2 d = fdiag[i];
          const double a = d.x * tr - d.y * ti, b = d.x * ti + d.y * tr;
          tr = a; ti = b;
        }
        out[i] = make_double2(tr, ti);
        if (DOT) {
          const double2 rv = rdot[i];
          dre += rv.x * tr - rv.y * ti;
          dim += rv.x * ti + rv.y * tr;
        }
      }
    }
    __syncthreads();
  }
  if (DOT) {
    block_partial<1024>(dre, part);
    block_partial<1024>(dim, part + kMaxBlocks);
  }
}

// -------------------------------------------------------------- utilities
__global__ void k_fill_sentinel(double* v, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    v[k] = Sent<double>::value();
}

__global__ void k_wait_selftest(const double* never, DevStatus* st, uint64_t wait_ns) {
  (void)poll_value(never, st, wait_ns, 99);
}

// ---------------------------------------------------------------- launches
static int coop_grid(const void* fn, int threads, int nsm, int cap) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0) != cudaSuccess) return -1;
  per_sm = std::max(1, std::min(per_sm, 8));
  return std::max(1, std::min(per_sm * nsm, cap));
}

// Co-resident persistent launch (cooperative attribute: all blocks resident).
template <typename... KArgs, typename... Args>
static cudaError_t launch_coop(void (*fn)(KArgs...), int grid, int threads, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, fn, static_cast<KArgs>(args)...);
}

int ilu_factor_launch(dfm_ilu M, dfm_mat A) {
  dfm_ctx c = M->ctx;
  cudaStream_t s = c->stream;
  const size_t vw = M->vw();
  DFM_CUDA_TRY(cudaMemcpyAsync(M->d_fdiag, A->d_diag, sizeof(double) * vw * M->N, cudaMemcpyDeviceToDevice, s));
  if (M->d_fillmap) {  // ILU(k): A's blocks into the filled pattern, zero elsewhere (SetValue_Initialize)
    const int rc = ilu_fill_values(M, A);
    if (rc) return rc;
  } else if (M->ncrs) {
    DFM_CUDA_TRY(cudaMemcpyAsync(M->d_foff, A->d_off, sizeof(double) * vw * M->ncrs, cudaMemcpyDeviceToDevice, s));
  }
  DFM_CUDA_TRY(cudaMemsetAsync(&c->d_status->nsing, 0, sizeof(unsigned), s));
  M->plan_f.stale = true;  // packed sweep values are re-gathered on next use
  M->plan_b.stale = true;
  M->plan32_f.stale = true;
  M->plan32_b.stale = true;
  M->epoch++;
  if (M->epoch == 0) {  // wrapped: clear the epochs
    DFM_CUDA_TRY(cudaMemsetAsync(M->d_flags, 0, sizeof(unsigned) * M->N, s));
    M->epoch = 1;
  }
  if (M->N == 0) return DFM_OK;
  cudaError_t e;
  if (M->vt == DFM_COMPLEX) {
    const int grid = coop_grid((const void*)k_zilu0_factor, 256, c->nsm, (M->N + 7) / 8);
    e = launch_coop(k_zilu0_factor, grid, 256, s, M->N, (const unsigned*)M->A->d_rowptr,
                    (const unsigned*)M->A->d_colind, (const unsigned*)M->d_diaind, (const unsigned*)M->d_order_f,
                    reinterpret_cast<double2*>(M->d_fdiag), reinterpret_cast<double2*>(M->d_foff), M->d_flags,
                    M->epoch, c->d_status, (uint64_t)c->wait_ns);
  } else {
#define DFM_ILU_CASE(BV)                                                                                      \
  case BV: {                                                                                                  \
    const int grid = coop_grid((const void*)k_ilu0_factor<BV>, 256, c->nsm, (M->N + 7) / 8);                  \
    e = launch_coop(k_ilu0_factor<BV>, grid, 256, s, M->N, (const unsigned*)M->A->d_rowptr,                   \
                    (const unsigned*)M->A->d_colind, (const unsigned*)M->d_diaind,                           \
                    (const unsigned*)M->d_order_f, M->d_fdiag, M->d_foff, M->d_flags, M->epoch, c->d_status, \
                    (uint64_t)c->wait_ns);                                                                    \
  } break;
    switch (M->b) {
      DFM_ILU_CASE(1)
      DFM_ILU_CASE(2)
      DFM_ILU_CASE(3)
      default: return DFM_ERR_UNSUPPORTED;
    }
#undef DFM_ILU_CASE
  }
  DFM_CUDA_TRY(e);
  return DFM_OK;
}

int ilu_fill_sentinel(dfm_ilu M, double* v, size_t n) {
  if (n == 0) return DFM_OK;
  const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)M->ctx->nsm * 8);
  k_fill_sentinel<<<grid, 256, 0, M->ctx->stream>>>(v, n);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

static int sweep_lanes(dfm_ilu M) { return M->b == 3 ? 16 : 8; }

template <int B, int LPR, bool FWD, bool DOT>
static const void* syncfree_fn() { return (const void*)k_sweep_syncfree<B, LPR, double, double, FWD, DOT>; }

int sweep_grid(dfm_ilu M, int sweep) {
  if (sweep == 2) return 1;
  if (sweep == 3) return std::max(1, M->plan_b.G);  // the backward sweep writes the (r, z) partials
  // every sync-free kernel here has the same resource profile class; size by the B=3 bwd+dot one
  const void* fn = (M->vt == DFM_COMPLEX) ? (const void*)k_zsweep_syncfree<8, false, true>
                                          : syncfree_fn<3, 16, false, true>();
  const int lpr = sweep_lanes(M);
  const int rows_per_block = 256 / lpr;
  int cap = (int)std::min<unsigned>((M->N + rows_per_block - 1) / rows_per_block, kMaxBlocks);
  if (M->sweep_blocks > 0) cap = std::min(cap, M->sweep_blocks);
  const int g = coop_grid(fn, 256, M->ctx->nsm, cap);
  return std::max(1, g);
}

int set_poll_sleep(unsigned ns) {
  DFM_CUDA_TRY(cudaMemcpyToSymbol(c_poll_sleep_ns, &ns, sizeof(ns)));
  return DFM_OK;
}

template <int B, int LPR, bool FWD, typename TV>
static cudaError_t sweep_real_tv(dfm_ilu M, const TV* foff, int sweep, const double* in, double* out,
                                 const double* rdot, double* part, KrylovScalars* sc, const double* rr_part,
                                 int rr_n) {
  dfm_ctx c = M->ctx;
  const unsigned* order = FWD ? M->d_order_f : M->d_order_b;
  if (sweep == 2) {
    const unsigned* lvl = FWD ? M->d_lvl_f : M->d_lvl_b;
    const unsigned nlev = FWD ? M->nlev_f : M->nlev_b;
    if (part)
      k_sweep_cta<B, LPR, TV, double, FWD, true><<<1, 1024, 0, c->stream>>>(
          nlev, lvl, order, M->A->d_rowptr, M->A->d_colind, M->d_diaind, M->d_fdiag, foff, in, out, rdot, part, sc,
          rr_part, rr_n);
    else
      k_sweep_cta<B, LPR, TV, double, FWD, false><<<1, 1024, 0, c->stream>>>(
          nlev, lvl, order, M->A->d_rowptr, M->A->d_colind, M->d_diaind, M->d_fdiag, foff, in, out, rdot, nullptr,
          sc, rr_part, rr_n);
    return cudaGetLastError();
  }
  const int grid = sweep_grid(M, 1);
  if (part)
    return launch_coop(k_sweep_syncfree<B, LPR, TV, double, FWD, true>, grid, 256, c->stream, M->N, order,
                       (const unsigned*)M->A->d_rowptr, (const unsigned*)M->A->d_colind,
                       (const unsigned*)M->d_diaind, (const double*)M->d_fdiag, foff, in, out, rdot, part, sc,
                       rr_part, rr_n, c->d_status, (uint64_t)c->wait_ns);
  return launch_coop(k_sweep_syncfree<B, LPR, TV, double, FWD, false>, grid, 256, c->stream, M->N, order,
                     (const unsigned*)M->A->d_rowptr, (const unsigned*)M->A->d_colind,
                     (const unsigned*)M->d_diaind, (const double*)M->d_fdiag, foff, in, out, rdot, (double*)nullptr,
                     sc, rr_part, rr_n, c->d_status, (uint64_t)c->wait_ns);
}

template <int B, int LPR, bool FWD>
static cudaError_t sweep_real(dfm_ilu M, int sweep, const double* in, double* out, const double* rdot,
                              double* part, KrylovScalars* sc, const double* rr_part, int rr_n, bool f32) {
  if (f32)
    return sweep_real_tv<B, LPR, FWD, float>(M, M->d_foff32, sweep, in, out, rdot, part, sc, rr_part, rr_n);
  return sweep_real_tv<B, LPR, FWD, double>(M, M->d_foff, sweep, in, out, rdot, part, sc, rr_part, rr_n);
}

template <int LPR, bool FWD, typename TV>
static cudaError_t sweep_cplx_tv(dfm_ilu M, const TV* fo, int sweep, const double* in, double* out,
                                 const double* rdot, double* part, KrylovScalars* sc, const double* rr_part,
                                 int rr_n) {
  dfm_ctx c = M->ctx;
  const unsigned* order = FWD ? M->d_order_f : M->d_order_b;
  auto* fd = reinterpret_cast<const double2*>(M->d_fdiag);
  auto* vi = reinterpret_cast<const double2*>(in);
  auto* vo = reinterpret_cast<double2*>(out);
  auto* rd = reinterpret_cast<const double2*>(rdot);
  if (sweep == 2) {
    const unsigned* lvl = FWD ? M->d_lvl_f : M->d_lvl_b;
    const unsigned nlev = FWD ? M->nlev_f : M->nlev_b;
    if (part)
      k_zsweep_cta<LPR, FWD, true, TV><<<1, 1024, 0, c->stream>>>(nlev, lvl, order, M->A->d_rowptr,
                                                                  M->A->d_colind, M->d_diaind, fd, fo, vi, vo, rd,
                                                                  part, sc, rr_part, rr_n);
    else
      k_zsweep_cta<LPR, FWD, false, TV><<<1, 1024, 0, c->stream>>>(nlev, lvl, order, M->A->d_rowptr,
                                                                   M->A->d_colind, M->d_diaind, fd, fo, vi, vo, rd,
                                                                   nullptr, sc, rr_part, rr_n);
    return cudaGetLastError();
  }
  const int grid = sweep_grid(M, 1);
  if (part)
    return launch_coop(k_zsweep_syncfree<LPR, FWD, true, TV>, grid, 256, c->stream, M->N, order,
                       (const unsigned*)M->A->d_rowptr, (const unsigned*)M->A->d_colind,
                       (const unsigned*)M->d_diaind, fd, fo, vi, vo, rd, part, sc, rr_part, rr_n, c->d_status,
                       (uint64_t)c->wait_ns);
  return launch_coop(k_zsweep_syncfree<LPR, FWD, false, TV>, grid, 256, c->stream, M->N, order,
                     (const unsigned*)M->A->d_rowptr, (const unsigned*)M->A->d_colind, (const unsigned*)M->d_diaind,
                     fd, fo, vi, vo, rd, (double*)nullptr, sc, rr_part, rr_n, c->d_status, (uint64_t)c->wait_ns);
}

template <int LPR, bool FWD>
static cudaError_t sweep_cplx(dfm_ilu M, int sweep, const double* in, double* out, const double* rdot,
                              double* part, KrylovScalars* sc, const double* rr_part, int rr_n, bool f32) {
  if (f32)
    return sweep_cplx_tv<LPR, FWD, float2>(M, reinterpret_cast<const float2*>(M->d_foff32), sweep, in, out, rdot,
                                           part, sc, rr_part, rr_n);
  return sweep_cplx_tv<LPR, FWD, double2>(M, reinterpret_cast<const double2*>(M->d_foff), sweep, in, out, rdot,
                                          part, sc, rr_part, rr_n);
}

static int sweep_dispatch(dfm_ilu M, bool fwd, int sweep, const double* in, double* out, const double* rdot,
                          double* part, KrylovScalars* sc, const double* rr_part, int rr_n, bool f32) {
  if (M->N == 0) return DFM_OK;
  if (sweep <= 0) sweep = M->sweep > 0 ? M->sweep : 1;
  if (f32 && !M->d_foff32) return DFM_ERR_INVALID;
  if (sweep == 3) return sweep_ranges_launch(M, fwd, in, out, rdot, part, sc, rr_part, rr_n, f32);
  cudaError_t e;
  if (M->vt == DFM_COMPLEX) {
    e = fwd ? sweep_cplx<8, true>(M, sweep, in, out, rdot, part, sc, rr_part, rr_n, f32)
            : sweep_cplx<8, false>(M, sweep, in, out, rdot, part, sc, rr_part, rr_n, f32);
  } else if (M->b == 1) {
    e = fwd ? sweep_real<1, 8, true>(M, sweep, in, out, rdot, part, sc, rr_part, rr_n, f32)
            : sweep_real<1, 8, false>(M, sweep, in, out, rdot, part, sc, rr_part, rr_n, f32);
  } else if (M->b == 2) {
    e = fwd ? sweep_real<2, 8, true>(M, sweep, in, out, rdot, part, sc, rr_part, rr_n, f32)
            : sweep_real<2, 8, false>(M, sweep, in, out, rdot, part, sc, rr_part, rr_n, f32);
  } else {
    e = fwd ? sweep_real<3, 16, true>(M, sweep, in, out, rdot, part, sc, rr_part, rr_n, f32)
            : sweep_real<3, 16, false>(M, sweep, in, out, rdot, part, sc, rr_part, rr_n, f32);
  }
  DFM_CUDA_TRY(e);
  return DFM_OK;
}

int ilu_fwd_launch(dfm_ilu M, const double* r, double* y, KrylovScalars* sc, int sweep, bool rr_check, bool f32) {
  const bool chk = sc && rr_check;
  return sweep_dispatch(M, true, sweep, r, y, nullptr, nullptr, sc, chk ? M->ctx->part(2) : nullptr,
                        chk ? spmv_grid(M->A) : 0, f32);
}

int ilu_bwd_launch(dfm_ilu M, const double* y, double* z, const double* rdot, double* dot_part, KrylovScalars* sc,
                   int sweep, bool f32) {
  return sweep_dispatch(M, false, sweep, y, z, rdot, dot_part, sc, nullptr, 0, f32);
}

int ilu_prepare(dfm_ilu M, bool f32) {
  if (M->sweep == 3) {
    if (M->plan_f.stale && (M->plan_f.valid) && sweep_plan_refresh(M, &M->plan_f)) return DFM_ERR_CUDA;
    if (M->plan_b.stale && (M->plan_b.valid) && sweep_plan_refresh(M, &M->plan_b)) return DFM_ERR_CUDA;
  }
  if (!f32) return DFM_OK;
  const size_t no = (size_t)M->ncrs * M->vw();
  if (!M->d_foff32) DFM_CUDA_TRY(cudaMalloc(&M->d_foff32, std::max<size_t>(no, 1) * sizeof(float)));
  int rc = to_f32(M->ctx, M->d_foff, M->d_foff32, no);
  if (rc) return rc;
  if (M->sweep == 3) {
    // FP32 plans with the FP64 plans' ranges and lanes
    for (int f = 0; f < 2; f++) {
      SweepPlan& P64 = f ? M->plan_b : M->plan_f;
      SweepPlan& P32 = f ? M->plan32_b : M->plan32_f;
      if (!P32.valid || P32.G != P64.G || P32.lpr != P64.lpr || P32.merged != P64.merged ||
          P32.halo != P64.halo || P32.cw != P64.cw || P32.hw != P64.hw) {
        if ((rc = sweep_plan_build(M, f == 0, P64.G, 4, 8, &P32, P64.merged, P64.part, P64.halo))) return rc;
        P32.lpr = P64.lpr;
        P32.cw = P64.cw;
        P32.hw = P64.hw;
        M->plan_gen++;  // captured graphs hold the old plan's buffers
      }
      P32.nb = P64.nb && P32.nb_ok;
      P32.pipe = P64.pipe;
      if ((rc = sweep_plan_refresh(M, &P32))) return rc;
    }
  }
  return DFM_OK;
}

// Autotuner for the sweep schedule: times one forward+backward application
// with each schedule (best of 3) and keeps the faster one.
int ilu_autotune(dfm_ilu M) {
  if (M->sweep > 0) return DFM_OK;
  if (M->N == 0) { M->sweep = 1; return DFM_OK; }
  cudaStream_t s = M->ctx->stream;
  const size_t n = (size_t)M->N * M->xw();
  double *r = nullptr, *z = nullptr;
  DFM_CUDA_TRY(cudaMallocAsync(&r, n * sizeof(double), s));
  DFM_CUDA_TRY(cudaMallocAsync(&z, n * sizeof(double), s));
  DFM_CUDA_TRY(cudaMemsetAsync(r, 0, n * sizeof(double), s));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto time_mode = [&](int mode, float* out_ms) -> int {
    float tmin = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
      int rc = ilu_fill_sentinel(M, M->d_tmp, n);
      rc |= ilu_fill_sentinel(M, z, n);
      cudaEventRecord(e0, s);
      if (!rc) rc = ilu_fwd_launch(M, r, M->d_tmp, nullptr, mode);
      if (!rc) rc = ilu_bwd_launch(M, M->d_tmp, z, nullptr, nullptr, nullptr, mode);
      cudaEventRecord(e1, s);
      if (rc) return rc;
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) tmin = std::min(tmin, ms);
    }
    *out_ms = tmin;
    return take_code(M->ctx);
  };
  float best = 1e30f;
  int best_mode = 1;
  for (int mode = 1; mode <= 2; mode++) {
    float ms;
    int rc = time_mode(mode, &ms);
    if (rc) return rc;
    if (ms < best) { best = ms; best_mode = mode; }
  }
  // range-partitioned schedule: every CTA count whose slice fits in shared memory,
  // then, at the best count, merged level pairs and the barrier-free kernel
  // (complex matrices run as real 2x2 blocks)
  {
    sweep_plan_free(&M->plan_f);
    sweep_plan_free(&M->plan_b);
    SweepPlan best_f, best_b;  // owned here until the end
    const int nsm = M->ctx->nsm;
    const int cand[] = {nsm, nsm / 2, nsm / 4, 16, 8, 4, 2, 1};
    int last = -1, best_G = 0;
    float best3 = 1e30f;
    // times the candidate plans (pf, pb) over lanes per row and the kernel
    // variants in `kinds` (0 = level barrier, 1 = barrier-free, 2 = level
    // barrier with the two-half row pipeline); keeps them in best_f/best_b if
    // they beat `best`
    auto try_plans = [&](SweepPlan& pf, SweepPlan& pb, std::initializer_list<int> kinds, float* tbest) -> int {
      std::swap(M->plan_f, pf);  // M holds the candidate
      std::swap(M->plan_b, pb);
      float ms = 1e30f;
      int rc = DFM_OK, best_lpr = 1, best_kind = 0;
      for (int kind : kinds) {
        if (rc) break;
        if (kind == 1 && !(M->plan_f.nb_ok && M->plan_b.nb_ok)) continue;
        for (int lpr : {1, 2, 4, 8}) {  // consumer lanes per row
          M->plan_f.lpr = M->plan_b.lpr = lpr;
          M->plan_f.nb = M->plan_b.nb = kind == 1;
          M->plan_f.pipe = M->plan_b.pipe = kind == 2;
          float t = 1e30f;
          rc = time_mode(3, &t);
          if (rc) break;
          if (t < ms) { ms = t; best_lpr = lpr; best_kind = kind; }
        }
      }
      M->plan_f.lpr = M->plan_b.lpr = best_lpr;
      M->plan_f.nb = M->plan_b.nb = best_kind == 1;
      M->plan_f.pipe = M->plan_b.pipe = best_kind == 2;
      std::swap(M->plan_f, pf);  // candidate back in pf/pb, M empty
      std::swap(M->plan_b, pb);
      if (tbest) *tbest = ms;
      if (rc == DFM_OK && ms < best) {
        best = ms;
        best_mode = 3;
        sweep_plan_free(&best_f);
        sweep_plan_free(&best_b);
        std::swap(best_f, pf);
        std::swap(best_b, pb);
      } else {
        sweep_plan_free(&pf);
        sweep_plan_free(&pb);
      }
      return rc;
    };
    // the caller's row partition (one CTA per part) first, then balanced
    // ranges of the natural order at every CTA count
    bool best_part = false;
    auto try_G = [&](int G, bool part) -> int {
      SweepPlan pf, pb;
      if (sweep_plan_build(M, true, G, 8, 8, &pf, false, part) != DFM_OK ||
          sweep_plan_build(M, false, G, 8, 8, &pb, false, part) != DFM_OK) {
        sweep_plan_free(&pf);
        sweep_plan_free(&pb);
        cudaGetLastError();
        return DFM_OK;  // slice does not fit in shared memory at this CTA count
      }
      float t = 1e30f;
      const int rc = try_plans(pf, pb, {0, 2}, &t);
      if (rc != DFM_OK && rc != DFM_ERR_UNSUPPORTED) return rc;
      if (rc == DFM_OK && t < best3) { best3 = t; best_G = G; best_part = part; }
      return DFM_OK;
    };
    if (M->nparts > 0 && M->nparts <= (unsigned)nsm) {
      const int rc = try_G((int)M->nparts, true);
      if (rc) {
        sweep_plan_free(&best_f);
        sweep_plan_free(&best_b);
        return rc;
      }
    }
    for (int G : cand) {
      if (G < 1 || G == last) continue;
      last = G;
      const int rc = try_G(G, false);
      if (rc) {
        sweep_plan_free(&best_f);
        sweep_plan_free(&best_b);
        return rc;
      }
    }
    if (best_G > 0) {
      for (int mg = 0; mg < 2; mg++) {  // barrier-free kernel unmerged, then merged pairs with every kernel
        SweepPlan pf, pb;
        if (sweep_plan_build(M, true, best_G, 8, 8, &pf, mg != 0, best_part) != DFM_OK ||
            sweep_plan_build(M, false, best_G, 8, 8, &pb, mg != 0, best_part) != DFM_OK) {
          sweep_plan_free(&pf);
          sweep_plan_free(&pb);
          cudaGetLastError();
          continue;
        }
        const int rc = mg ? try_plans(pf, pb, {0, 1, 2}, nullptr) : try_plans(pf, pb, {1}, nullptr);
        if (rc != DFM_OK && rc != DFM_ERR_UNSUPPORTED) {
          sweep_plan_free(&best_f);
          sweep_plan_free(&best_b);
          return rc;
        }
      }
    }
    // the shared-memory-only schedule (modes 9 and 10) at the partition and at
    // one CTA per SM: compute warps x lanes per row, producer warps
    {
      const unsigned bx = M->vt == DFM_COMPLEX ? 2u : M->b;
      struct Cfg { int cw, lpr, hw; };
      const Cfg cfgs3[] = {{1, 4, 4}, {2, 4, 4}, {4, 4, 4}, {4, 8, 4}, {2, 8, 4}, {4, 4, 8}};
      const Cfg cfgs1[] = {{1, 2, 4}, {1, 4, 4}, {2, 4, 4}, {4, 4, 4}, {2, 2, 4}, {4, 4, 8}};
      const Cfg* cfgs = bx == 1 ? cfgs1 : cfgs3;
      auto try_halo = [&](int G, bool part, bool merge) -> int {
        SweepPlan pf, pb;
        if (sweep_plan_build(M, true, G, 8, 8, &pf, merge, part, true) != DFM_OK ||
            sweep_plan_build(M, false, G, 8, 8, &pb, merge, part, true) != DFM_OK) {
          sweep_plan_free(&pf);
          sweep_plan_free(&pb);
          cudaGetLastError();
          return DFM_OK;
        }
        std::swap(M->plan_f, pf);
        std::swap(M->plan_b, pb);
        float ms = 1e30f;
        Cfg bc = cfgs[0];
        int rc = DFM_OK;
        for (int q = 0; q < 6 && rc == DFM_OK; q++) {
          M->plan_f.cw = M->plan_b.cw = cfgs[q].cw;
          M->plan_f.lpr = M->plan_b.lpr = cfgs[q].lpr;
          M->plan_f.hw = M->plan_b.hw = cfgs[q].hw;
          float t = 1e30f;
          rc = time_mode(3, &t);
          if (rc == DFM_OK && t < ms) { ms = t; bc = cfgs[q]; }
          if (rc == DFM_ERR_CUDA || rc == DFM_ERR_UNSUPPORTED) {  // a launch this configuration cannot have
            cudaGetLastError();
            rc = DFM_OK;
          }
        }
        M->plan_f.cw = M->plan_b.cw = bc.cw;
        M->plan_f.lpr = M->plan_b.lpr = bc.lpr;
        M->plan_f.hw = M->plan_b.hw = bc.hw;
        std::swap(M->plan_f, pf);
        std::swap(M->plan_b, pb);
        if (rc == DFM_OK && ms < best) {
          best = ms;
          best_mode = 3;
          sweep_plan_free(&best_f);
          sweep_plan_free(&best_b);
          std::swap(best_f, pf);
          std::swap(best_b, pb);
        } else {
          sweep_plan_free(&pf);
          sweep_plan_free(&pb);
        }
        return rc == DFM_ERR_UNSUPPORTED ? DFM_OK : rc;
      };
      int rc = DFM_OK;
      for (int mg = 0; mg < 2 && rc == DFM_OK; mg++) {  // levels one by one (mode 9), in merged pairs (mode 10)
        if (M->nparts > 0 && M->nparts <= (unsigned)nsm) rc = try_halo((int)M->nparts, true, mg != 0);
        if (rc == DFM_OK) rc = try_halo(nsm, false, mg != 0);
      }
      if (rc) {
        sweep_plan_free(&best_f);
        sweep_plan_free(&best_b);
        return rc;
      }
    }
    std::swap(M->plan_f, best_f);
    std::swap(M->plan_b, best_b);
    M->plan_gen++;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(r, s);
  cudaFreeAsync(z, s);
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  M->sweep = best_mode;
  M->sweep_ms = best;
  return DFM_OK;
}

int ilu_set_ranges(dfm_ilu M, int G, bool merge, bool halo) {
  SweepPlan pf, pb;
  const bool part = M->nparts > 0;  // a row partition, when set, fixes the CTAs
  if (part) G = (int)M->nparts;
  int rc = sweep_plan_build(M, true, G, 8, 8, &pf, merge, part, halo);
  if (!rc) rc = sweep_plan_build(M, false, G, 8, 8, &pb, merge, part, halo);
  if (rc) {
    sweep_plan_free(&pf);
    sweep_plan_free(&pb);
    return rc;
  }
  sweep_plan_free(&M->plan_f);
  sweep_plan_free(&M->plan_b);
  std::swap(M->plan_f, pf);
  std::swap(M->plan_b, pb);
  M->sweep = 3;
  M->plan_gen++;
  return DFM_OK;
}

int ilu_wait_selftest(dfm_ctx ctx, unsigned long long limit_ns) {
  double* flag = nullptr;
  DFM_CUDA_TRY(cudaMallocAsync(&flag, sizeof(double), ctx->stream));
  k_fill_sentinel<<<1, 32, 0, ctx->stream>>>(flag, 1);
  k_wait_selftest<<<1, 1, 0, ctx->stream>>>(flag, ctx->d_status, (uint64_t)limit_ns);
  DFM_CUDA_TRY(cudaGetLastError());
  DFM_CUDA_TRY(cudaFreeAsync(flag, ctx->stream));
  DFM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DFM_OK;
}

}  // namespace dfm
