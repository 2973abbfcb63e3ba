// Device helpers shared by the range-partitioned sweep kernels (sweep.cu,
// sweep_halo.cu): mbarrier and TMA bulk-copy PTX, bounded waits, the batched
// re-poll of remote operands and the fused dot of a finished slice.
#pragma once
#include <stdint.h>

#include "dfm_internal.h"
#include "sweep.h"

namespace dfm {

constexpr int kOpBatch = 4;  // operands of one lane loaded together in the range sweeps

// ------------------------------------------------------------ PTX helpers
DFM_DEVINL unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

DFM_DEVINL void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
DFM_DEVINL void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
DFM_DEVINL void mbar_arrive_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
DFM_DEVINL bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 1-D bulk copy global -> this CTA's shared memory (addresses and size 16-byte multiples).
DFM_DEVINL void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

DFM_DEVINL int ld_status2(const DevStatus* st) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(&st->code) : "memory");
  return v;
}

// Re-reads the remote operands of a batch that still hold the sentinel: every
// missing value is re-read in each pass, so a batch whose producers are just
// publishing costs one L2 round trip per pass instead of one per value (a
// b x b row of B values would otherwise wait for B round trips in a row).
// xo[u]: operand codes (remote = 0x80000000 | row); xv[u][c]: values read so
// far.  The wait is bounded: past wait_ns (or once another wait has failed)
// it records DFM_WAIT_TIMEOUT and returns.
template <int B, int NB, typename TX>
DFM_DEVINL void repoll_batch(const unsigned* xo, TX (*xv)[B], const TX* out, DevStatus* st, uint64_t wait_ns,
                             int where) {
  auto missing = [&]() {
    bool m = false;
#pragma unroll
    for (int u = 0; u < NB; u++)
      if ((xo[u] & 0xc0000000u) == 0x80000000u)
#pragma unroll
        for (int c = 0; c < B; c++) m |= Sent<TX>::is(xv[u][c]);
    return m;
  };
  if (!missing()) return;
  SpinGuard g(wait_ns);
  for (;;) {
#pragma unroll
    for (int u = 0; u < NB; u++)
      if ((xo[u] & 0xc0000000u) == 0x80000000u)
#pragma unroll
        for (int c = 0; c < B; c++)
          if (Sent<TX>::is(xv[u][c])) xv[u][c] = ld_relaxed(out + (size_t)(xo[u] & 0x7fffffffu) * B + c);
    if (!missing()) return;
    if (g.expired() || ((g.n & 1023u) == 0 && ld_status2(st) != 0)) {
      raise_error(st, DFM_WAIT_TIMEOUT, where);
      return;
    }
  }
}

// Waits for a stage phase; false (after recording the error) if it never completes.
DFM_DEVINL bool wait_stage(uint64_t* bar, unsigned parity, DevStatus* st, uint64_t wait_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  SpinGuard g(wait_ns);
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (g.expired()) {
      raise_error(st, DFM_WAIT_TIMEOUT, 10);
      return false;
    }
  }
}

// Block partial of the CTA's share of (rdot, out) from its finished slice X.
// DOT 1: real dot over len*B entries; DOT 2: complex matrices run as real 2x2
// blocks (re, im per row), the unconjugated sum of rdot_i out_i with the real
// and imaginary parts in part[] and part[kMaxBlocks + ...].
// rows: the plan's row order (slot k of the slice is row rows[a0 + k]), or
// nullptr for the natural order (row a0 + k).
DFM_DEVINL size_t slot_row(const unsigned* rows, unsigned p) { return rows ? (size_t)rows[p] : (size_t)p; }

// The CTA's slice X[k] = v[row of slot a0 + k / B][k % B], k < len * B.  A
// thread takes k = tid, tid + T, ... (T threads) as U independent loads at a
// time (the slot -> row lookups of a batch, then their values): the slice is
// read from L2 at the start of every sweep, on the critical path, and one
// dependent round trip per element would serialise ~len * B / T of them.
template <int B, int U, typename TX, typename TI>
DFM_DEVINL void load_slice(TX* X, const TI* __restrict__ v, const unsigned* __restrict__ rows, unsigned a0,
                           unsigned len) {
  const unsigned tot = len * B, T = blockDim.x;
  for (unsigned k0 = threadIdx.x; k0 < tot; k0 += U * T) {
    TI w[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const unsigned k = k0 + (unsigned)u * T;
      w[u] = k < tot ? v[slot_row(rows, a0 + k / B) * B + k % B] : TI(0);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const unsigned k = k0 + (unsigned)u * T;
      if (k < tot) X[k] = w[u];
    }
  }
}

// This thread's share of sum_k rdot[row of slot a0 + k / B][k % B] * X[k]
// (real) in ascending k, U loads of rdot at a time; the same sum, in the same
// order, as one load per term.
template <int B, int U, typename TX, typename TR>
DFM_DEVINL double slice_dot(const TR* __restrict__ rdot, const TX* X, const unsigned* __restrict__ rows,
                            unsigned a0, unsigned len) {
  const unsigned tot = len * B, T = blockDim.x;
  double acc = 0.0;
  for (unsigned k0 = threadIdx.x; k0 < tot; k0 += U * T) {
    TR w[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const unsigned k = k0 + (unsigned)u * T;
      w[u] = k < tot ? rdot[slot_row(rows, a0 + k / B) * B + k % B] : TR(0);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const unsigned k = k0 + (unsigned)u * T;
      if (k < tot) acc += (double)w[u] * (double)X[k];
    }
  }
  return acc;
}

// The complex form (rows as (re, im) pairs): this thread's share of the
// unconjugated sum_k rdot_k X_k over slots k = tid, tid + T, ..., U at a time.
template <int U, typename TX, typename TR>
DFM_DEVINL void slice_zdot(const TR* __restrict__ rdot, const TX* X, const unsigned* __restrict__ rows,
                           unsigned a0, unsigned len, double& re, double& im) {
  const unsigned T = blockDim.x;
  for (unsigned k0 = threadIdx.x; k0 < len; k0 += U * T) {
    TR wr[U], wi[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const unsigned k = k0 + (unsigned)u * T;
      const size_t gi = k < len ? slot_row(rows, a0 + k) : 0;
      wr[u] = k < len ? rdot[gi * 2] : TR(0);
      wi[u] = k < len ? rdot[gi * 2 + 1] : TR(0);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const unsigned k = k0 + (unsigned)u * T;
      if (k < len) {
        const double rr = (double)wr[u], ri = (double)wi[u];
        const double xr = (double)X[2 * k], xi = (double)X[2 * k + 1];
        re += rr * xr - ri * xi;
        im += rr * xi + ri * xr;
      }
    }
  }
}

template <int B, int DOT, typename TX>
DFM_DEVINL void range_dot(const TX* __restrict__ rdot, const TX* X, unsigned a0, unsigned len, bool alive,
                          double* part, const unsigned* rows) {
  if constexpr (DOT == 2) {
    static_assert(B == 2, "complex rows are 2x2 real blocks");
    double re = 0.0, im = 0.0;
    if (alive) slice_zdot<4>(rdot, X, rows, a0, len, re, im);
    block_partial<kSweepThreads>(re, part);
    block_partial<kSweepThreads>(im, part + kMaxBlocks);
  } else {
    double dacc = 0.0;
    if (alive) dacc = slice_dot<B, 8>(rdot, X, rows, a0, len);
    block_partial<kSweepThreads>(dacc, part);
  }
}

DFM_DEVINL double ld_volatile_s(const double* p) { return *reinterpret_cast<const volatile double*>(p); }
DFM_DEVINL float ld_volatile_s(const float* p) { return *reinterpret_cast<const volatile float*>(p); }
DFM_DEVINL void st_volatile_s(double* p, double v) { *reinterpret_cast<volatile double*>(p) = v; }
DFM_DEVINL void st_volatile_s(float* p, float v) { *reinterpret_cast<volatile float*>(p) = v; }
DFM_DEVINL void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }


}  // namespace dfm
