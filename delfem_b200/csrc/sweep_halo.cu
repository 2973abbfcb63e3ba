// Range-partitioned ILU triangular sweeps whose level path reads shared
// memory only (schedule mode 9).
//
// The rows are split among co-resident CTAs as in the range schedule
// (sweep.cu): contiguous ranges of the natural order, or the parts of the
// caller's row partition.  A CTA walks its rows level by level.  What differs
// is who waits for what:
//
//  * A few compute warps (1, 2 or 4) take the rows of a level, LPR lanes per
//    row, and read every operand from shared memory: a row of the CTA's own
//    range from its vector slice, a row of another CTA from the level's halo,
//    a small per-stage area filled ahead of time.  Between levels they meet
//    at a named barrier of their own (bar.sync 1, or __syncwarp for a single
//    warp) instead of a barrier of the whole CTA.
//  * Producer warps run ahead of them.  Producer p takes the CTA's chunks
//    (a level, or a slice of one) p, p + P, p + 2P, ...: it waits until the
//    compute warps have released the chunk's stage, copies the chunk (row
//    descriptors, operand offsets, halo row ids, factor blocks, D^-1 rows)
//    into the stage with one TMA bulk copy (cp.async.bulk, no multicast),
//    waits for it to land, then polls the halo rows' published values in
//    global memory (NaN sentinel = not yet written) until all are in, copies
//    them into the stage's halo area, puts the chunk's own right-hand sides
//    (the input vector's entries of its rows) into their slots of the slice,
//    and marks the stage ready for that chunk.  The slice is never loaded as a
//    whole: a launch starts on its first level at once.
//
// The critical path of a level is then the compute warps' own work plus a
// barrier of at most four warps; the L2 round trips for other CTAs' rows and
// the copies of the level data overlap with earlier levels, up to the depth of
// the stage ring.
//
// Every operand is addressed by a precomputed element offset into X =
// [slice | halo area of stage 0 | ... | halo area of stage nstage-1]; a chunk's
// halo offsets name the stage the chunk lands in (its index within the CTA's
// chunks modulo nstage), so the compute warps never branch on where a value
// lives.
//
// Progress: a row waits only for rows of lower level; every CTA takes its
// chunks in level order and all CTAs are co-resident (cooperative launch), so
// every wait ends.  All waits are bounded as well: past the context's limit a
// wait records DFM_WAIT_TIMEOUT, the CTA stops computing (every compute warp
// still passes each level's barrier, so no warp is left behind at a barrier),
// and copies in flight land before the CTA exits.
#include <algorithm>
#include <cstring>

#include "dfm_internal.h"
#include "sweep.h"
#include "sweep_dev.cuh"

namespace dfm {

constexpr int kHaloMaxStages = 16;
constexpr int kHaloMaxWarps = 16;
constexpr int kHaloMaxThreads = 32 * kHaloMaxWarps;

// Header of a chunk of a halo plan: 32 bytes, then the row descriptors at +32
// as in every plan (the factor gather of sweep.cu serves both).
struct HaloHeader {
  unsigned nrows, xoff, vals, dinv, hids, nhalo, pad0, pad1;
};
static_assert(sizeof(HaloHeader) == 32, "halo chunk header is 32 bytes");

DFM_DEVINL int ld_volatile_i(const int* p) { return *reinterpret_cast<const volatile int*>(p); }
DFM_DEVINL void st_volatile_i(int* p, int v) { *reinterpret_cast<volatile int*>(p) = v; }

DFM_DEVINL void compute_barrier(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Deterministic block sum of the CTA's share of (rdot, out) over its finished
// slice, for any block size (fixed order: threads, then warps).  DOT 2:
// complex rows as real 2x2 blocks, the unconjugated product, re / im parts in
// part[] and part[kMaxBlocks + ...].
template <int B, int DOT>
DFM_DEVINL void halo_dot(const double* __restrict__ rdot, const double* X, unsigned a0, unsigned len, double* part,
                         const unsigned* rows) {
  __shared__ double s_w[2][kHaloMaxWarps];
  double re = 0.0, im = 0.0;
  if constexpr (DOT == 2) {
    slice_zdot<8>(rdot, X, rows, a0, len, re, im);
  } else {
    re = slice_dot<B, 16>(rdot, X, rows, a0, len);
  }
  re = group_sum<32>(re);
  im = group_sum<32>(im);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (int)(blockDim.x >> 5);
  if (l == 0) {
    s_w[0][w] = re;
    s_w[1][w] = im;
  }
  __syncthreads();
  if (w == 0) {
    double t0 = l < nw ? s_w[0][l] : 0.0, t1 = l < nw ? s_w[1][l] : 0.0;
    t0 = group_sum<32>(t0);
    t1 = group_sum<32>(t1);
    if (l == 0) {
      part[blockIdx.x] = t0;
      if (DOT == 2) part[kMaxBlocks + blockIdx.x] = t1;
    }
  }
}

// What a lane needs of one row that does not depend on the level before it:
// the row descriptor, its first two blocks and their operand offsets, and for
// the lanes that finish components (lane c takes components c, c + LPR, ...)
// the row's right-hand side and (forward) those rows of its D^-1.  Loaded
// ahead, before the previous level's barrier where the stage is ready, so
// that only the reads of X follow that barrier.
template <int B, int LPR, typename TV>
struct RowPre {
  static constexpr int NC = (B + LPR - 1) / LPR;  // components per finishing lane
  uint4 rd;
  unsigned o0, o1;
  bool h0, h1;
  TV m0[B * B], m1[B * B];
  double xr[B], dr[NC][B];
};

template <int B, int LPR, typename TV, bool FWD>
DFM_DEVINL void row_prefetch(RowPre<B, LPR, TV>& P, const char* sb, const double* X, unsigned r, int lane) {
  constexpr int BB = B * B;
  const HaloHeader* hdr = reinterpret_cast<const HaloHeader*>(sb);
  const unsigned* xoff = reinterpret_cast<const unsigned*>(sb + hdr->xoff);
  const TV* vals = reinterpret_cast<const TV*>(sb + hdr->vals);
  P.rd = reinterpret_cast<const uint4*>(sb + 32)[r];
  const unsigned k0 = P.rd.y + (unsigned)lane, k1 = k0 + LPR;
  P.h0 = k0 < P.rd.z;
  P.h1 = k1 < P.rd.z;
  if (P.h0) {
    P.o0 = xoff[k0];
#pragma unroll
    for (int e = 0; e < BB; e++) P.m0[e] = vals[(size_t)k0 * BB + e];
  }
  if (P.h1) {
    P.o1 = xoff[k1];
#pragma unroll
    for (int e = 0; e < BB; e++) P.m1[e] = vals[(size_t)k1 * BB + e];
  }
  if (lane < B) {
    const double* xi = X + (size_t)P.rd.x * B;  // the row's right-hand side: only this row writes it
#pragma unroll
    for (int c = 0; c < B; c++) P.xr[c] = xi[c];
    if (FWD) {
      const double* d = reinterpret_cast<const double*>(sb + hdr->dinv) + (size_t)r * BB;
#pragma unroll
      for (int j = 0; j < P.NC; j++) {
        const int cc = lane + j * LPR;
        if (cc < B)
#pragma unroll
          for (int c = 0; c < B; c++) P.dr[j][c] = d[cc * B + c];
      }
    }
  }
}

// One row from its prefetched part: the operand reads, the lane sums (blocks
// kk, kk + LPR, ... in order), the butterfly over the row's lanes (every lane
// ends with the same sum), then lane c finishes components c, c + LPR, ... < B:
// x_i[c] = (D^-1 (b_i - sum))[c] forward, (b_i - sum)[c] backward, into the
// slice and published to `out`.  The same operations in the same order as
// the reference's row loop (up to the lanes' summation order).
template <int B, int LPR, typename TV, bool FWD>
DFM_DEVINL void row_finish(const RowPre<B, LPR, TV>& P, const char* sb, double* X, double* out, int lane,
                           unsigned gmask) {
  constexpr int BB = B * B;
  double acc[B];
#pragma unroll
  for (int c = 0; c < B; c++) acc[c] = 0.0;
  if (P.h0) {
    double x0[B];
#pragma unroll
    for (int c = 0; c < B; c++) x0[c] = X[P.o0 + c];
#pragma unroll
    for (int rr = 0; rr < B; rr++)
#pragma unroll
      for (int c = 0; c < B; c++) acc[rr] += (double)P.m0[rr * B + c] * x0[c];
  }
  if (P.h1) {
    double x1[B];
#pragma unroll
    for (int c = 0; c < B; c++) x1[c] = X[P.o1 + c];
#pragma unroll
    for (int rr = 0; rr < B; rr++)
#pragma unroll
      for (int c = 0; c < B; c++) acc[rr] += (double)P.m1[rr * B + c] * x1[c];
  }
  if (P.h1) {  // rows with more than 2 LPR blocks
    const HaloHeader* hdr = reinterpret_cast<const HaloHeader*>(sb);
    const unsigned* xoff = reinterpret_cast<const unsigned*>(sb + hdr->xoff);
    const TV* vals = reinterpret_cast<const TV*>(sb + hdr->vals);
    for (unsigned kk = P.rd.y + (unsigned)lane + 2 * LPR; kk < P.rd.z; kk += LPR) {
      const unsigned o = xoff[kk];
      const TV* m = vals + (size_t)kk * BB;
#pragma unroll
      for (int rr = 0; rr < B; rr++)
#pragma unroll
        for (int c = 0; c < B; c++) acc[rr] += (double)m[rr * B + c] * X[o + c];
    }
  }
  if (LPR > 1) {
#pragma unroll
    for (int rr = 0; rr < B; rr++)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[rr] += __shfl_xor_sync(gmask, acc[rr], o);
  }
  if (lane < B) {
    double t[B];
#pragma unroll
    for (int c = 0; c < B; c++) t[c] = P.xr[c] - acc[c];
#pragma unroll
    for (int j = 0; j < P.NC; j++) {
      const int cc = lane + j * LPR;
      if (cc < B) {
        double v;
        if (FWD) {
          v = 0.0;
#pragma unroll
          for (int c = 0; c < B; c++) v += P.dr[j][c] * t[c];
        } else {
          v = t[0];
#pragma unroll
          for (int c = 1; c < B; c++)
            if (c == cc) v = t[c];
        }
        X[(size_t)P.rd.x * B + cc] = v;
        st_relaxed(out + (size_t)P.rd.w * B + cc, v);
      }
    }
  }
}

// One producer lane's halo entries e0, e0 + 32, ... (NP of them, those below
// nh) into H: every entry's values are read, then each pass re-reads all the
// values that still hold the sentinel, so a lane's second entry costs no L2
// round trip of its own after the first.  Entries flagged 0x80000000 are rows
// of the input vector (merged level pairs) and need no wait.  False when the
// wait ran out (recorded) or the CTA is shutting down.
template <int B, int NP>
DFM_DEVINL bool halo_poll(const unsigned* hids, unsigned e0, unsigned nh, const double* __restrict__ in,
                          const double* out, double* H, int* s_alive, DevStatus* st, uint64_t wait_ns) {
  size_t row[NP];
  bool from_out[NP];
  double v[NP][B];
#pragma unroll
  for (int u = 0; u < NP; u++) {
    const unsigned e = e0 + 32u * u;
    const unsigned hid = e < nh ? hids[e] : 0x80000000u;
    row[u] = hid & 0x7fffffffu;
    from_out[u] = e < nh && !(hid & 0x80000000u);
#pragma unroll
    for (int c = 0; c < B; c++)
      v[u][c] = e >= nh ? 0.0 : from_out[u] ? ld_relaxed(out + row[u] * B + c) : in[row[u] * B + c];
  }
  auto missing = [&]() {
    bool m = false;
#pragma unroll
    for (int u = 0; u < NP; u++)
#pragma unroll
      for (int c = 0; c < B; c++) m |= from_out[u] && Sent<double>::is(v[u][c]);
    return m;
  };
  if (missing()) {
    SpinGuard g(wait_ns);
    for (;;) {
#pragma unroll
      for (int u = 0; u < NP; u++)
#pragma unroll
        for (int c = 0; c < B; c++)
          if (from_out[u] && Sent<double>::is(v[u][c])) v[u][c] = ld_relaxed(out + row[u] * B + c);
      if (!missing()) break;
      const bool late = g.expired();
      if (late || ((g.n & 1023u) == 0 && !ld_volatile_i(s_alive))) {
        if (late) raise_error(st, DFM_WAIT_TIMEOUT, 22);
        st_volatile_i(s_alive, 0);
        return false;
      }
    }
  }
#pragma unroll
  for (int u = 0; u < NP; u++) {
    const unsigned e = e0 + 32u * u;
    if (e < nh)
#pragma unroll
      for (int c = 0; c < B; c++) H[e * B + c] = v[u][c];
  }
  return true;
}

template <int B, int LPR, typename TV, bool FWD, int DOT>
__global__ void __launch_bounds__(kHaloMaxThreads, 1)
k_sweep_halo(const ChunkDesc* __restrict__ chunks, const unsigned* __restrict__ cta_chunk,
             const unsigned* __restrict__ range, const unsigned* __restrict__ rows, const char* __restrict__ blob,
             unsigned stage_bytes, int nstage, unsigned x_bytes, unsigned x_slice, unsigned halo_stride, int ncw,
             const double* __restrict__ in, double* out, const double* __restrict__ rdot, double* part,
             KrylovScalars* sc, const double* rr_part, int rr_nparts, DevStatus* st, uint64_t wait_ns) {
  extern __shared__ __align__(128) char smem[];
  __shared__ int s_alive;
  __shared__ int s_released;               // chunks the compute warps are done with
  __shared__ int s_ready[kHaloMaxStages];  // the chunk whose data and halo a stage holds (-1: none)
  if (sc) {
    if (block_flag(&sc->done)) return;
    if (FWD && rr_part) {
      const double rr = reduce_partials(rr_part, rr_nparts);
      if (rr * sc->inv0 < sc->tol2) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
          sc->conv = sqrt(rr * sc->inv0);
          sc->conv_it = sc->it;
          sc->done = sc->conv_code;
        }
        return;
      }
    }
  }
  const unsigned a0 = range[blockIdx.x], a1 = range[blockIdx.x + 1];
  const unsigned q0 = cta_chunk[blockIdx.x], q1 = cta_chunk[blockIdx.x + 1];
  const unsigned K = q1 - q0, len = a1 - a0;
  double* X = reinterpret_cast<double*>(smem);
  char* stages = smem + x_bytes;
  uint64_t* bar = reinterpret_cast<uint64_t*>(stages + (size_t)nstage * stage_bytes);

  if (threadIdx.x == 0) {
    s_alive = 1;
    s_released = 0;
    for (int s = 0; s < nstage; s++) {
      mbar_init(&bar[s], 1);
      s_ready[s] = -1;
    }
    fence_mbar_init();
  }
  __syncthreads();
  const int warp = (int)(threadIdx.x >> 5), wl = (int)(threadIdx.x & 31);
  const int nwarps = (int)(blockDim.x >> 5);
  // A producer's first chunk (pw < nstage: its stage has not been used yet) is
  // requested here, at the start.  The slice is not loaded here: the
  // producers put each chunk's right-hand sides into their slots with the
  // chunk's halo, off the compute warps' path.
  const int pw0 = warp - ncw;
  const bool pre_issued = warp >= ncw && pw0 < nstage && (unsigned)pw0 < K;
  if (pre_issued && wl == 0) {
    const ChunkDesc cd = chunks[q0 + (unsigned)pw0];
    mbar_arrive_tx(&bar[pw0], cd.bytes);
    bulk_g2s(stages + (size_t)pw0 * stage_bytes, blob + cd.off, cd.bytes, &bar[pw0]);
  }

  if (warp >= ncw) {
    // ------------------------------------------------------------ producer
    const int pw = warp - ncw, npw = nwarps - ncw;
    for (unsigned k = (unsigned)pw; k < K; k += (unsigned)npw) {
      // (the pre-issued first chunk goes on to its landing wait whatever happens)
      const bool first = pre_issued && k == (unsigned)pw;
      if (!first && __any_sync(0xffffffffu, !ld_volatile_i(&s_alive))) break;  // warp-uniform
      const int s = (int)(k % (unsigned)nstage);
      // the stage is free once the compute warps are done with chunk k - nstage
      bool ok = true;
      if (k >= (unsigned)nstage && ld_volatile_i(&s_released) < (int)(k - nstage + 1)) {
        SpinGuard g(wait_ns);
        while (ld_volatile_i(&s_released) < (int)(k - nstage + 1)) {
          if (!ld_volatile_i(&s_alive)) { ok = false; break; }
          if (g.expired()) {
            raise_error(st, DFM_WAIT_TIMEOUT, 20);
            st_volatile_i(&s_alive, 0);
            ok = false;
            break;
          }
        }
      }
      if (!__all_sync(0xffffffffu, ok)) break;  // every lane votes, waited or not
      __threadfence_block();
      const ChunkDesc cd = chunks[q0 + k];
      char* sb = stages + (size_t)s * stage_bytes;
      if (wl == 0 && !first) {
        fence_proxy_async_smem();  // the compute warps' reads of the stage precede the copy into it
        mbar_arrive_tx(&bar[s], cd.bytes);
        bulk_g2s(sb, blob + cd.off, cd.bytes, &bar[s]);
      }
      __syncwarp();
      const unsigned par = (k / (unsigned)nstage) & 1u;
      if (!mbar_try_wait(&bar[s], par)) {
        SpinGuard g(wait_ns);
        while (!mbar_try_wait(&bar[s], par)) {
          if (g.expired()) {
            raise_error(st, DFM_WAIT_TIMEOUT, 21);
            st_volatile_i(&s_alive, 0);
            ok = false;
            break;
          }
        }
      }
      if (!__all_sync(0xffffffffu, ok)) {
        // the copy must land before the CTA exits (bounded again)
        if (wl == 0) (void)wait_stage(&bar[s], par, st, wait_ns);
        break;
      }
      // halo: the other CTAs' rows this chunk reads, polled until published;
      // a lane takes entries wl, wl + 32, ..., two at a time past 32 entries
      const HaloHeader* hdr = reinterpret_cast<const HaloHeader*>(sb);
      const unsigned nh = hdr->nhalo;
      const unsigned* hids = reinterpret_cast<const unsigned*>(sb + hdr->hids);
      double* H = X + x_slice + (size_t)s * halo_stride;
      // the chunk's own right-hand sides (in[] of its rows) go into their slots
      // of the slice: lane l reads row l's before the halo poll and stores them
      // after it, rows past 32 follow (the slice is not loaded up front)
      const unsigned nr = hdr->nrows;
      const uint4* rdesc = reinterpret_cast<const uint4*>(sb + 32);
      double rhs[B];
      const bool has_row = (unsigned)wl < nr;
      unsigned slot = 0;
      if (has_row) {
        const uint4 rd = rdesc[wl];
        slot = rd.x;
#pragma unroll
        for (int c = 0; c < B; c++) rhs[c] = in[(size_t)rd.w * B + c];
      }
      if (nh > 32u) {
        for (unsigned e0 = (unsigned)wl; e0 < nh && ok; e0 += 64u)
          ok = halo_poll<B, 2>(hids, e0, nh, in, out, H, &s_alive, st, wait_ns);
      } else if ((unsigned)wl < nh) {
        ok = halo_poll<B, 1>(hids, (unsigned)wl, nh, in, out, H, &s_alive, st, wait_ns);
      }
      if (has_row)
#pragma unroll
        for (int c = 0; c < B; c++) X[(size_t)slot * B + c] = rhs[c];
      for (unsigned rr = (unsigned)wl + 32u; rr < nr; rr += 32u) {
        const uint4 rd = rdesc[rr];
#pragma unroll
        for (int c = 0; c < B; c++) X[(size_t)rd.x * B + c] = in[(size_t)rd.w * B + c];
      }
      if (!__all_sync(0xffffffffu, ok)) break;
      __syncwarp();  // every lane's halo stores precede lane 0's release
      if (wl == 0) {
        __threadfence_block();
        st_volatile_i(&s_ready[s], (int)k);
      }
    }
  } else {
    // ------------------------------------------------------------- compute
    const int nct = ncw * 32;
    const int lane = (int)threadIdx.x % LPR;
    const unsigned g = threadIdx.x / LPR, ng = (unsigned)nct / LPR;
    const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
    bool alive = true;
    RowPre<B, LPR, TV> pre;
    bool have_pre = false;     // pre holds row g of chunk k (loaded before chunk k-1's barrier)
    unsigned nrows = 0;        // chunk k's rows, read with the look-ahead
    unsigned s = 0;            // chunk k's stage
    for (unsigned k = 0; k < K; k++) {
      const char* sb = stages + (size_t)s * stage_bytes;
      if (!have_pre) {
        // wait until the producer marked the stage ready for chunk k
        if (alive && ld_volatile_i(&s_ready[s]) != (int)k) {
          SpinGuard gd(wait_ns);
          while (ld_volatile_i(&s_ready[s]) != (int)k) {
            if (!ld_volatile_i(&s_alive)) { alive = false; break; }
            if (gd.expired()) {
              raise_error(st, DFM_WAIT_TIMEOUT, 23);
              st_volatile_i(&s_alive, 0);
              alive = false;
              break;
            }
          }
        }
        // the stage's copy landed before the producer released the flag (it
        // waited for the copy's mbarrier phase), so the fence suffices here
        __threadfence_block();
        alive = __all_sync(0xffffffffu, alive);  // the lanes of a row's group agree
        nrows = alive ? reinterpret_cast<const HaloHeader*>(sb)->nrows : 0u;
        if (g < nrows) row_prefetch<B, LPR, TV, FWD>(pre, sb, X, g, lane);
      }
      if (alive) {
        for (unsigned r = g; r < nrows; r += ng) {
          if (r != g) row_prefetch<B, LPR, TV, FWD>(pre, sb, X, r, lane);
          row_finish<B, LPR, TV, FWD>(pre, sb, X, out, lane, gmask);
        }
      }
      // look ahead: chunk k + 1's first row, if the producer already made its
      // stage ready (nothing is waited for here)
      const unsigned s1 = s + 1 == (unsigned)nstage ? 0u : s + 1;
      have_pre = false;
      if (alive && k + 1 < K) {
        bool rdy = ld_volatile_i(&s_ready[s1]) == (int)(k + 1);
        __threadfence_block();
        rdy = __all_sync(0xffffffffu, rdy);
        if (rdy) {
          nrows = reinterpret_cast<const HaloHeader*>(stages + (size_t)s1 * stage_bytes)->nrows;
          if (g < nrows) row_prefetch<B, LPR, TV, FWD>(pre, stages + (size_t)s1 * stage_bytes, X, g, lane);
          have_pre = true;
        }
      }
      // every compute warp passes every level's barrier, alive or not
      if (ncw > 1) compute_barrier(nct);
      else __syncwarp();
      if (threadIdx.x == 0) {
        __threadfence_block();
        st_volatile_i(&s_released, (int)k + 1);
      }
      s = s1;
    }
  }
  __syncthreads();
  if (DOT) halo_dot<B, DOT>(rdot, X, a0, len, part, rows);
}

// ------------------------------------------------------------------ plan
// The halo plan of one sweep direction over G CTAs (contiguous ranges of the
// natural order balanced by dependency blocks, or the ILU's row partition):
// chunks per level with their halo row lists, operand offsets into X.
int sweep_halo_plan_build(dfm_ilu M, bool fwd, int G, int val_bytes, SweepPlan* P, bool part, bool merge) {
  const unsigned N = M->N;
  const unsigned b = M->vt == DFM_COMPLEX ? 2u : M->b;  // complex scalars as real 2x2 blocks
  const unsigned bb = b * b;
  const unsigned vblk = (unsigned)val_bytes * bb;
  const unsigned drow = fwd ? 8u * bb : 0u;
  const std::vector<unsigned>& rp = M->A->h_rowptr;
  const std::vector<unsigned>& ci = M->A->h_colind;
  const std::vector<unsigned>& dia = M->h_diaind;
  const std::vector<unsigned>& lev = fwd ? M->lev_f : M->lev_b;
  sweep_plan_free(P);
  if (N >= 0x40000000u) return DFM_ERR_UNSUPPORTED;
  std::vector<unsigned> order, pos, range;
  if (part) {
    if ((unsigned)G != M->nparts || M->part_of.size() != N) return DFM_ERR_INVALID;
    range.assign(G + 1, 0);
    for (unsigned i = 0; i < N; i++) range[M->part_of[i] + 1]++;
    for (int c = 0; c < G; c++) range[c + 1] += range[c];
    order.assign(N, 0);
    pos.assign(N, 0);
    std::vector<unsigned> fill(range.begin(), range.end() - 1);
    for (unsigned i = 0; i < N; i++) {
      pos[i] = fill[M->part_of[i]]++;
      order[pos[i]] = i;
    }
  } else {
    if (G < 1) G = 1;
    if ((unsigned)G > std::max(N, 1u)) G = (int)std::max(N, 1u);
    std::vector<unsigned long long> wpre(N + 1, 0);
    for (unsigned i = 0; i < N; i++) {
      const unsigned nb = fwd ? dia[i] - rp[i] : rp[i + 1] - dia[i];
      wpre[i + 1] = wpre[i] + nb + 1;
    }
    range.assign(G + 1, N);
    range[0] = 0;
    for (int c = 1; c < G; c++) {
      const unsigned long long target = wpre[N] * (unsigned long long)c / (unsigned)G;
      range[c] = (unsigned)(std::lower_bound(wpre.begin(), wpre.end(), target) - wpre.begin());
      range[c] = std::max(range[c], range[c - 1]);
    }
  }
  const auto pos_of = [&](unsigned row) { return pos.empty() ? row : pos[row]; };
  const auto row_at = [&](unsigned p) { return order.empty() ? p : order[p]; };
  unsigned maxlen = 0;
  for (int c = 0; c < G; c++) maxlen = std::max(maxlen, range[c + 1] - range[c]);
  const size_t x_slice = (size_t)maxlen * b;
  if (x_slice * 8 + 8 * 1024 > kSweepSmemBudget) return DFM_ERR_UNSUPPORTED;  // use more CTAs

  struct Pend {
    std::vector<uint4> rd;
    std::vector<unsigned> xo, hids;
  };
  std::vector<ChunkDesc> chunks;
  std::vector<Pend> pend;
  std::vector<unsigned> cta_chunk(G + 1, 0);
  std::vector<uint4> recipe, terms;
  constexpr unsigned NONE = 0xffffffffu;
  // halo entries: another CTA's output row, or (kInput) an entry of the input
  // vector, which the second level of a merged pair reads in place of the
  // first level's output
  constexpr unsigned kInput = 0x80000000u;
  std::vector<unsigned> hmap(N, NONE);                   // scratch: output row -> halo index in the chunk
  std::vector<unsigned> hmap_in(merge ? N : 0u, NONE);   // scratch: input entry -> halo index
  unsigned maxhalo = 1, stage_max = 32;
  // step of a row: its level, or with merged level pairs its level / 2
  auto step = [&](unsigned i) { return merge ? lev[i] / 2 : lev[i]; };
  // operands of row i: kind 0 = a slot of this CTA's slice (v = slot), 1 =
  // another CTA's output row v, 2 = the input vector's row v; with the recipe
  // of the packed block (the same substitutions as the range plans, sweep.cu)
  struct Op {
    unsigned kind, v;
    uint4 rc;
  };
  std::vector<Op> ops;
  std::vector<unsigned> kmap(merge ? N : 0u, NONE);  // scratch: column -> position in ops
  auto slots = [&](unsigned i, unsigned& s0, unsigned& s1) {
    s0 = fwd ? rp[i] : dia[i];
    s1 = fwd ? dia[i] : rp[i + 1];
  };
  auto row_ops = [&](unsigned i, unsigned a0, unsigned a1) {
    ops.clear();
    auto opnd = [&](unsigned col, uint4 rc) -> Op {
      const unsigned pc = pos_of(col);
      return (pc >= a0 && pc < a1) ? Op{0u, pc - a0, rc} : Op{1u, col, rc};
    };
    unsigned s0, s1;
    slots(i, s0, s1);
    if (!(merge && (lev[i] & 1u))) {
      for (unsigned s = s0; s < s1; s++) ops.push_back(opnd(ci[s], make_uint4(s, 0u, 0u, 0u)));
      return;
    }
    // second level of a pair: operands on the first level are substituted
    for (unsigned s = s0; s < s1; s++) {
      const unsigned j = ci[s];
      if (lev[j] + 1 != lev[i]) continue;
      const unsigned t0 = (unsigned)terms.size();
      terms.push_back(make_uint4(s, fwd ? j : NONE, NONE, 0u));  // L_ij D_j^-1  |  U'_ij
      ops.push_back(Op{2u, j, make_uint4(NONE, t0, t0 + 1, 0u)});
    }
    const size_t first_c = ops.size();
    for (unsigned s = s0; s < s1; s++) {
      const unsigned k = ci[s];
      if (lev[k] + 1 == lev[i]) continue;
      kmap[k] = (unsigned)ops.size();
      ops.push_back(opnd(k, make_uint4(s, 0u, 0u, 1u)));
    }
    // fill terms F_ij (D_j^-1) F_jk, grouped per column k
    std::vector<std::vector<uint4>> tl(ops.size() - first_c);
    for (unsigned s = s0; s < s1; s++) {
      const unsigned j = ci[s];
      if (lev[j] + 1 != lev[i]) continue;
      unsigned t0, t1;
      slots(j, t0, t1);
      for (unsigned t = t0; t < t1; t++) {
        const unsigned k = ci[t];
        if (kmap[k] == NONE) {
          kmap[k] = (unsigned)ops.size();
          ops.push_back(opnd(k, make_uint4(NONE, 0u, 0u, 1u)));
          tl.emplace_back();
        }
        tl[kmap[k] - first_c].push_back(make_uint4(s, fwd ? j : NONE, t, 0u));
      }
    }
    for (size_t q = first_c; q < ops.size(); q++) {
      ops[q].rc.y = (unsigned)terms.size();
      for (const uint4& t : tl[q - first_c]) terms.push_back(t);
      ops[q].rc.z = (unsigned)terms.size();
      kmap[ops[q].kind == 0 ? row_at(a0 + ops[q].v) : ops[q].v] = NONE;
    }
  };
  for (int c = 0; c < G; c++) {
    cta_chunk[c] = (unsigned)chunks.size();
    const unsigned a0 = range[c], a1 = range[c + 1];
    std::vector<unsigned> rows(a1 - a0);
    for (unsigned q = a0; q < a1; q++) rows[q - a0] = row_at(fwd ? q : (a1 - 1 - (q - a0)));
    std::stable_sort(rows.begin(), rows.end(), [&](unsigned x, unsigned y) { return step(x) < step(y); });
    size_t p = 0;
    while (p < rows.size()) {
      const unsigned L = step(rows[p]);
      Pend pd;
      unsigned nblk = 0;
      const size_t rec0 = recipe.size();
      while (p < rows.size() && step(rows[p]) == L) {
        const unsigned i = rows[p];
        const size_t tmark = terms.size();
        row_ops(i, a0, a1);
        unsigned newh = 0;
        for (const Op& o : ops)
          if ((o.kind == 1 && hmap[o.v] == NONE) || (o.kind == 2 && hmap_in[o.v] == NONE)) newh++;
        const unsigned nb = (unsigned)ops.size();
        const ChunkLayout est = chunk_layout((unsigned)pd.rd.size() + 1, ((nblk + nb) + 3) & ~3u,
                                             (unsigned)pd.hids.size() + newh, vblk, drow);
        if (!pd.rd.empty() && (est.bytes > kChunkMaxBytes || pd.rd.size() >= kChunkMaxRows)) {
          terms.resize(tmark);  // this row starts the next chunk
          break;
        }
        pd.rd.push_back(make_uint4(pos_of(i) - a0, nblk, nblk + nb, i));  // {slot, blocks, global row}
        for (const Op& o : ops) {
          unsigned code;
          if (o.kind == 0) {
            code = o.v * b;
          } else {
            std::vector<unsigned>& hm = o.kind == 1 ? hmap : hmap_in;
            if (hm[o.v] == NONE) {
              hm[o.v] = (unsigned)pd.hids.size();
              pd.hids.push_back(o.kind == 1 ? o.v : (kInput | o.v));
            }
            code = 0x80000000u | hm[o.v];
          }
          pd.xo.push_back(code);
          recipe.push_back(o.rc);
        }
        nblk += nb;
        p++;
      }
      for (unsigned h : pd.hids) (h & kInput ? hmap_in[h & ~kInput] : hmap[h]) = NONE;
      const unsigned nblk_pad = (nblk + 3) & ~3u;
      for (unsigned k = nblk; k < nblk_pad; k++) {
        pd.xo.push_back(0);  // padding: outside every row's block range
        recipe.push_back(make_uint4(0xffffffffu, 0u, 0u, 0u));
      }
      ChunkDesc cd = {};
      cd.nrows = (unsigned)pd.rd.size();
      cd.nblk_pad = nblk_pad;
      cd.nhalo = (unsigned)pd.hids.size();
      cd.blk0 = (unsigned)rec0;
      cd.row0 = a0;
      const ChunkLayout cl = chunk_layout(cd.nrows, nblk_pad, cd.nhalo, vblk, drow);
      cd.vals_off = cl.vals;
      cd.dinv_off = cl.dinv;
      cd.bytes = cl.bytes;
      maxhalo = std::max(maxhalo, cd.nhalo);
      stage_max = std::max(stage_max, cl.bytes);
      chunks.push_back(cd);
      pend.push_back(std::move(pd));
    }
  }
  cta_chunk[G] = (unsigned)chunks.size();
  const unsigned stage_bytes = (stage_max + 15u) & ~15u;
  const size_t bar_bytes = 8 * (size_t)kHaloMaxStages;
  const size_t halo_stride = (size_t)maxhalo * b;
  auto xbytes = [&](int t) { return ((x_slice + (size_t)t * halo_stride) * 8 + 127) & ~(size_t)127; };
  int ns = 0;
  for (int t = kHaloMaxStages; t >= 2; t--)
    if (xbytes(t) + (size_t)t * stage_bytes + bar_bytes <= kSweepSmemBudget) { ns = t; break; }
  if (ns < 2) return DFM_ERR_UNSUPPORTED;
  if (x_slice + (size_t)ns * halo_stride >= 0x80000000ull) return DFM_ERR_UNSUPPORTED;

  size_t blob_size = 0;
  for (ChunkDesc& cd : chunks) {
    cd.off = blob_size;
    blob_size += cd.bytes;
  }
  std::vector<char> hblob(std::max<size_t>(blob_size, 16), 0);
  for (int c = 0; c < G; c++) {
    for (unsigned q = cta_chunk[c]; q < cta_chunk[c + 1]; q++) {
      const ChunkDesc& cd = chunks[q];
      const ChunkLayout cl = chunk_layout(cd.nrows, cd.nblk_pad, cd.nhalo, vblk, drow);
      const size_t hbase = x_slice + (size_t)((q - cta_chunk[c]) % (unsigned)ns) * halo_stride;
      Pend& pd = pend[q];
      for (unsigned& code : pd.xo)
        if (code & 0x80000000u) code = (unsigned)(hbase + (size_t)(code & 0x7fffffffu) * b);
      char* base = hblob.data() + cd.off;
      HaloHeader hdr = {cd.nrows, cl.xoff, cl.vals, cl.dinv, cl.hids, cd.nhalo, 0u, 0u};
      std::memcpy(base, &hdr, sizeof(hdr));
      std::memcpy(base + cl.roff, pd.rd.data(), 16 * pd.rd.size());
      std::memcpy(base + cl.xoff, pd.xo.data(), 4 * pd.xo.size());
      if (!pd.hids.empty()) std::memcpy(base + cl.hids, pd.hids.data(), 4 * pd.hids.size());
    }
  }
  P->G = G;
  P->fwd = fwd;
  P->halo = true;
  P->nchunks = (unsigned)chunks.size();
  P->stage_bytes = stage_bytes;
  P->x_bytes = (unsigned)xbytes(ns);
  P->x_slice = (unsigned)x_slice;
  P->halo_stride = (unsigned)halo_stride;
  P->val_bytes = val_bytes;
  P->vec_bytes = 8;
  P->nstage = ns;
  P->smem = xbytes(ns) + (size_t)ns * stage_bytes + bar_bytes;
  for (int c = 0; c < G; c++) P->max_cta_chunks = std::max(P->max_cta_chunks, cta_chunk[c + 1] - cta_chunk[c]);
  P->lpr = b == 1 ? 2 : 4;
  P->cw = 4;
  P->hw = 4;
  cudaStream_t s = M->ctx->stream;
  DFM_CUDA_TRY(cudaMalloc(&P->d_chunks, sizeof(ChunkDesc) * std::max<size_t>(chunks.size(), 1)));
  DFM_CUDA_TRY(cudaMalloc(&P->d_cta_chunk, sizeof(unsigned) * (G + 1)));
  DFM_CUDA_TRY(cudaMalloc(&P->d_range, sizeof(unsigned) * (G + 1)));
  DFM_CUDA_TRY(cudaMalloc(&P->d_blob, hblob.size()));
  DFM_CUDA_TRY(cudaMalloc(&P->d_recipe, sizeof(uint4) * std::max<size_t>(recipe.size(), 1)));
  DFM_CUDA_TRY(cudaMalloc(&P->d_terms, sizeof(uint4) * std::max<size_t>(terms.size(), 1)));
  if (!terms.empty())
    DFM_CUDA_TRY(cudaMemcpyAsync(P->d_terms, terms.data(), sizeof(uint4) * terms.size(), cudaMemcpyHostToDevice, s));
  if (!chunks.empty())
    DFM_CUDA_TRY(cudaMemcpyAsync(P->d_chunks, chunks.data(), sizeof(ChunkDesc) * chunks.size(),
                                 cudaMemcpyHostToDevice, s));
  DFM_CUDA_TRY(cudaMemcpyAsync(P->d_cta_chunk, cta_chunk.data(), sizeof(unsigned) * (G + 1), cudaMemcpyHostToDevice, s));
  DFM_CUDA_TRY(cudaMemcpyAsync(P->d_range, range.data(), sizeof(unsigned) * (G + 1), cudaMemcpyHostToDevice, s));
  if (!order.empty()) {
    DFM_CUDA_TRY(cudaMalloc(&P->d_rows, sizeof(unsigned) * order.size()));
    DFM_CUDA_TRY(cudaMemcpyAsync(P->d_rows, order.data(), sizeof(unsigned) * order.size(), cudaMemcpyHostToDevice, s));
  }
  P->part = part;
  DFM_CUDA_TRY(cudaMemcpyAsync(P->d_blob, hblob.data(), hblob.size(), cudaMemcpyHostToDevice, s));
  if (!recipe.empty())
    DFM_CUDA_TRY(cudaMemcpyAsync(P->d_recipe, recipe.data(), sizeof(uint4) * recipe.size(), cudaMemcpyHostToDevice, s));
  P->merged = merge;
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  P->valid = true;
  P->stale = true;
  return DFM_OK;
}

// ---------------------------------------------------------------- launch
template <int B, int LPR, typename TV, bool FWD, int DK>
static cudaError_t launch_halo(dfm_ilu M, const SweepPlan* P, const double* in, double* out, const double* rdot,
                               double* part, KrylovScalars* sc, const double* rr_part, int rr_n) {
  dfm_ctx c = M->ctx;
  const int ncw = P->cw, nhw = P->hw;
  if (ncw < 1 || nhw < 1 || ncw + nhw > kHaloMaxWarps || (ncw * 32) % LPR) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P->G);
  cfg.blockDim = dim3(32 * (ncw + nhw));
  cfg.dynamicSmemBytes = P->smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  auto go = [&](auto fn) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P->smem);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, fn, (const ChunkDesc*)P->d_chunks, (const unsigned*)P->d_cta_chunk,
                              (const unsigned*)P->d_range, (const unsigned*)P->d_rows, (const char*)P->d_blob,
                              P->stage_bytes, P->nstage, P->x_bytes, P->x_slice, P->halo_stride, ncw, in, out, rdot,
                              part, sc, rr_part, rr_n, c->d_status, (uint64_t)c->wait_ns);
  };
  // forward sweeps carry no fused dot; backward ones take it when asked
  if constexpr (FWD) {
    return go(k_sweep_halo<B, LPR, TV, true, 0>);
  } else {
    if (part) return go(k_sweep_halo<B, LPR, TV, false, DK>);
    return go(k_sweep_halo<B, LPR, TV, false, 0>);
  }
}

template <int B, typename TV, bool FWD, int DK>
static cudaError_t launch_halo_lpr(dfm_ilu M, const SweepPlan* P, const double* in, double* out, const double* rdot,
                                   double* part, KrylovScalars* sc, const double* rr_part, int rr_n) {
  switch (P->lpr) {
    case 2: return launch_halo<B, 2, TV, FWD, DK>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    case 4: return launch_halo<B, 4, TV, FWD, DK>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    default: return launch_halo<B, 8, TV, FWD, DK>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
  }
}

template <typename TV, bool FWD>
static cudaError_t launch_halo_b(dfm_ilu M, const SweepPlan* P, const double* in, double* out, const double* rdot,
                                 double* part, KrylovScalars* sc, const double* rr_part, int rr_n) {
  if (M->vt == DFM_COMPLEX) return launch_halo_lpr<2, TV, FWD, 2>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
  switch (M->b) {
    case 1: return launch_halo_lpr<1, TV, FWD, 1>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    case 2: return launch_halo_lpr<2, TV, FWD, 1>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    default: return launch_halo_lpr<3, TV, FWD, 1>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
  }
}

cudaError_t sweep_halo_launch(dfm_ilu M, bool fwd, const SweepPlan* P, const double* in, double* out,
                              const double* rdot, double* part, KrylovScalars* sc, const double* rr_part, int rr_n,
                              bool f32) {
  if (f32)
    return fwd ? launch_halo_b<float, true>(M, P, in, out, rdot, part, sc, rr_part, rr_n)
               : launch_halo_b<float, false>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
  return fwd ? launch_halo_b<double, true>(M, P, in, out, rdot, part, sc, rr_part, rr_n)
             : launch_halo_b<double, false>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
}

}  // namespace dfm
