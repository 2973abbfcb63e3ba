// Range-partitioned ILU(0) triangular sweeps (schedule mode 3).
//
// The rows are split into G contiguous ranges, one per CTA (a persistent,
// co-resident grid).  A CTA walks its range level by level (a level's rows are
// independent): a dependency on a row of its own range is always on an earlier
// level and is read from the CTA's shared-memory copy of the range's vector
// slice; a dependency on another range is polled in global memory, where the
// owning CTA publishes each row as soon as it is computed (the output vector
// starts as a NaN sentinel).  With the reference's natural FEM ordering most
// dependencies are local, so most steps of the critical path cost a CTA
// barrier plus shared-memory latency instead of a round trip through L2.
//
// Everything a level needs (a 16-byte descriptor per row, the shared-memory
// offset or global row of every block's operand, factor blocks, D^-1 for the
// forward sweep) is packed per "chunk" (a level, or a slice of one) into one
// contiguous, 16-byte aligned blob in chunk order and streamed into a ring of
// shared-memory stages by TMA bulk copies (cp.async.bulk, no multicast)
// completing on mbarriers, several chunks ahead.  Thread 0 alone drives the
// ring: before each level barrier it makes sure the next chunk has landed, and
// after it refills the stage just released.  The per-level path of every other
// thread is one descriptor load, its blocks, and the barrier.  The blob's
// values are re-gathered from the factor after every numeric factorisation.
//
// Every row waits only for rows of lower level, each CTA handles its chunks in
// increasing level order and all CTAs are co-resident, so every wait ends
// (induction on the level); all waits are also bounded.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "dfm_internal.h"
#include "sweep.h"
#include "sweep_dev.cuh"

namespace dfm {

constexpr int kStageThread = kSweepThreads - 32;  // drives the stage ring of the range sweep

// ------------------------------------------------- row helpers (mode 3)
// A row's first batch of operands as issued ahead of time: codes and values
// (remote and input-vector entries loaded, local ones filled in later).
template <int B, typename TX>
struct RowPF {
  bool valid;
  uint4 rd;
  unsigned xo[kOpBatch];
  TX xv[kOpBatch][B];
};

template <int B, int LPR, typename TX>
DFM_DEVINL void row_prefetch(const char* sb, unsigned r, int lane, const TX* __restrict__ in, const TX* out,
                             RowPF<B, TX>& pf) {
  const ChunkHeader* hdr = reinterpret_cast<const ChunkHeader*>(sb);
  const unsigned* xoff = reinterpret_cast<const unsigned*>(sb + hdr->xoff);
  pf.rd = reinterpret_cast<const uint4*>(sb + 32)[r];
  pf.valid = true;
#pragma unroll
  for (int u = 0; u < kOpBatch; u++) {
    const unsigned kk = pf.rd.y + lane + u * LPR;
    pf.xo[u] = kk < pf.rd.z ? xoff[kk] : 0xffffffffu;
  }
#pragma unroll
  for (int u = 0; u < kOpBatch; u++) {
    const unsigned o = pf.xo[u];
    if (o != 0xffffffffu && (o & 0x40000000u)) {  // an entry of the input vector (merged level pairs)
#pragma unroll
      for (int c = 0; c < B; c++) pf.xv[u][c] = __ldg(in + (size_t)(o & 0x3fffffffu) * B + c);
    } else if (o != 0xffffffffu && (o & 0x80000000u)) {  // another range's row (may not be published yet)
#pragma unroll
      for (int c = 0; c < B; c++) pf.xv[u][c] = ld_relaxed(out + (size_t)(o & 0x7fffffffu) * B + c);
    } else {
#pragma unroll
      for (int c = 0; c < B; c++) pf.xv[u][c] = (TX)0;
    }
  }
}

// Finishes a prefetched row: local operands, re-polls, the remaining operand
// batches, the group reduction and the row's output (slice and global).
template <int B, int LPR, typename TV, typename TX, bool FWD>
DFM_DEVINL void row_finish(const char* sb, unsigned r, int lane, unsigned gmask, unsigned a0, TX* X,
                           const TX* __restrict__ in, TX* out, RowPF<B, TX>& pf, DevStatus* st, uint64_t wait_ns) {
  constexpr int BB = B * B;
  const ChunkHeader* hdr = reinterpret_cast<const ChunkHeader*>(sb);
  const unsigned* xoff = reinterpret_cast<const unsigned*>(sb + hdr->xoff);
  const TV* vals = reinterpret_cast<const TV*>(sb + hdr->vals);
  const uint4 rd = pf.rd;
  double acc[B];
#pragma unroll
  for (int c = 0; c < B; c++) acc[c] = 0.0;
  // first batch: prefetched codes
#pragma unroll
  for (int u = 0; u < kOpBatch; u++) {
    const unsigned o = pf.xo[u];
    if (o != 0xffffffffu && (o & 0xc0000000u) == 0u)
#pragma unroll
      for (int c = 0; c < B; c++) pf.xv[u][c] = X[o + c];
  }
  repoll_batch<B, kOpBatch, TX>(pf.xo, pf.xv, out, st, wait_ns, FWD ? 11 : 12);
#pragma unroll
  for (int u = 0; u < kOpBatch; u++) {
    const unsigned kk = rd.y + lane + u * LPR;
    if (kk >= rd.z) break;
    const TV* m = vals + (size_t)kk * BB;
#pragma unroll
    for (int rr = 0; rr < B; rr++)
#pragma unroll
      for (int c = 0; c < B; c++) acc[rr] += (double)m[rr * B + c] * (double)pf.xv[u][c];
  }
  // remaining batches (rows with more than kOpBatch * LPR operands)
  for (unsigned kb = rd.y + lane + kOpBatch * LPR; kb < rd.z; kb += kOpBatch * LPR) {
    unsigned xo[kOpBatch];
    TX xv[kOpBatch][B];
#pragma unroll
    for (int u = 0; u < kOpBatch; u++) {
      const unsigned kk = kb + u * LPR;
      xo[u] = kk < rd.z ? xoff[kk] : 0xffffffffu;
    }
#pragma unroll
    for (int u = 0; u < kOpBatch; u++) {
      const unsigned o = xo[u];
      if (o == 0xffffffffu) {
#pragma unroll
        for (int c = 0; c < B; c++) xv[u][c] = (TX)0;
      } else if (o & 0x40000000u) {
#pragma unroll
        for (int c = 0; c < B; c++) xv[u][c] = __ldg(in + (size_t)(o & 0x3fffffffu) * B + c);
      } else if (o & 0x80000000u) {
#pragma unroll
        for (int c = 0; c < B; c++) xv[u][c] = ld_relaxed(out + (size_t)(o & 0x7fffffffu) * B + c);
      } else {
#pragma unroll
        for (int c = 0; c < B; c++) xv[u][c] = X[o + c];
      }
    }
    repoll_batch<B, kOpBatch, TX>(xo, xv, out, st, wait_ns, FWD ? 11 : 12);
#pragma unroll
    for (int u = 0; u < kOpBatch; u++) {
      const unsigned kk = kb + u * LPR;
      if (kk >= rd.z) break;
      const TV* m = vals + (size_t)kk * BB;
#pragma unroll
      for (int rr = 0; rr < B; rr++)
#pragma unroll
        for (int c = 0; c < B; c++) acc[rr] += (double)m[rr * B + c] * (double)xv[u][c];
    }
  }
  if (LPR > 1) {
#pragma unroll
    for (int rr = 0; rr < B; rr++)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[rr] += __shfl_xor_sync(gmask, acc[rr], o);
  }
  if (lane == 0) {
    TX* xi = X + rd.x * B;
    double t[B];
#pragma unroll
    for (int rr = 0; rr < B; rr++) t[rr] = (double)xi[rr] - acc[rr];
    TX o[B];
    if (FWD) {
      const double* d = reinterpret_cast<const double*>(sb + hdr->dinv) + (size_t)r * BB;
#pragma unroll
      for (int rr = 0; rr < B; rr++) {
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < B; c++) v += d[rr * B + c] * t[c];
        o[rr] = (TX)v;
      }
    } else {
#pragma unroll
      for (int rr = 0; rr < B; rr++) o[rr] = (TX)t[rr];
    }
#pragma unroll
    for (int rr = 0; rr < B; rr++) {
      xi[rr] = o[rr];
      st_relaxed(out + (size_t)rd.w * B + rr, o[rr]);
    }
  }
}

// --------------------------------------------------------------- kernel
template <int B, int LPR, typename TV, typename TX, bool FWD, int DOT, bool PIPE>
__global__ void __launch_bounds__(kSweepThreads, 1)
k_sweep_ranges(const ChunkDesc* __restrict__ chunks, const unsigned* __restrict__ cta_chunk,
               const unsigned* __restrict__ range, const unsigned* __restrict__ rows,
               const char* __restrict__ blob, unsigned stage_bytes,
               int nstage, unsigned x_bytes, const TX* __restrict__ in, TX* out, const TX* __restrict__ rdot,
               double* part, KrylovScalars* sc, const double* rr_part, int rr_nparts, DevStatus* st,
               uint64_t wait_ns) {
  extern __shared__ __align__(128) char smem[];
  __shared__ int s_alive;
  // guards (block-uniform)
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
  const unsigned len = a1 - a0;
  TX* X = reinterpret_cast<TX*>(smem);
  char* stages = smem + x_bytes;
  uint64_t* bar_data = reinterpret_cast<uint64_t*>(stages + (size_t)nstage * stage_bytes);

  unsigned issued_end = q0;  // stage thread: chunks [q0, issued_end) requested
  if (threadIdx.x == kStageThread) {
    s_alive = 1;
    for (int s = 0; s < nstage; s++) mbar_init(&bar_data[s], 1);
    fence_mbar_init();
    for (unsigned q = q0; q < q1 && q < q0 + (unsigned)nstage; q++) {
      const ChunkDesc cd = chunks[q];
      const int s = (int)((q - q0) % (unsigned)nstage);
      mbar_arrive_tx(&bar_data[s], cd.bytes);
      bulk_g2s(stages + (size_t)s * stage_bytes, blob + cd.off, cd.bytes, &bar_data[s]);
      issued_end = q + 1;
    }
  }
  // X slice <- in[a0:a1) while the first chunks are in flight (rows
  // overwrite their entry with the output)
  load_slice<B, 8>(X, in, rows, a0, len);
  if (threadIdx.x == kStageThread && q0 < q1 && !wait_stage(&bar_data[0], 0u, st, wait_ns)) s_alive = 0;
  __syncthreads();
  const int lane = threadIdx.x % LPR;
  const unsigned g = threadIdx.x / LPR, ng = kSweepThreads / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  if constexpr (PIPE) {
  // Software pipeline across levels: the lane groups form two halves that
  // take alternate levels.  While one half computes level k, the other waits
  // for level k+1's stage and, for its first row there, reads the descriptor
  // and operand offsets and issues the remote and input-vector loads; after
  // the barrier that ends level k it only loads its local operands, re-polls
  // a remote value that was not yet published, and finishes the row.
  const unsigned half = ng / 2, h = g >= half ? 1u : 0u, gl = g - h * half;
  RowPF<B, TX> pf;
  pf.valid = false;
  if (s_alive && q0 < q1 && h == 0 && gl < reinterpret_cast<const ChunkHeader*>(stages)->nrows)
    row_prefetch<B, LPR, TX>(stages, gl, lane, in, out, pf);
  for (unsigned q = q0; q < q1; q++) {
    const unsigned k = q - q0;
    const int s = (int)(k % (unsigned)nstage);
    const char* sb = stages + (size_t)s * stage_bytes;
    if (s_alive && h == (k & 1u)) {  // this half computes level k
      const unsigned nrows = reinterpret_cast<const ChunkHeader*>(sb)->nrows;
      if (pf.valid) row_finish<B, LPR, TV, TX, FWD>(sb, gl, lane, gmask, a0, X, in, out, pf, st, wait_ns);
      pf.valid = false;
      for (unsigned r = gl + half; r < nrows; r += half) {  // more rows than the half has groups
        RowPF<B, TX> ex;
        row_prefetch<B, LPR, TX>(sb, r, lane, in, out, ex);
        row_finish<B, LPR, TV, TX, FWD>(sb, r, lane, gmask, a0, X, in, out, ex, st, wait_ns);
      }
    } else if (s_alive && q + 1 < q1) {  // the other half prepares level k+1
      const unsigned k1 = k + 1;
      const int s1 = (int)(k1 % (unsigned)nstage);
      if (!wait_stage(&bar_data[s1], (k1 / (unsigned)nstage) & 1u, st, wait_ns)) s_alive = 0;
      const char* sb1 = stages + (size_t)s1 * stage_bytes;
      if (s_alive && gl < reinterpret_cast<const ChunkHeader*>(sb1)->nrows)
        row_prefetch<B, LPR, TX>(sb1, gl, lane, in, out, pf);
    }
    __syncthreads();  // level done: slice entries visible, stage s free
    if (threadIdx.x == kStageThread && s_alive) {
      const ChunkHeader* hdr = reinterpret_cast<const ChunkHeader*>(sb);
      if (hdr->next_bytes) {
        mbar_arrive_tx(&bar_data[s], hdr->next_bytes);
        bulk_g2s(stages + (size_t)s * stage_bytes, blob + hdr->next_off, hdr->next_bytes, &bar_data[s]);
        issued_end = q + nstage + 1;
      }
    }
  }
  } else {  // every group loads its rows after the level barrier
  for (unsigned q = q0; q < q1; q++) {
    const unsigned k = q - q0;
    const int s = (int)(k % (unsigned)nstage);
    const char* sb = stages + (size_t)s * stage_bytes;
    if (s_alive) {
      const ChunkHeader* hdr = reinterpret_cast<const ChunkHeader*>(sb);
      const unsigned nrows = hdr->nrows;
      const uint4* rdesc = reinterpret_cast<const uint4*>(sb + 32);
      const unsigned* xoff = reinterpret_cast<const unsigned*>(sb + hdr->xoff);
      const TV* vals = reinterpret_cast<const TV*>(sb + hdr->vals);
      const double* dinv = reinterpret_cast<const double*>(sb + hdr->dinv);
      constexpr int BB = B * B;
      for (unsigned r = g; r < nrows; r += ng) {  // uniform within a group (lanes share r)
        const uint4 rd = rdesc[r];
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; c++) acc[c] = 0.0;
        // a lane's operands in batches of kOpBatch: every load of a batch is
        // issued before any is waited on, so remote operands cost one round
        // trip per batch instead of one each
        for (unsigned kb = rd.y + lane; kb < rd.z; kb += kOpBatch * LPR) {
          unsigned xo[kOpBatch];
          TX xv[kOpBatch][B];
#pragma unroll
          for (int u = 0; u < kOpBatch; u++) {
            const unsigned kk = kb + u * LPR;
            xo[u] = kk < rd.z ? xoff[kk] : 0xffffffffu;
          }
#pragma unroll
          for (int u = 0; u < kOpBatch; u++) {
            const unsigned o = xo[u];
            if (o == 0xffffffffu) {
#pragma unroll
              for (int c = 0; c < B; c++) xv[u][c] = (TX)0;
            } else if (o & 0x40000000u) {  // an entry of the input vector (merged level pairs)
#pragma unroll
              for (int c = 0; c < B; c++) xv[u][c] = __ldg(in + (size_t)(o & 0x3fffffffu) * B + c);
            } else if (o & 0x80000000u) {  // another range's row: its published value (may not be ready)
#pragma unroll
              for (int c = 0; c < B; c++) xv[u][c] = ld_relaxed(out + (size_t)(o & 0x7fffffffu) * B + c);
            } else {
#pragma unroll
              for (int c = 0; c < B; c++) xv[u][c] = X[o + c];
            }
          }
          repoll_batch<B, kOpBatch, TX>(xo, xv, out, st, wait_ns, FWD ? 11 : 12);
#pragma unroll
          for (int u = 0; u < kOpBatch; u++) {
            const unsigned kk = kb + u * LPR;
            if (kk >= rd.z) break;
            const TV* m = vals + (size_t)kk * BB;
#pragma unroll
            for (int rr = 0; rr < B; rr++)
#pragma unroll
              for (int c = 0; c < B; c++) acc[rr] += (double)m[rr * B + c] * (double)xv[u][c];
          }
        }
        if (LPR > 1) {
#pragma unroll
          for (int rr = 0; rr < B; rr++)
#pragma unroll
            for (int o = LPR / 2; o > 0; o >>= 1) acc[rr] += __shfl_xor_sync(gmask, acc[rr], o);
        }
        if (lane == 0) {
          TX* xi = X + rd.x * B;
          double t[B];
#pragma unroll
          for (int rr = 0; rr < B; rr++) t[rr] = (double)xi[rr] - acc[rr];
          TX o[B];
          if (FWD) {
            const double* d = dinv + (size_t)r * BB;
#pragma unroll
            for (int rr = 0; rr < B; rr++) {
              double v = 0.0;
#pragma unroll
              for (int c = 0; c < B; c++) v += d[rr * B + c] * t[c];
              o[rr] = (TX)v;
            }
          } else {
#pragma unroll
            for (int rr = 0; rr < B; rr++) o[rr] = (TX)t[rr];
          }
#pragma unroll
          for (int rr = 0; rr < B; rr++) {
            xi[rr] = o[rr];
            st_relaxed(out + (size_t)rd.w * B + rr, o[rr]);
          }
        }
      }
    }
    // the stage thread (lane 0 of the last warp, which rarely has rows): the next
    // level's chunk must have landed before the barrier
    if (threadIdx.x == kStageThread && s_alive && q + 1 < q1) {
      const unsigned k1 = k + 1;
      if (!wait_stage(&bar_data[k1 % (unsigned)nstage], (k1 / (unsigned)nstage) & 1u, st, wait_ns)) s_alive = 0;
    }
    __syncthreads();  // level done: slice entries visible, stage s free
    if (threadIdx.x == kStageThread && s_alive) {
      const ChunkHeader* hdr = reinterpret_cast<const ChunkHeader*>(sb);
      if (hdr->next_bytes) {
        mbar_arrive_tx(&bar_data[s], hdr->next_bytes);
        bulk_g2s(stages + (size_t)s * stage_bytes, blob + hdr->next_off, hdr->next_bytes, &bar_data[s]);
        issued_end = q + nstage + 1;
      }
    }
  }
  }
  if (DOT) range_dot<B, DOT, TX>(rdot, X, a0, len, true, part, rows);  // (rdot, out) over this CTA's range
  // after an aborted wait, copies already requested must land before the CTA exits
  if (threadIdx.x == kStageThread && !s_alive) {
    for (unsigned q = q0; q < issued_end; q++) {
      const unsigned k = q - q0;
      (void)wait_stage(&bar_data[k % (unsigned)nstage], (k / (unsigned)nstage) & 1u, st, wait_ns);
    }
  }
}

// ------------------------------------------------ barrier-free variant
// The same plan, without the per-level CTA barrier: the CTA's rows (in chunk,
// i.e. level, order) are dealt round-robin to the lane groups, and each row
// waits only for its own operands - a local one until its shared-memory slot
// (initialised to the sentinel) holds a value, a remote one in global memory as
// before.  Rows of consecutive levels therefore overlap.  A stage is released
// when its chunk's last row completes (a shared-memory counter): the thread
// that completes it records which chunk the stage will hold next and issues
// that chunk's bulk copy.  A group reading a chunk first waits until the stage
// is assigned to that chunk, then for the copy's mbarrier phase.  Every wait is
// bounded; after an expired wait the CTA stops and drains its copies.
template <typename TX>
DFM_DEVINL TX poll_local(const TX* p, volatile int* alive, DevStatus* st, uint64_t wait_ns) {
  TX v = ld_volatile_s(p);
  if (!Sent<TX>::is(v)) return v;
  SpinGuard g(wait_ns);
  for (;;) {
    v = ld_volatile_s(p);
    if (!Sent<TX>::is(v)) return v;
    if (!*alive) return v;
    if (g.expired()) {
      raise_error(st, DFM_WAIT_TIMEOUT, 13);
      *alive = 0;
      return v;
    }
  }
}

template <int B, int LPR, typename TV, typename TX, bool FWD, int DOT>
__global__ void __launch_bounds__(kSweepThreads, 1)
k_sweep_ranges_nb(const ChunkDesc* __restrict__ chunks, const unsigned* __restrict__ cta_chunk,
                  const unsigned* __restrict__ range, const unsigned* __restrict__ rows,
                  const char* __restrict__ blob, unsigned stage_bytes,
                  int nstage, unsigned x_bytes, unsigned max_chunks, const TX* __restrict__ in, TX* out,
                  const TX* __restrict__ rdot, double* part, KrylovScalars* sc, const double* rr_part,
                  int rr_nparts, DevStatus* st, uint64_t wait_ns) {
  constexpr int BB = B * B;
  extern __shared__ __align__(128) char smem[];
  __shared__ int s_alive;
  __shared__ int s_issued[kMaxStages];      // chunk (CTA-local index) a stage holds or is loading
  __shared__ unsigned s_done[kMaxStages];   // rows of that chunk completed
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
  TX* X = reinterpret_cast<TX*>(smem);
  char* stages = smem + x_bytes;
  uint64_t* bar = reinterpret_cast<uint64_t*>(stages + (size_t)nstage * stage_bytes);
  unsigned* rowpre = reinterpret_cast<unsigned*>(bar + kMaxStages);  // K + 1 prefix row counts
  volatile int* alive = &s_alive;

  for (unsigned k = threadIdx.x; k < len * B; k += blockDim.x) X[k] = Sent<TX>::value();
  if (threadIdx.x == 0) {  // prefix of rows per chunk (K is at most max_chunks)
    unsigned acc = 0;
    for (unsigned k = 0; k < K && k < max_chunks; k++) {
      rowpre[k] = acc;
      acc += chunks[q0 + k].nrows;
    }
    rowpre[K < max_chunks ? K : max_chunks] = acc;
    s_alive = K <= max_chunks ? 1 : 0;
    if (K > max_chunks) raise_error(st, DFM_ERR_INVALID, 14);
    for (int s = 0; s < nstage; s++) {
      mbar_init(&bar[s], 1);
      s_issued[s] = -1;
      s_done[s] = 0;
    }
    fence_mbar_init();
    if (s_alive)
      for (unsigned k = 0; k < K && k < (unsigned)nstage; k++) {
        const ChunkDesc cd = chunks[q0 + k];
        s_issued[k] = (int)k;
        mbar_arrive_tx(&bar[k], cd.bytes);
        bulk_g2s(stages + (size_t)k * stage_bytes, blob + cd.off, cd.bytes, &bar[k]);
      }
  }
  __syncthreads();
  const int lane = threadIdx.x % LPR;
  const unsigned g = threadIdx.x / LPR, ng = kSweepThreads / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  const unsigned R = s_alive ? rowpre[K] : 0u;
  unsigned k = 0;
  for (unsigned t = g; t < R; t += ng) {
    while (rowpre[k + 1] <= t) k++;  // group-uniform
    const int s = (int)(k % (unsigned)nstage);
    // the stage must hold chunk k, and its copy must have landed
    bool ok = true;
    if (*reinterpret_cast<volatile int*>(&s_issued[s]) != (int)k) {
      SpinGuard gd(wait_ns);
      while (*reinterpret_cast<volatile int*>(&s_issued[s]) != (int)k) {
        if (!*alive) { ok = false; break; }
        if (gd.expired()) {
          raise_error(st, DFM_WAIT_TIMEOUT, 15);
          *alive = 0;
          ok = false;
          break;
        }
      }
    }
    if (ok && !mbar_try_wait(&bar[s], (k / (unsigned)nstage) & 1u)) {
      SpinGuard gd(wait_ns);
      while (!mbar_try_wait(&bar[s], (k / (unsigned)nstage) & 1u)) {
        if (!*alive) { ok = false; break; }
        if (gd.expired()) {
          raise_error(st, DFM_WAIT_TIMEOUT, 16);
          *alive = 0;
          ok = false;
          break;
        }
      }
    }
    ok = __all_sync(gmask, ok) != 0;  // group-uniform decision (only the group's lanes vote)
    if (!ok) break;
    const char* sb = stages + (size_t)s * stage_bytes;
    const ChunkHeader* hdr = reinterpret_cast<const ChunkHeader*>(sb);
    const unsigned r = t - rowpre[k];
    const uint4 rd = reinterpret_cast<const uint4*>(sb + 32)[r];
    const unsigned* xoff = reinterpret_cast<const unsigned*>(sb + hdr->xoff);
    const TV* vals = reinterpret_cast<const TV*>(sb + hdr->vals);
    TX vin[B];
    if (lane == 0)
#pragma unroll
      for (int c = 0; c < B; c++) vin[c] = in[(size_t)rd.w * B + c];
    double acc[B];
#pragma unroll
    for (int c = 0; c < B; c++) acc[c] = 0.0;
    for (unsigned kk = rd.y + lane; kk < rd.z; kk += LPR) {
      const unsigned xo = xoff[kk];
      TX xv[B];
      if (xo & 0x40000000u) {  // an entry of the input vector (merged level pairs)
        const unsigned col = xo & 0x3fffffffu;
#pragma unroll
        for (int c = 0; c < B; c++) xv[c] = __ldg(in + (size_t)col * B + c);
      } else if (xo & 0x80000000u) {
        const unsigned col = xo & 0x7fffffffu;
#pragma unroll
        for (int c = 0; c < B; c++) xv[c] = ld_relaxed(out + (size_t)col * B + c);
        repoll_batch<B, 1, TX>(&xo, reinterpret_cast<TX(*)[B]>(xv), out, st, wait_ns, FWD ? 11 : 12);
      } else {
#pragma unroll
        for (int c = 0; c < B; c++) xv[c] = poll_local(X + xo + c, alive, st, wait_ns);
      }
      const TV* m = vals + (size_t)kk * BB;
#pragma unroll
      for (int rr = 0; rr < B; rr++)
#pragma unroll
        for (int c = 0; c < B; c++) acc[rr] += (double)m[rr * B + c] * (double)xv[c];
    }
    if (LPR > 1) {
#pragma unroll
      for (int rr = 0; rr < B; rr++)
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) acc[rr] += __shfl_xor_sync(gmask, acc[rr], o);
    }
    if (lane == 0) {
      double tt[B];
#pragma unroll
      for (int rr = 0; rr < B; rr++) tt[rr] = (double)vin[rr] - acc[rr];
      TX o[B];
      if (FWD) {
        const double* d = reinterpret_cast<const double*>(sb + hdr->dinv) + (size_t)r * BB;
#pragma unroll
        for (int rr = 0; rr < B; rr++) {
          double v = 0.0;
#pragma unroll
          for (int c = 0; c < B; c++) v += d[rr * B + c] * tt[c];
          o[rr] = (TX)v;
        }
      } else {
#pragma unroll
        for (int rr = 0; rr < B; rr++) o[rr] = (TX)tt[rr];
      }
#pragma unroll
      for (int rr = 0; rr < B; rr++) {
        st_relaxed(out + (size_t)rd.w * B + rr, o[rr]);
        st_volatile_s(X + rd.x * B + rr, o[rr]);
      }
      // release the stage after the chunk's last row (its reads are all done:
      // every lane of this group passed the shuffles above)
      __threadfence_block();
      const unsigned old = atomicAdd(&s_done[s], 1u);
      if (old + 1 == hdr->nrows) {
        __threadfence_block();
        s_done[s] = 0;
        const unsigned nb = hdr->next_bytes;
        if (nb && *alive) {
          const unsigned long long noff = hdr->next_off;
          const unsigned k2 = k + (unsigned)nstage;
          fence_proxy_async_smem();
          *reinterpret_cast<volatile int*>(&s_issued[s]) = (int)k2;
          mbar_arrive_tx(&bar[s], nb);
          bulk_g2s(stages + (size_t)s * stage_bytes, blob + noff, nb, &bar[s]);
        }
      }
    }
    __syncwarp(gmask);
  }
  __syncthreads();
  if (DOT) range_dot<B, DOT, TX>(rdot, X, a0, len, s_alive != 0, part, rows);
  // every stage's last issued copy must have landed before the CTA exits
  if (threadIdx.x == 0)
    for (int s2 = 0; s2 < nstage; s2++) {
      const int kl = s_issued[s2];
      if (kl >= 0) (void)wait_stage(&bar[s2], ((unsigned)kl / (unsigned)nstage) & 1u, st, wait_ns);
    }
}

// Refreshes the blob's values from the factor after a numeric factorisation.
// Every packed block has a recipe {base, t0, t1, sign}:
//   value = (base != NONE ? F[base] : 0) + sign * sum_{t0 <= t < t1} F[s1] (D_j^-1) (F[s2])
// with a term {s1, j, s2} (j or s2 NONE = identity), F the factor's off-diagonal
// blocks.  Plain operands are copies (no terms); the merged plans' operands of
// the second level of a pair are the products L_ij D_j^-1 (forward input
// terms), U'_ij (backward input terms) and the fill blocks
// F_ik - sum_j F_ij (D_j^-1) F_jk.  One thread per packed block; D^-1 rows of the
// forward sweep are copied alongside.  CPLX: the factor holds complex scalars
// (re, im), packed as the real 2x2 blocks [re -im; im re] (B = 2), whose
// products are the complex products.
template <int B, bool CPLX>
DFM_DEVINL void load_factor_blk(const double* __restrict__ src, size_t k, double* v) {
  if constexpr (CPLX) {
    const double re = src[2 * k], im = src[2 * k + 1];
    v[0] = re;
    v[1] = -im;
    v[2] = im;
    v[3] = re;
  } else {
#pragma unroll
    for (int e = 0; e < B * B; e++) v[e] = src[k * (B * B) + e];
  }
}

template <int B, typename TV, bool CPLX>
__global__ void k_gather_recipes(const ChunkDesc* __restrict__ chunks, unsigned nchunks,
                                 const uint4* __restrict__ recipe, const uint4* __restrict__ terms,
                                 const double* __restrict__ fdiag, const double* __restrict__ foff, char* blob,
                                 int with_dinv) {
  static_assert(!CPLX || B == 2, "complex scalars pack as 2x2 blocks");
  constexpr int BB = B * B;
  constexpr unsigned NONE = 0xffffffffu;
  for (unsigned q = blockIdx.x; q < nchunks; q += gridDim.x) {
    const ChunkDesc cd = chunks[q];
    char* base = blob + cd.off;
    TV* vals = reinterpret_cast<TV*>(base + cd.vals_off);
    for (unsigned k = threadIdx.x; k < cd.nblk_pad; k += blockDim.x) {
      const uint4 rc = recipe[cd.blk0 + k];
      double v[BB];
      if (rc.x != NONE) {
        load_factor_blk<B, CPLX>(foff, rc.x, v);
      } else {
#pragma unroll
        for (int e = 0; e < BB; e++) v[e] = 0.0;
      }
      const double sg = rc.w ? -1.0 : 1.0;
      for (unsigned t = rc.y; t < rc.z; t++) {
        const uint4 tm = terms[t];
        double a[BB], m[BB], d[BB];
        load_factor_blk<B, CPLX>(foff, tm.x, a);
        if (tm.y != NONE) {  // a = a * D_j^-1
          load_factor_blk<B, CPLX>(fdiag, tm.y, d);
#pragma unroll
          for (int r = 0; r < B; r++)
#pragma unroll
            for (int c = 0; c < B; c++) {
              double acc = 0.0;
#pragma unroll
              for (int l = 0; l < B; l++) acc += a[r * B + l] * d[l * B + c];
              m[r * B + c] = acc;
            }
#pragma unroll
          for (int e = 0; e < BB; e++) a[e] = m[e];
        }
        if (tm.z != NONE) {  // a = a * F[s2]
          double f[BB];
          load_factor_blk<B, CPLX>(foff, tm.z, f);
#pragma unroll
          for (int r = 0; r < B; r++)
#pragma unroll
            for (int c = 0; c < B; c++) {
              double acc = 0.0;
#pragma unroll
              for (int l = 0; l < B; l++) acc += a[r * B + l] * f[l * B + c];
              m[r * B + c] = acc;
            }
#pragma unroll
          for (int e = 0; e < BB; e++) a[e] = m[e];
        }
#pragma unroll
        for (int e = 0; e < BB; e++) v[e] += sg * a[e];
      }
#pragma unroll
      for (int e = 0; e < BB; e++) vals[(size_t)k * BB + e] = (TV)v[e];
    }
    if (with_dinv) {
      const uint4* rd = reinterpret_cast<const uint4*>(base + 32);
      double* dinv = reinterpret_cast<double*>(base + cd.dinv_off);
      for (unsigned r = threadIdx.x; r < cd.nrows; r += blockDim.x) {
        double v[BB];
        load_factor_blk<B, CPLX>(fdiag, (size_t)rd[r].w, v);  // w: the row's global index
#pragma unroll
        for (int e = 0; e < BB; e++) dinv[(size_t)r * BB + e] = v[e];
      }
    }
  }
}

// ------------------------------------------------------------- host plan
void sweep_plan_free(SweepPlan* P) {
  if (!P) return;
  cudaFree(P->d_chunks);
  cudaFree(P->d_cta_chunk);
  cudaFree(P->d_range);
  cudaFree(P->d_rows);
  cudaFree(P->d_blob);
  cudaFree(P->d_recipe);
  cudaFree(P->d_terms);
  *P = SweepPlan();
}

int sweep_plan_build(dfm_ilu M, bool fwd, int G, int val_bytes, int vec_bytes, SweepPlan* P, bool merge,
                     bool part, bool halo) {
  if (halo) {
    if (vec_bytes != 8) return DFM_ERR_UNSUPPORTED;
    return sweep_halo_plan_build(M, fwd, G, val_bytes, P, part, merge);
  }
  const unsigned N = M->N;
  const unsigned b = M->vt == DFM_COMPLEX ? 2u : M->b;  // complex scalars as real 2x2 blocks
  const unsigned bb = b * b;
  const unsigned vblk = (unsigned)val_bytes * bb;     // bytes per packed block
  const unsigned drow = fwd ? 8u * bb : 0u;           // D^-1 bytes per row (FP64)
  const std::vector<unsigned>& rp = M->A->h_rowptr;
  const std::vector<unsigned>& ci = M->A->h_colind;
  const std::vector<unsigned>& dia = M->h_diaind;
  const std::vector<unsigned>& lev = fwd ? M->lev_f : M->lev_b;
  sweep_plan_free(P);
  if (N >= 0x40000000u) return DFM_ERR_UNSUPPORTED;  // operand encodings use the top two bits
  // Rows are laid out in an order of positions; CTA c owns the positions
  // [range[c], range[c+1]) and keeps their vector entries in its slice in that
  // order.  Natural order: positions are rows, ranges balanced by (dependency
  // blocks + 1) per row.  With the ILU's row partition: the rows of part c,
  // ascending, are CTA c's positions.
  std::vector<unsigned> order, pos;  // position -> row, row -> position (empty: the identity)
  std::vector<unsigned> range;
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
    if ((unsigned)G > std::max(N, 1u)) G = std::max(N, 1u);
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
  const size_t x_bytes = ((size_t)maxlen * b * vec_bytes + 127) & ~(size_t)127;
  if (x_bytes + 4 * 1024 > kSweepSmemBudget) return DFM_ERR_UNSUPPORTED;  // use more CTAs

  struct Pend {
    std::vector<uint4> rd;
    std::vector<unsigned> xo;
  };
  std::vector<ChunkDesc> chunks;
  std::vector<Pend> pend;
  std::vector<unsigned> cta_chunk(G + 1, 0);
  std::vector<uint4> recipe, terms;
  size_t blob_size = 0;
  unsigned stage_max = 0;
  constexpr unsigned NONE = 0xffffffffu;
  // step of a row: its level, or with merged level pairs its level / 2
  auto step = [&](unsigned i) { return merge ? lev[i] / 2 : lev[i]; };
  // operands of row i: {encoded operand, recipe}.  Encoding: local slice
  // offset, 0x80000000|row (an output of another range), 0x40000000|row (an
  // entry of the input vector).
  struct Op { unsigned xo; uint4 rc; };
  std::vector<Op> ops;
  std::vector<unsigned> kmap(N, NONE);  // scratch: column -> position in ops
  auto slots = [&](unsigned i, unsigned& s0, unsigned& s1) {
    s0 = fwd ? rp[i] : dia[i];
    s1 = fwd ? dia[i] : rp[i + 1];
  };
  auto row_ops = [&](unsigned i, unsigned a0, unsigned a1) {
    ops.clear();
    unsigned s0, s1;
    slots(i, s0, s1);
    auto out_code = [&](unsigned col) {
      const unsigned p = pos_of(col);
      return (p >= a0 && p < a1) ? (p - a0) * b : (0x80000000u | col);
    };
    const bool second = merge && (lev[i] & 1u);
    if (!second) {
      for (unsigned s = s0; s < s1; s++) ops.push_back({out_code(ci[s]), make_uint4(s, 0u, 0u, 0u)});
      return;
    }
    // second level of a pair: operands on the first level are substituted
    for (unsigned s = s0; s < s1; s++) {
      const unsigned j = ci[s];
      if (lev[j] + 1 != lev[i]) continue;
      const unsigned t0 = (unsigned)terms.size();
      terms.push_back(make_uint4(s, fwd ? j : NONE, NONE, 0u));  // L_ij D_j^-1  |  U'_ij
      ops.push_back({0x40000000u | j, make_uint4(NONE, t0, t0 + 1, 0u)});
    }
    const size_t first_c = ops.size();
    for (unsigned s = s0; s < s1; s++) {
      const unsigned k = ci[s];
      if (lev[k] + 1 == lev[i]) continue;
      kmap[k] = (unsigned)ops.size();
      ops.push_back({out_code(k), make_uint4(s, 0u, 0u, 1u)});
    }
    // fill terms, grouped per column
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
          ops.push_back({out_code(k), make_uint4(NONE, 0u, 0u, 1u)});
          tl.emplace_back();
        }
        tl[kmap[k] - first_c].push_back(make_uint4(s, fwd ? j : NONE, t, 0u));
      }
    }
    for (size_t q = first_c; q < ops.size(); q++) {
      const unsigned t0 = (unsigned)terms.size();
      for (const uint4& t : tl[q - first_c]) terms.push_back(t);
      ops[q].rc.y = t0;
      ops[q].rc.z = (unsigned)terms.size();
      // an operand with neither base nor terms cannot occur (each came from one)
    }
    for (size_t q = first_c; q < ops.size(); q++) {
      unsigned col;
      const unsigned code = ops[q].xo;
      if (code & 0x80000000u) col = code & 0x3fffffffu;
      else col = row_at(a0 + code / b);
      kmap[col] = NONE;
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
      // one chunk: rows of one step, capped in rows and bytes
      Pend pd;
      unsigned nblk = 0;
      const size_t rec0 = recipe.size();
      while (p < rows.size() && step(rows[p]) == L) {
        const unsigned i = rows[p];
        const size_t tmark = terms.size();
        row_ops(i, a0, a1);
        const unsigned nb = (unsigned)ops.size();
        const ChunkLayout est = chunk_layout((unsigned)pd.rd.size() + 1, ((nblk + nb) + 3) & ~3u, 0u, vblk, drow);
        if (!pd.rd.empty() && (est.bytes > kChunkMaxBytes || pd.rd.size() >= kChunkMaxRows)) {
          terms.resize(tmark);  // this row starts the next chunk
          break;
        }
        pd.rd.push_back(make_uint4(pos_of(i) - a0, nblk, nblk + nb, i));  // {slot, blocks, global row}
        for (const Op& o : ops) {
          pd.xo.push_back(o.xo);
          recipe.push_back(o.rc);
        }
        nblk += nb;
        p++;
      }
      const unsigned nblk_pad = (nblk + 3) & ~3u;
      for (unsigned k = nblk; k < nblk_pad; k++) {
        pd.xo.push_back(0);  // padding: never referenced (outside every row's block range)
        recipe.push_back(make_uint4(NONE, 0u, 0u, 0u));
      }
      ChunkDesc cd = {};
      cd.nrows = (unsigned)pd.rd.size();
      cd.nblk_pad = nblk_pad;
      cd.blk0 = (unsigned)rec0;
      cd.row0 = a0;
      const ChunkLayout cl = chunk_layout(cd.nrows, nblk_pad, 0u, vblk, drow);
      cd.vals_off = cl.vals;
      cd.dinv_off = cl.dinv;
      cd.bytes = cl.bytes;
      cd.off = blob_size;
      blob_size += cl.bytes;
      stage_max = std::max(stage_max, cl.bytes);
      chunks.push_back(cd);
      pend.push_back(std::move(pd));
    }
  }
  cta_chunk[G] = (unsigned)chunks.size();
  const unsigned stage_bytes = (std::max(stage_max, 32u) + 15u) & ~15u;
  const size_t bar_bytes = 8 * (size_t)kMaxStages;
  int ns = 0;
  for (int t = kMaxStages; t >= 2; t--)
    if (x_bytes + (size_t)t * stage_bytes + bar_bytes <= kSweepSmemBudget) { ns = t; break; }
  if (ns < 2) return DFM_ERR_UNSUPPORTED;  // the slice does not fit: use more CTAs

  std::vector<char> hblob(std::max<size_t>(blob_size, 16), 0);
  for (int c = 0; c < G; c++) {
    for (unsigned q = cta_chunk[c]; q < cta_chunk[c + 1]; q++) {
      const ChunkDesc& cd = chunks[q];
      const ChunkLayout cl = chunk_layout(cd.nrows, cd.nblk_pad, 0u, vblk, drow);
      char* base = hblob.data() + cd.off;
      ChunkHeader hdr = {};
      hdr.nrows = cd.nrows;
      hdr.xoff = cl.xoff;
      hdr.vals = cl.vals;
      hdr.dinv = cl.dinv;
      if (q + ns < cta_chunk[c + 1]) {
        hdr.next_off = chunks[q + ns].off;
        hdr.next_bytes = chunks[q + ns].bytes;
      }
      std::memcpy(base, &hdr, sizeof(hdr));
      std::memcpy(base + cl.roff, pend[q].rd.data(), 16 * pend[q].rd.size());
      std::memcpy(base + cl.xoff, pend[q].xo.data(), 4 * pend[q].xo.size());
    }
  }
  P->G = G;
  P->fwd = fwd;
  P->nchunks = (unsigned)chunks.size();
  P->stage_bytes = stage_bytes;
  P->x_bytes = (unsigned)x_bytes;
  P->val_bytes = val_bytes;
  P->vec_bytes = vec_bytes;
  P->nstage = ns;
  P->smem = x_bytes + (size_t)ns * stage_bytes + bar_bytes;
  for (int c = 0; c < G; c++) P->max_cta_chunks = std::max(P->max_cta_chunks, cta_chunk[c + 1] - cta_chunk[c]);
  P->nb_ok = P->smem + ((size_t)P->max_cta_chunks + 1) * 4 + 16 + 1024 <= (size_t)227 * 1024;
  P->lpr = (b == 3) ? 4 : 1;
  cudaStream_t s = M->ctx->stream;
  DFM_CUDA_TRY(cudaMalloc(&P->d_chunks, sizeof(ChunkDesc) * std::max<size_t>(chunks.size(), 1)));
  DFM_CUDA_TRY(cudaMalloc(&P->d_cta_chunk, sizeof(unsigned) * (G + 1)));
  DFM_CUDA_TRY(cudaMalloc(&P->d_range, sizeof(unsigned) * (G + 1)));
  DFM_CUDA_TRY(cudaMalloc(&P->d_blob, hblob.size()));
  DFM_CUDA_TRY(cudaMalloc(&P->d_recipe, sizeof(uint4) * std::max<size_t>(recipe.size(), 1)));
  DFM_CUDA_TRY(cudaMalloc(&P->d_terms, sizeof(uint4) * std::max<size_t>(terms.size(), 1)));
  if (!chunks.empty())
    DFM_CUDA_TRY(cudaMemcpyAsync(P->d_chunks, chunks.data(), sizeof(ChunkDesc) * chunks.size(), cudaMemcpyHostToDevice, s));
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
  if (!terms.empty())
    DFM_CUDA_TRY(cudaMemcpyAsync(P->d_terms, terms.data(), sizeof(uint4) * terms.size(), cudaMemcpyHostToDevice, s));
  P->merged = merge;
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  P->valid = true;
  P->stale = true;
  return DFM_OK;
}

int sweep_plan_refresh(dfm_ilu M, SweepPlan* P) {
  if (!P->valid || P->nchunks == 0) { P->stale = false; return DFM_OK; }
  const int grid = (int)std::min<unsigned>(P->nchunks, (unsigned)M->ctx->nsm * 8);
  const int wd = P->fwd ? 1 : 0;
  cudaStream_t s = M->ctx->stream;
#define DFM_GATHER(BV, TV, CX)                                                                                 \
  k_gather_recipes<BV, TV, CX><<<grid, 128, 0, s>>>(P->d_chunks, P->nchunks, P->d_recipe, P->d_terms, M->d_fdiag, \
                                                    M->d_foff, P->d_blob, wd)
  if (M->vt == DFM_COMPLEX) {
    if (P->val_bytes == 8) DFM_GATHER(2, double, true); else DFM_GATHER(2, float, true);
  } else if (P->val_bytes == 8) {
    if (M->b == 1) DFM_GATHER(1, double, false); else if (M->b == 2) DFM_GATHER(2, double, false);
    else DFM_GATHER(3, double, false);
  } else {
    if (M->b == 1) DFM_GATHER(1, float, false); else if (M->b == 2) DFM_GATHER(2, float, false);
    else DFM_GATHER(3, float, false);
  }
#undef DFM_GATHER
  DFM_CUDA_TRY(cudaGetLastError());
  P->stale = false;
  return DFM_OK;
}

template <int B, int LPR, typename TV, typename TX, bool FWD, bool CPLX>
static cudaError_t launch_ranges(dfm_ilu M, const SweepPlan* P, const TX* in, TX* out, const TX* rdot,
                                 double* part, KrylovScalars* sc, const double* rr_part, int rr_n) {
  constexpr int DK = CPLX ? 2 : 1;  // fused dot kind
  dfm_ctx c = M->ctx;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P->G);
  cfg.blockDim = dim3(kSweepThreads);
  cfg.dynamicSmemBytes = P->smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (P->nb) {  // barrier-free variant: the same plan plus the per-chunk row prefix
    if (!P->nb_ok) return cudaErrorInvalidValue;
    const size_t smem = P->smem + (((size_t)P->max_cta_chunks + 1) * 4 + 15) / 16 * 16;
    cfg.dynamicSmemBytes = smem;
    auto fn = part ? k_sweep_ranges_nb<B, LPR, TV, TX, FWD, DK> : k_sweep_ranges_nb<B, LPR, TV, TX, FWD, 0>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, fn, (const ChunkDesc*)P->d_chunks, (const unsigned*)P->d_cta_chunk,
                              (const unsigned*)P->d_range, (const unsigned*)P->d_rows, (const char*)P->d_blob,
                              P->stage_bytes, P->nstage,
                              P->x_bytes, P->max_cta_chunks, in, out, rdot, part, sc, rr_part, rr_n, c->d_status,
                              (uint64_t)c->wait_ns);
  }
  auto fn = part ? (P->pipe ? k_sweep_ranges<B, LPR, TV, TX, FWD, DK, true> : k_sweep_ranges<B, LPR, TV, TX, FWD, DK, false>)
                 : (P->pipe ? k_sweep_ranges<B, LPR, TV, TX, FWD, 0, true> : k_sweep_ranges<B, LPR, TV, TX, FWD, 0, false>);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P->smem);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernelEx(&cfg, fn, (const ChunkDesc*)P->d_chunks, (const unsigned*)P->d_cta_chunk,
                            (const unsigned*)P->d_range, (const unsigned*)P->d_rows, (const char*)P->d_blob,
                            P->stage_bytes, P->nstage,
                            P->x_bytes, in, out, rdot, part, sc, rr_part, rr_n, c->d_status, (uint64_t)c->wait_ns);
}

template <int B, typename TV, typename TX, bool FWD, bool CPLX = false>
static cudaError_t launch_ranges_lpr(dfm_ilu M, const SweepPlan* P, const TX* in, TX* out, const TX* rdot,
                                     double* part, KrylovScalars* sc, const double* rr_part, int rr_n) {
  switch (P->lpr) {
    case 1: return launch_ranges<B, 1, TV, TX, FWD, CPLX>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    case 2: return launch_ranges<B, 2, TV, TX, FWD, CPLX>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    case 4: return launch_ranges<B, 4, TV, TX, FWD, CPLX>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    default: return launch_ranges<B, 8, TV, TX, FWD, CPLX>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
  }
}

template <typename TV>
static cudaError_t launch_ranges_b(dfm_ilu M, bool fwd, const SweepPlan* P, const double* in, double* out,
                                   const double* rdot, double* part, KrylovScalars* sc, const double* rr_part,
                                   int rr_n) {
  if (M->vt == DFM_COMPLEX)  // complex scalars run as real 2x2 blocks [re -im; im re]
    return fwd ? launch_ranges_lpr<2, TV, double, true, true>(M, P, in, out, rdot, part, sc, rr_part, rr_n)
               : launch_ranges_lpr<2, TV, double, false, true>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
  switch (M->b) {
    case 1: return fwd ? launch_ranges_lpr<1, TV, double, true>(M, P, in, out, rdot, part, sc, rr_part, rr_n)
                       : launch_ranges_lpr<1, TV, double, false>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    case 2: return fwd ? launch_ranges_lpr<2, TV, double, true>(M, P, in, out, rdot, part, sc, rr_part, rr_n)
                       : launch_ranges_lpr<2, TV, double, false>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
    default: return fwd ? launch_ranges_lpr<3, TV, double, true>(M, P, in, out, rdot, part, sc, rr_part, rr_n)
                        : launch_ranges_lpr<3, TV, double, false>(M, P, in, out, rdot, part, sc, rr_part, rr_n);
  }
}

int sweep_ranges_launch(dfm_ilu M, bool fwd, const double* in, double* out, const double* rdot, double* part,
                        KrylovScalars* sc, const double* rr_part, int rr_n, bool f32) {
  SweepPlan* P = f32 ? (fwd ? &M->plan32_f : &M->plan32_b) : (fwd ? &M->plan_f : &M->plan_b);
  if (!P->valid || P->val_bytes != (f32 ? 4 : 8) || P->vec_bytes != 8) return DFM_ERR_INVALID;
  if (P->stale) {
    int rc = sweep_plan_refresh(M, P);
    if (rc) return rc;
  }
  if (P->halo) {
    DFM_CUDA_TRY(sweep_halo_launch(M, fwd, P, in, out, rdot, part, sc, rr_part, rr_n, f32));
    return DFM_OK;
  }
  DFM_CUDA_TRY(f32 ? launch_ranges_b<float>(M, fwd, P, in, out, rdot, part, sc, rr_part, rr_n)
                   : launch_ranges_b<double>(M, fwd, P, in, out, rdot, part, sc, rr_part, rr_n));
  return DFM_OK;
}

}  // namespace dfm

extern "C" {

// Patches across the mesh's longest bounding-box axis (the direction the
// level sets of a lexicographically numbered structured mesh advance along
// farthest): the other axes' extent is cut into a grid of nj x nk cells (a row
// of nj cells in 2-D) with nj * nk <= max_parts, the cells as close to square
// as the extents allow, and a node's part is the cell its coordinates fall in.
// Every line of nodes along the long axis then lies in one part, and a chain
// of dependencies crosses at most about nj + nk parts.
int dfm_sweep_partition_patches(unsigned nnode, int ndim, const double* coord, unsigned max_parts, unsigned* part,
                                unsigned* nparts) {
  if ((ndim != 2 && ndim != 3) || max_parts == 0 || !nparts || (nnode && (!coord || !part))) return DFM_ERR_INVALID;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int d = 0; d < ndim; d++) {
    lo[d] = hi[d] = nnode ? coord[d] : 0.0;
    for (unsigned i = 1; i < nnode; i++) {
      lo[d] = std::min(lo[d], coord[(size_t)i * ndim + d]);
      hi[d] = std::max(hi[d], coord[(size_t)i * ndim + d]);
    }
  }
  int axis = 0;
  for (int d = 1; d < ndim; d++)
    if (hi[d] - lo[d] > hi[axis] - lo[axis]) axis = d;
  int a = -1, bax = -1;  // the cross-section axes
  for (int d = 0; d < ndim; d++) {
    if (d == axis) continue;
    if (a < 0) a = d; else bax = d;
  }
  unsigned nj = max_parts, nk = 1;
  if (bax >= 0) {
    const double ea = hi[a] - lo[a], eb = hi[bax] - lo[bax];
    const double ratio = (ea > 0 && eb > 0) ? ea / eb : 1.0;
    nj = (unsigned)std::max(1.0, std::min((double)max_parts, std::floor(std::sqrt((double)max_parts * ratio) + 0.5)));
    nk = std::max(1u, max_parts / nj);
  }
  auto cell = [](double v, double l, double h, unsigned n) -> unsigned {
    if (!(h > l) || n <= 1) return 0u;
    const double t = (v - l) / (h - l) * (double)n;
    return (unsigned)std::min<double>((double)(n - 1), std::max(0.0, std::floor(t)));
  };
  for (unsigned i = 0; i < nnode; i++) {
    const unsigned qa = cell(coord[(size_t)i * ndim + a], lo[a], hi[a], nj);
    const unsigned qb = bax >= 0 ? cell(coord[(size_t)i * ndim + bax], lo[bax], hi[bax], nk) : 0u;
    part[i] = qa * nk + qb;
  }
  *nparts = nj * nk;
  return DFM_OK;
}

}  // extern "C"
