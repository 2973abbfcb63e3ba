// Block-CRS SpMV, y = beta*y + alpha*A x, for the reference's storage
// (CMatDia_BlkCrs::MatVec, src/matvec/matdia_blkcrs.cpp:921-1094; complex:
// CZMatDia_BlkCrs::MatVec, src/matvec/zmatdia_blkcrs.cpp:737-801).
//
// A group of LPR lanes owns one block row at a time.  Lane j takes the row's
// off-diagonal blocks j, j+LPR, ... and the lane whose turn falls on index
// nnz takes the diagonal block, so a row's contiguous b*b*8-byte blocks are
// read by consecutive lanes (coalesced, streamed with evict-first hints) while
// x is gathered through L1/L2.  Partial products are summed inside the group
// with shuffles; lane 0 writes the b outputs.  Optional fused dots: w.y
// (w = x unless given) and y.y, reduced per block into deterministic
// partial arrays.
#include <algorithm>

#include "dfm_internal.h"

namespace dfm {

static unsigned al16_host(unsigned x) { return (x + 15u) & ~15u; }

template <int B, int LPR, typename TV, typename TX, int NDOT>
__global__ void __launch_bounds__(256)
k_spmv(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
       const TV* __restrict__ diag, const TV* __restrict__ off, double alpha,
       const TX* __restrict__ x, double beta, TX* __restrict__ y, double* __restrict__ part,
       const int* done, const TX* __restrict__ w, double* __restrict__ part2, const TX* __restrict__ y0) {
  if (done && block_flag(done)) return;
  constexpr int BB = B * B;
  const int lane = threadIdx.x % LPR;
  const unsigned g0 = (blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const unsigned ng = gridDim.x * blockDim.x / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  double dacc = 0.0, dacc2 = 0.0;
  for (unsigned i = g0; i < N; i += ng) {
    const unsigned s0 = __ldg(rowptr + i), s1 = __ldg(rowptr + i + 1);
    double acc[B];
#pragma unroll
    for (int r = 0; r < B; r++) acc[r] = 0.0;
    for (unsigned s = s0 + lane; s <= s1; s += LPR) {
      const TV* m;
      unsigned col;
      if (s < s1) {
        m = off + (size_t)s * BB;
        col = __ldcs(colind + s);
      } else {
        m = diag + (size_t)i * BB;
        col = i;
      }
      TV mv[BB];
#pragma unroll
      for (int e = 0; e < BB; e++) mv[e] = __ldcs(m + e);
      TX xv[B];
#pragma unroll
      for (int c = 0; c < B; c++) xv[c] = __ldg(x + (size_t)col * B + c);
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int c = 0; c < B; c++) acc[r] += (double)mv[r * B + c] * (double)xv[c];
    }
#pragma unroll
    for (int r = 0; r < B; r++)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
    if (lane == 0) {
#pragma unroll
      for (int r = 0; r < B; r++) {
        double v = alpha * acc[r];
        if (y0) v += (double)y0[(size_t)i * B + r];
        else if (beta != 0.0) v += beta * (double)y[(size_t)i * B + r];
        const TX out = (TX)v;
        y[(size_t)i * B + r] = out;
        if (NDOT == 1 || NDOT == 2) dacc += (double)w[(size_t)i * B + r] * (double)out;
        if (NDOT == 2) dacc2 += (double)out * (double)out;
        if (NDOT == 3) dacc += (double)out * (double)out;
      }
    }
  }
  if (NDOT >= 1) block_partial<256>(dacc, part);
  if (NDOT == 2) block_partial<256>(dacc2, part2);
}

// Complex b = 1: values and vectors interleaved (re, im).  NDOT: 0 none,
// 1 unconjugated x^T y (re / im partials), 3 |y|^2 (one partial).  TV is the
// value type (double2, or float2 for the mixed-precision solve).
template <int LPR, int NDOT, typename TV>
__global__ void __launch_bounds__(256)
k_zspmv(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
        const TV* __restrict__ diag, const TV* __restrict__ off, double alpha,
        const double2* __restrict__ x, double beta, double2* __restrict__ y, double* __restrict__ part,
        const int* done, const double2* __restrict__ y0) {
  if (done && block_flag(done)) return;
  const int lane = threadIdx.x % LPR;
  const unsigned g0 = (blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const unsigned ng = gridDim.x * blockDim.x / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  double dre = 0.0, dim = 0.0;
  for (unsigned i = g0; i < N; i += ng) {
    const unsigned s0 = __ldg(rowptr + i), s1 = __ldg(rowptr + i + 1);
    double re = 0.0, im = 0.0;
    for (unsigned s = s0 + lane; s <= s1; s += LPR) {
      TV mv;
      unsigned col;
      if (s < s1) { mv = __ldcs(off + s); col = __ldcs(colind + s); }
      else { mv = diag[i]; col = i; }
      const double2 m = make_double2((double)mv.x, (double)mv.y);
      const double2 xv = __ldg(x + col);
      re += m.x * xv.x - m.y * xv.y;
      im += m.x * xv.y + m.y * xv.x;
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      re += __shfl_xor_sync(gmask, re, o);
      im += __shfl_xor_sync(gmask, im, o);
    }
    if (lane == 0) {
      double2 v = make_double2(alpha * re, alpha * im);
      if (y0) { const double2 a = y0[i]; v.x += a.x; v.y += a.y; }
      else if (beta != 0.0) { const double2 yo = y[i]; v.x += beta * yo.x; v.y += beta * yo.y; }
      y[i] = v;
      if (NDOT == 1) {  // unconjugated x^T y (CZVector_Blk operator*, src/matvec/zvector_blk.cpp:39-59)
        const double2 xi = x[i];
        dre += xi.x * v.x - xi.y * v.y;
        dim += xi.x * v.y + xi.y * v.x;
      }
      if (NDOT == 3) dre += v.x * v.x + v.y * v.y;
    }
  }
  if (NDOT >= 1) block_partial<256>(dre, part);
  if (NDOT == 1) block_partial<256>(dim, part + kMaxBlocks);
}

// --------------------------------------------- element-wise coalesced SpMV
// A group of LPR lanes per block row walks the row's off-diagonal values as
// one contiguous run of doubles (lane e takes elements e, e+LPR, ...), so every
// load instruction of the group reads consecutive addresses; the diagonal
// block follows as the run's last b*b elements.  Element e belongs to block
// e / b^2, row (e % b^2) / b and column (e % b^2) % b of the block; the column
// index of its block and the matching x entry come through L1.
template <int B, int LPR, typename TV, int NDOT>
__global__ void __launch_bounds__(256)
k_spmv_elem(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
            const TV* __restrict__ diag, const TV* __restrict__ off, double alpha, const double* __restrict__ x,
            double beta, double* __restrict__ y, double* __restrict__ part, const int* done,
            const double* __restrict__ w, double* __restrict__ part2, const double* __restrict__ y0) {
  if (done && block_flag(done)) return;
  constexpr unsigned BB = B * B;
  const int lane = threadIdx.x % LPR;
  const unsigned g0 = (blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const unsigned ng = gridDim.x * blockDim.x / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  double dacc = 0.0, dacc2 = 0.0;
  for (unsigned i = g0; i < N; i += ng) {
    const unsigned s0 = __ldg(rowptr + i), s1 = __ldg(rowptr + i + 1);
    const unsigned nbo = s1 - s0, ne = (nbo + 1) * BB;
    const TV* vo = off + (size_t)s0 * BB;
    double acc[B];
#pragma unroll
    for (int r = 0; r < B; r++) acc[r] = 0.0;
#pragma unroll 2
    for (unsigned e = lane; e < ne; e += LPR) {
      const unsigned blk = e / BB, q = e - blk * BB;
      const unsigned rr = q / B, c = q - rr * B;
      double v;
      unsigned col;
      if (blk < nbo) {
        v = (double)__ldcs(vo + e);
        col = __ldg(colind + s0 + blk);
      } else {
        v = (double)__ldg(diag + (size_t)i * BB + q);
        col = i;
      }
      const double xv = __ldg(x + (size_t)col * B + c);
#pragma unroll
      for (int r = 0; r < B; r++)
        if (rr == (unsigned)r) acc[r] += v * xv;
    }
#pragma unroll
    for (int r = 0; r < B; r++)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
    if (lane == 0) {
#pragma unroll
      for (int r = 0; r < B; r++) {
        double v = alpha * acc[r];
        if (y0) v += y0[(size_t)i * B + r];
        else if (beta != 0.0) v += beta * y[(size_t)i * B + r];
        y[(size_t)i * B + r] = v;
        if (NDOT == 1 || NDOT == 2) dacc += w[(size_t)i * B + r] * v;
        if (NDOT == 2) dacc2 += v * v;
        if (NDOT == 3) dacc += v * v;
      }
    }
  }
  if (NDOT >= 1) block_partial<256>(dacc, part);
  if (NDOT == 2) block_partial<256>(dacc2, part2);
}

// ------------------------------------------------------ warp-staged SpMV
// A warp takes R = 32/LPR consecutive block rows per pass.  Their off-diagonal
// blocks form one contiguous run of the value array and their diagonal blocks
// another; the warp copies both runs into its own slice of shared memory with
// 16-byte cp.async copies (each instruction covers 512 contiguous bytes and
// holds no registers), then every group of LPR lanes multiplies its row as the
// lane-per-block kernel does, reading the b*b values of a block from shared
// memory.  The lane-per-block kernel reads a block with b*b 8-byte loads at a
// b*b*8-byte lane stride, so each of its load instructions touches ~20 cache
// lines and the L1 (one line per cycle), not DRAM, sets its speed; here a span
// of 32 3x3 blocks costs 5 coalesced copies and 9 shared loads per lane.
// Blocks past the slice (rows longer than it holds) are read
// from global memory directly.  The copy starts at the 16-byte boundary below
// the run and ends at the one above it (the arrays carry kArrayPad spare
// elements).
constexpr int kWsUnroll = 2;  // blocks per lane whose column and x loads are issued together
constexpr int kWsChunks = 8;  // 16-byte chunks per lane and pass: a 4,096-byte slice of off-diagonal values

template <int B, int LPR, typename TV>
struct WsShape {
  static constexpr unsigned R = 32 / LPR;
  static constexpr unsigned VB = B * B * sizeof(TV);
  static constexpr unsigned OFF = 32u * kWsChunks * 16u;
  static constexpr unsigned DIAG = (R * VB + 16u + 15u) & ~15u;
  static constexpr int DCH = (int)((DIAG / 16 + 31) / 32);
  static constexpr unsigned WARP = OFF + DIAG;
};

// 16-byte global -> shared copy that bypasses L1 and registers (cp.async.cg)
DFM_DEVINL void ws_cp16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
DFM_DEVINL void ws_cp_wait() { asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory"); }

template <int B, typename TV>
DFM_DEVINL void ws_mac(double* acc, const TV* m, const double* xv) {
#pragma unroll
  for (int r = 0; r < B; r++)
#pragma unroll
    for (int c = 0; c < B; c++) acc[r] += (double)m[r * B + c] * xv[c];
}

template <int B, int LPR, typename TV, int NDOT>
__global__ void __launch_bounds__(256)
k_spmv_ws(unsigned N, const unsigned* __restrict__ rowptr, const unsigned* __restrict__ colind,
          const TV* __restrict__ diag, const TV* __restrict__ off, double alpha, const double* __restrict__ x,
          double beta, double* __restrict__ y, double* __restrict__ part, const int* done,
          const double* __restrict__ w, double* __restrict__ part2, const double* __restrict__ y0, int npart) {
  using S = WsShape<B, LPR, TV>;
  constexpr unsigned BB = B * B;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) char ws_smem[];
  if (done && block_flag(done)) return;
  if (blockIdx.x == 0)  // partial slots past this grid belong to nobody: zero for the consumer's fixed count
    for (int k = gridDim.x + threadIdx.x; k < npart; k += blockDim.x) {
      if (NDOT >= 1) part[k] = 0.0;
      if (NDOT == 2) part2[k] = 0.0;
    }
  const unsigned l = threadIdx.x & 31u, wi = threadIdx.x >> 5;
  char* wb = ws_smem + wi * S::WARP;
  int4* wv = reinterpret_cast<int4*>(wb);
  int4* wd = reinterpret_cast<int4*>(wb + S::OFF);
  const unsigned g = l / LPR, lane = l % LPR;
  const unsigned gmask = (LPR == 32) ? FULL : (((1u << LPR) - 1u) << (g * LPR));
  const unsigned wpb = blockDim.x >> 5;
  const unsigned step = gridDim.x * wpb * S::R;
  double dacc = 0.0, dacc2 = 0.0;
  for (unsigned r0 = (blockIdx.x * wpb + wi) * S::R; r0 < N; r0 += step) {
    const unsigned rend = min(r0 + S::R, N);
    const unsigned rp = __ldg(rowptr + min(r0 + l, rend));
    const unsigned sb = __shfl_sync(FULL, rp, 0);
    const unsigned se = __shfl_sync(FULL, rp, S::R);
    const uintptr_t va = reinterpret_cast<uintptr_t>(off + (size_t)sb * BB);
    const unsigned dv = (unsigned)(va & 15u);
    const int4* vsrc = reinterpret_cast<const int4*>(va - dv);
    const size_t want = (size_t)(se - sb) * S::VB + dv;
    const unsigned nch = (unsigned)((min(want, (size_t)S::OFF) + 15u) / 16u);
    const uintptr_t da = reinterpret_cast<uintptr_t>(diag + (size_t)r0 * BB);
    const unsigned dd = (unsigned)(da & 15u);
    const int4* dsrc = reinterpret_cast<const int4*>(da - dd);
    const unsigned nchd = ((rend - r0) * S::VB + dd + 15u) / 16u;
    __syncwarp();  // the previous pass's reads of the slice are done
#pragma unroll
    for (int c = 0; c < kWsChunks; c++)
      if (l + 32u * c < nch) ws_cp16(wv + l + 32u * c, vsrc + l + 32u * c);
#pragma unroll
    for (int c = 0; c < S::DCH; c++)
      if (l + 32u * c < nchd) ws_cp16(wd + l + 32u * c, dsrc + l + 32u * c);
    ws_cp_wait();
    __syncwarp();  // every lane's copies visible to the warp
    const unsigned i = r0 + g;
    const unsigned s0 = __shfl_sync(FULL, rp, g), s1 = __shfl_sync(FULL, rp, g + 1);
    if (i < rend) {  // group-uniform
      double acc[B];
#pragma unroll
      for (int r = 0; r < B; r++) acc[r] = 0.0;
      // the lane's blocks s0 + lane, + LPR, ... (the diagonal block last, as
      // slot s1) in that order, kWsUnroll at a time: their column indices,
      // then their x entries are requested together before the products
      constexpr int U = kWsUnroll;
      for (unsigned sb0 = s0 + lane; sb0 <= s1; sb0 += U * LPR) {
        unsigned col[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const unsigned s = sb0 + u * LPR;
          col[u] = s < s1 ? __ldcs(colind + s) : i;
        }
        double xv[U][B];
#pragma unroll
        for (int u = 0; u < U; u++)
          if (sb0 + u * LPR <= s1)
#pragma unroll
            for (int c = 0; c < B; c++) xv[u][c] = __ldg(x + (size_t)col[u] * B + c);
#pragma unroll
        for (int u = 0; u < U; u++) {
          const unsigned s = sb0 + u * LPR;
          if (s < s1) {
            const size_t boff = (size_t)(s - sb) * S::VB + dv;
            if (boff + S::VB <= S::OFF) ws_mac<B>(acc, reinterpret_cast<const TV*>(wb + boff), xv[u]);
            else ws_mac<B>(acc, off + (size_t)s * BB, xv[u]);
          } else if (s == s1) {
            ws_mac<B>(acc, reinterpret_cast<const TV*>(wb + S::OFF + dd + g * S::VB), xv[u]);
          }
        }
      }
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
      if (lane == 0) {
#pragma unroll
        for (int r = 0; r < B; r++) {
          double val = alpha * acc[r];
          if (y0) val += y0[(size_t)i * B + r];
          else if (beta != 0.0) val += beta * y[(size_t)i * B + r];
          y[(size_t)i * B + r] = val;
          if (NDOT == 1 || NDOT == 2) dacc += w[(size_t)i * B + r] * val;
          if (NDOT == 2) dacc2 += val * val;
          if (NDOT == 3) dacc += val * val;
        }
      }
    }
  }
  if (NDOT >= 1) block_partial<256>(dacc, part);
  if (NDOT == 2) block_partial<256>(dacc2, part2);
}

template <int B, int LPR, typename TV, int NDOT>
static cudaError_t launch_ws_n(dfm_mat A, const TV* diag, const TV* off, int npart, cudaStream_t s, double alpha,
                               const double* x, double beta, double* y, double* part, const int* done,
                               const double* w, double* part2, const double* y0) {
  using S = WsShape<B, LPR, TV>;
  auto fn = k_spmv_ws<B, LPR, TV, NDOT>;
  const int smem = (int)(8 * S::WARP);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, smem);
  if (e != cudaSuccess) return e;
  // one resident wave: a second partial wave would leave most SMs idle at the end
  const int cap = npart > 0 ? npart : kMaxBlocks;
  const int grid = std::max(1, std::min(A->ctx->nsm * std::max(occ, 1), cap));
  fn<<<grid, 256, smem, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y, part, done, w, part2, y0,
                             part ? npart : 0);
  return cudaGetLastError();
}

template <int B, int LPR, typename TV>
static cudaError_t launch_ws_t(dfm_mat A, const TV* diag, const TV* off, int npart, cudaStream_t s, double alpha,
                               const double* x, double beta, double* y, double* part, const int* done,
                               const SpmvOpts& o) {
  const double* w = o.dot_w ? o.dot_w : x;
  if (part && o.yy)
    return launch_ws_n<B, LPR, TV, 3>(A, diag, off, npart, s, alpha, x, beta, y, part, done, nullptr, nullptr, o.y0);
  if (part && o.dot_part2)
    return launch_ws_n<B, LPR, TV, 2>(A, diag, off, npart, s, alpha, x, beta, y, part, done, w, o.dot_part2, o.y0);
  if (part)
    return launch_ws_n<B, LPR, TV, 1>(A, diag, off, npart, s, alpha, x, beta, y, part, done, w, nullptr, o.y0);
  return launch_ws_n<B, LPR, TV, 0>(A, diag, off, npart, s, alpha, x, beta, y, nullptr, done, nullptr, nullptr,
                                    o.y0);
}

template <int B>
static cudaError_t launch_ws(dfm_mat A, int lanes, int npart, cudaStream_t s, double alpha, const double* x,
                             double beta, double* y, double* part, const int* done, const SpmvOpts& o) {
#define DFM_WS_L(L)                                                                                              \
  return o.f32 ? launch_ws_t<B, L, float>(A, A->d_diag32, A->d_off32, npart, s, alpha, x, beta, y, part, done, o) \
               : launch_ws_t<B, L, double>(A, A->d_diag, A->d_off, npart, s, alpha, x, beta, y, part, done, o)
  switch (lanes) {
    case 4: DFM_WS_L(4);
    case 8: DFM_WS_L(8);
    case 16: DFM_WS_L(16);
    default: DFM_WS_L(32);
  }
#undef DFM_WS_L
}

template <int B, int LPR, typename TV>
static void launch_elem_t(dfm_mat A, const TV* diag, const TV* off, int grid, cudaStream_t s, double alpha,
                          const double* x, double beta, double* y, double* part, const int* done,
                          const SpmvOpts& o) {
  const double* w = o.dot_w ? o.dot_w : x;
  if (part && o.yy)
    k_spmv_elem<B, LPR, TV, 3><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                    part, done, nullptr, nullptr, o.y0);
  else if (part && o.dot_part2)
    k_spmv_elem<B, LPR, TV, 2><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                    part, done, w, o.dot_part2, o.y0);
  else if (part)
    k_spmv_elem<B, LPR, TV, 1><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                    part, done, w, nullptr, o.y0);
  else
    k_spmv_elem<B, LPR, TV, 0><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                    nullptr, done, nullptr, nullptr, o.y0);
}

template <int B>
static void launch_elem(dfm_mat A, int lanes, int grid, cudaStream_t s, double alpha, const double* x, double beta,
                        double* y, double* part, const int* done, const SpmvOpts& o) {
#define DFM_ELEM_L(L)                                                                                        \
  if (o.f32) launch_elem_t<B, L, float>(A, A->d_diag32, A->d_off32, grid, s, alpha, x, beta, y, part, done, o); \
  else launch_elem_t<B, L, double>(A, A->d_diag, A->d_off, grid, s, alpha, x, beta, y, part, done, o);          \
  return
  switch (lanes) {
    case 4: DFM_ELEM_L(4);
    case 8: DFM_ELEM_L(8);
    case 16: DFM_ELEM_L(16);
    default: DFM_ELEM_L(32);
  }
#undef DFM_ELEM_L
}

// ------------------------------------------------------ TMA-staged SpMV
// Rows are cut into tiles (at most kTileRows rows and kTileValBytes of
// off-diagonal values).  A persistent CTA walks its tiles (t = blockIdx.x +
// k*gridDim.x); for each, thread 0 issues four 1-D bulk copies (values,
// column indices, diagonal blocks, row pointers; no multicast) into a stage
// of a shared-memory ring several tiles ahead, completing on the stage's
// mbarrier.  The value stream thus reaches shared memory as whole contiguous
// lines, instead of as the scattered per-lane 8-byte pieces of the
// lane-per-block kernel (whose every load instruction touches ~32 sectors).
// Lane groups then take a row each, lane j the row's blocks j, j+LPR, ... (the
// diagonal block last), reading b*b values from shared memory and gathering b
// entries of x through L1/L2; with 1024 threads a tile's rows are covered in
// about one pass, so a tile costs one round of x-gather latency.  A copy
// starts at the 16-byte boundary below its first byte and is rounded up to 16
// bytes (the arrays carry kArrayPad spare elements); the offsets of the first
// element are kept per stage.
constexpr unsigned kTileRows = 256;
constexpr unsigned kTileValBytes = 48 * 1024;
constexpr int kTmaThreads = 1024;

DFM_DEVINL unsigned sp_smem(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
DFM_DEVINL void sp_mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sp_smem(bar)), "r"(count) : "memory");
}
DFM_DEVINL void sp_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
DFM_DEVINL void sp_arrive_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(sp_smem(bar)), "r"(bytes)
               : "memory");
}
DFM_DEVINL bool sp_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(sp_smem(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
DFM_DEVINL void sp_bulk(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   sp_smem(dst)),
               "l"(src), "r"(bytes), "r"(sp_smem(bar))
               : "memory");
}
DFM_DEVINL void sp_fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

struct TileHdr {
  unsigned r0, r1, s0, dv, dc, dd, dr, pad;  // rows, first block, byte offsets of the first elements
};

template <typename TV>
struct TmaArgs {
  unsigned N;
  const unsigned* rowptr;
  const unsigned* colind;
  const TV* diag;
  const TV* off;
  const unsigned* tiles;
  unsigned ntiles, stage_bytes, vals_bytes, col_bytes, diag_bytes;
  int nstage;
  double alpha, beta;
  const double* x;
  double* y;
  const double* y0;
  const double* w;
  double* part;
  double* part2;
  int npart;
  const int* done;
  DevStatus* st;
  uint64_t wait_ns;
};

DFM_DEVINL const char* al16_down(const void* p, unsigned* delta) {
  const uintptr_t a = (uintptr_t)p;
  *delta = (unsigned)(a & 15u);
  return reinterpret_cast<const char*>(a & ~(uintptr_t)15);
}
DFM_DEVINL unsigned al16_up(unsigned x) { return (x + 15u) & ~15u; }

// thread 0: stage s <- tile t
template <int B, typename TV>
DFM_DEVINL void tma_issue(const TmaArgs<TV>& a, char* stage, uint64_t* bar, TileHdr* hdr, unsigned t) {
  constexpr unsigned BB = B * B;
  const unsigned r0 = a.tiles[t], r1 = a.tiles[t + 1];
  const unsigned s0 = a.rowptr[r0], s1 = a.rowptr[r1];
  TileHdr h;
  h.r0 = r0;
  h.r1 = r1;
  h.s0 = s0;
  const char* pv = al16_down(a.off + (size_t)s0 * BB, &h.dv);
  const char* pc = al16_down(a.colind + s0, &h.dc);
  const char* pd = al16_down(a.diag + (size_t)r0 * BB, &h.dd);
  const char* pr = al16_down(a.rowptr + r0, &h.dr);
  const unsigned nv = al16_up((s1 - s0) * BB * (unsigned)sizeof(TV) + h.dv);
  const unsigned nc = al16_up((s1 - s0) * 4u + h.dc);
  const unsigned nd = al16_up((r1 - r0) * BB * (unsigned)sizeof(TV) + h.dd);
  const unsigned nr = al16_up((r1 - r0 + 1) * 4u + h.dr);
  *hdr = h;
  sp_fence_proxy();
  sp_arrive_tx(bar, nv + nc + nd + nr);
  if (nv) sp_bulk(stage, pv, nv, bar);
  if (nc) sp_bulk(stage + a.vals_bytes, pc, nc, bar);
  if (nd) sp_bulk(stage + a.vals_bytes + a.col_bytes, pd, nd, bar);
  sp_bulk(stage + a.vals_bytes + a.col_bytes + a.diag_bytes, pr, nr, bar);  // nr >= 16
}

template <int B, int LPR, typename TV, int NDOT>
__global__ void __launch_bounds__(kTmaThreads)
k_spmv_tma(TmaArgs<TV> a) {
  constexpr unsigned BB = B * B;
  extern __shared__ __align__(128) char smem[];
  __shared__ uint64_t bar[8];
  __shared__ TileHdr hdr[8];
  __shared__ int s_alive;
  if (a.done && block_flag(a.done)) return;
  const int ns = a.nstage;
  const unsigned my_tiles = a.ntiles > blockIdx.x ? (a.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
  if (threadIdx.x == 0) {
    s_alive = 1;
    for (int s = 0; s < ns; s++) sp_mbar_init(&bar[s], 1);
    sp_fence_init();
    for (unsigned k = 0; k < my_tiles && k < (unsigned)ns; k++)
      tma_issue<B, TV>(a, smem + (size_t)k * a.stage_bytes, &bar[k], &hdr[k], blockIdx.x + k * gridDim.x);
  }
  if (blockIdx.x == 0)  // partial slots past this grid belong to nobody: zero for the consumer's fixed count
    for (int k = gridDim.x + threadIdx.x; k < a.npart; k += blockDim.x) {
      if (NDOT >= 1) a.part[k] = 0.0;
      if (NDOT == 2) a.part2[k] = 0.0;
    }
  __syncthreads();
  const int lane = threadIdx.x % LPR;
  const unsigned g = threadIdx.x / LPR, ng = kTmaThreads / LPR;
  const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) / LPR * LPR));
  double dacc = 0.0, dacc2 = 0.0;
  unsigned consumed = 0;
  for (unsigned k = 0; k < my_tiles; k++) {
    const int s = (int)(k % (unsigned)ns);
    char* stage = smem + (size_t)s * a.stage_bytes;
    if (threadIdx.x == 0 && s_alive) {
      const unsigned par = (k / (unsigned)ns) & 1u;
      if (!sp_try_wait(&bar[s], par)) {
        SpinGuard gd(a.wait_ns);
        while (!sp_try_wait(&bar[s], par))
          if (gd.expired()) {
            raise_error(a.st, DFM_WAIT_TIMEOUT, 20);
            s_alive = 0;
            break;
          }
      }
    }
    __syncthreads();
    if (!s_alive) break;
    const TileHdr h = hdr[s];
    const TV* vals = reinterpret_cast<const TV*>(stage + h.dv);
    const unsigned* cols = reinterpret_cast<const unsigned*>(stage + a.vals_bytes + h.dc);
    const TV* dg = reinterpret_cast<const TV*>(stage + a.vals_bytes + a.col_bytes + h.dd);
    const unsigned* rp = reinterpret_cast<const unsigned*>(stage + a.vals_bytes + a.col_bytes + a.diag_bytes + h.dr);
    for (unsigned i = h.r0 + g; i < h.r1; i += ng) {  // group-uniform
      const unsigned li = i - h.r0;
      const unsigned b0 = rp[li] - h.s0, b1 = rp[li + 1] - h.s0;
      const unsigned nb = b1 - b0;  // off-diagonal blocks; index nb is the diagonal block
      double acc[B];
#pragma unroll
      for (int r = 0; r < B; r++) acc[r] = 0.0;
      for (unsigned k = lane; k <= nb; k += LPR) {
        const TV* m;
        unsigned col;
        if (k < nb) {
          m = vals + (size_t)(b0 + k) * BB;
          col = cols[b0 + k];
        } else {
          m = dg + (size_t)li * BB;
          col = i;
        }
        double xv[B];
#pragma unroll
        for (int c = 0; c < B; c++) xv[c] = __ldg(a.x + (size_t)col * B + c);
#pragma unroll
        for (int r = 0; r < B; r++)
#pragma unroll
          for (int c = 0; c < B; c++) acc[r] += (double)m[r * B + c] * xv[c];
      }
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(gmask, acc[r], o);
      if (lane == 0) {
#pragma unroll
        for (int r = 0; r < B; r++) {
          double v = a.alpha * acc[r];
          if (a.y0) v += a.y0[(size_t)i * B + r];
          else if (a.beta != 0.0) v += a.beta * a.y[(size_t)i * B + r];
          a.y[(size_t)i * B + r] = v;
          if (NDOT == 1 || NDOT == 2) dacc += a.w[(size_t)i * B + r] * v;
          if (NDOT == 2) dacc2 += v * v;
          if (NDOT == 3) dacc += v * v;
        }
      }
    }
    __syncthreads();  // stage s free
    consumed = k + 1;
    if (threadIdx.x == 0 && k + ns < my_tiles && s_alive)
      tma_issue<B, TV>(a, stage, &bar[s], &hdr[s], blockIdx.x + (k + ns) * gridDim.x);
  }
  if (NDOT >= 1) block_partial<kTmaThreads>(dacc, a.part);
  if (NDOT == 2) block_partial<kTmaThreads>(dacc2, a.part2);
  // copies issued but not consumed (after an expired wait) must land before the CTA exits
  if (threadIdx.x == 0 && !s_alive) {
    const unsigned issued = std::min(my_tiles, consumed + (unsigned)ns);
    for (unsigned j = consumed; j < issued; j++) {
      const unsigned par = (j / (unsigned)ns) & 1u;
      SpinGuard gd(a.wait_ns);
      while (!sp_try_wait(&bar[j % (unsigned)ns], par))
        if (gd.expired()) break;
    }
  }
}

// Tiles for value width sv (bytes); stage sizes from the largest tile.
static int build_tiles(dfm_mat A, int which) {
  SpmvTiles& T = A->tiles[which];
  if (T.valid) return DFM_OK;
  const unsigned bb = A->b * A->b, sv = which ? 4u : 8u;
  std::vector<unsigned> t(1, 0);
  unsigned r = 0, mr = 0, mb = 0;
  while (r < A->N) {
    unsigned r1 = r, nb = 0;
    while (r1 < A->N && r1 - r < kTileRows) {
      const unsigned rb = A->h_rowptr[r1 + 1] - A->h_rowptr[r1];
      if (r1 > r && (nb + rb) * bb * sv > kTileValBytes) break;
      nb += rb;
      r1++;
    }
    mr = std::max(mr, r1 - r);
    mb = std::max(mb, nb);
    t.push_back(r1);
    r = r1;
  }
  T.ntiles = (unsigned)t.size() - 1;
  T.max_rows = mr;
  T.max_blocks = mb;
  T.vals_bytes = al16_host(mb * bb * sv + 16);
  T.col_bytes = al16_host(mb * 4 + 16);
  T.diag_bytes = al16_host(mr * bb * sv + 16);
  T.rp_bytes = al16_host((mr + 1) * 4 + 16);
  T.stage_bytes = T.vals_bytes + T.col_bytes + T.diag_bytes + T.rp_bytes;
  T.nstage = (int)std::min<size_t>(8, (size_t)(200 * 1024) / T.stage_bytes);
  if (T.nstage < 2) return DFM_ERR_UNSUPPORTED;
  DFM_CUDA_TRY(cudaMalloc(&T.d_tiles, t.size() * sizeof(unsigned)));
  DFM_CUDA_TRY(cudaMemcpy(T.d_tiles, t.data(), t.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
  T.valid = true;
  return DFM_OK;
}

void spmv_free_tiles(dfm_mat A) {
  for (SpmvTiles& T : A->tiles) {
    cudaFree(T.d_tiles);
    T = SpmvTiles();
  }
}

template <int B, int LPR, typename TV>
static cudaError_t launch_tma_t(dfm_mat A, const SpmvTiles& T, const TV* diag, const TV* off, int npart,
                                cudaStream_t s, double alpha, const double* x, double beta, double* y,
                                double* part, const int* done, const SpmvOpts& o) {
  TmaArgs<TV> a;
  a.N = A->N;
  a.rowptr = A->d_rowptr;
  a.colind = A->d_colind;
  a.diag = diag;
  a.off = off;
  a.tiles = T.d_tiles;
  a.ntiles = T.ntiles;
  a.stage_bytes = T.stage_bytes;
  a.vals_bytes = T.vals_bytes;
  a.col_bytes = T.col_bytes;
  a.diag_bytes = T.diag_bytes;
  a.nstage = T.nstage;
  a.alpha = alpha;
  a.beta = beta;
  a.x = x;
  a.y = y;
  a.y0 = o.y0;
  a.w = o.dot_w ? o.dot_w : x;
  a.part = part;
  a.part2 = o.dot_part2;
  a.npart = npart;
  a.done = done;
  a.st = A->ctx->d_status;
  a.wait_ns = A->ctx->wait_ns;
  const size_t smem = (size_t)T.nstage * T.stage_bytes;
  const int per_sm = std::max(1, (int)((227 * 1024) / (smem + 2048)));
  const int grid = std::max(1, std::min<int>((int)T.ntiles, std::min(A->ctx->nsm * per_sm, npart > 0 ? npart
                                                                                                       : kMaxBlocks)));
  auto fn = (part && o.yy) ? k_spmv_tma<B, LPR, TV, 3>
            : (part && o.dot_part2) ? k_spmv_tma<B, LPR, TV, 2>
            : part ? k_spmv_tma<B, LPR, TV, 1> : k_spmv_tma<B, LPR, TV, 0>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<grid, kTmaThreads, smem, s>>>(a);
  return cudaGetLastError();
}

template <int B>
static cudaError_t launch_tma(dfm_mat A, int lanes, int npart, cudaStream_t s, double alpha, const double* x,
                              double beta, double* y, double* part, const int* done, const SpmvOpts& o) {
  const SpmvTiles& T = A->tiles[o.f32 ? 1 : 0];
#define DFM_TMA_L(L)                                                                                             \
  return o.f32 ? launch_tma_t<B, L, float>(A, T, A->d_diag32, A->d_off32, npart, s, alpha, x, beta, y, part, done, \
                                           o)                                                                    \
               : launch_tma_t<B, L, double>(A, T, A->d_diag, A->d_off, npart, s, alpha, x, beta, y, part, done, o)
  switch (lanes) {
    case 4: DFM_TMA_L(4);
    case 8: DFM_TMA_L(8);
    case 16: DFM_TMA_L(16);
    default: DFM_TMA_L(32);
  }
#undef DFM_TMA_L
}

int spmv_grid(dfm_mat A) {
  // grid-stride: 8 blocks of 256 threads per SM keep enough loads in flight
  const int want = A->ctx->nsm * 8;
  return std::max(1, std::min(want, kMaxBlocks));
}

template <int B, int LPR, typename TV>
static void launch_real_tv(dfm_mat A, const TV* diag, const TV* off, int grid, cudaStream_t s, double alpha,
                           const double* x, double beta, double* y, double* part, const int* done,
                           const SpmvOpts& o) {
  const double* w = o.dot_w ? o.dot_w : x;
  if (part && o.yy)
    k_spmv<B, LPR, TV, double, 3><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                       part, done, nullptr, nullptr, o.y0);
  else if (part && o.dot_part2)
    k_spmv<B, LPR, TV, double, 2><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                       part, done, w, o.dot_part2, o.y0);
  else if (part)
    k_spmv<B, LPR, TV, double, 1><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                       part, done, w, nullptr, o.y0);
  else
    k_spmv<B, LPR, TV, double, 0><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, diag, off, alpha, x, beta, y,
                                                       nullptr, done, nullptr, nullptr, o.y0);
}

template <int B, int LPR>
static void launch_real(dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x, double beta,
                        double* y, double* part, const int* done, const SpmvOpts& o) {
  if (o.f32)
    launch_real_tv<B, LPR, float>(A, A->d_diag32, A->d_off32, grid, s, alpha, x, beta, y, part, done, o);
  else
    launch_real_tv<B, LPR, double>(A, A->d_diag, A->d_off, grid, s, alpha, x, beta, y, part, done, o);
}

template <int B>
static void launch_real_lpr(int lanes, dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x,
                            double beta, double* y, double* part, const int* done, const SpmvOpts& o) {
  switch (lanes) {
    case 4: launch_real<B, 4>(A, grid, s, alpha, x, beta, y, part, done, o); break;
    case 8: launch_real<B, 8>(A, grid, s, alpha, x, beta, y, part, done, o); break;
    case 16: launch_real<B, 16>(A, grid, s, alpha, x, beta, y, part, done, o); break;
    default: launch_real<B, 32>(A, grid, s, alpha, x, beta, y, part, done, o); break;
  }
}

template <int LPR, typename TV>
static void launch_cplx_tv(dfm_mat A, const TV* d, const TV* o, int grid, cudaStream_t s, double alpha,
                           const double* x, double beta, double* y, double* part, const int* done,
                           const SpmvOpts& op) {
  auto* xx = reinterpret_cast<const double2*>(x);
  auto* yy = reinterpret_cast<double2*>(y);
  auto* y0 = reinterpret_cast<const double2*>(op.y0);
  if (part && op.yy)
    k_zspmv<LPR, 3, TV><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, d, o, alpha, xx, beta, yy, part, done,
                                             y0);
  else if (part)
    k_zspmv<LPR, 1, TV><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, d, o, alpha, xx, beta, yy, part, done,
                                             y0);
  else
    k_zspmv<LPR, 0, TV><<<grid, 256, 0, s>>>(A->N, A->d_rowptr, A->d_colind, d, o, alpha, xx, beta, yy, nullptr,
                                             done, y0);
}

template <int LPR>
static void launch_cplx(dfm_mat A, int grid, cudaStream_t s, double alpha, const double* x, double beta,
                        double* y, double* part, const int* done, const SpmvOpts& op) {
  if (op.f32)
    launch_cplx_tv<LPR, float2>(A, reinterpret_cast<const float2*>(A->d_diag32),
                                reinterpret_cast<const float2*>(A->d_off32), grid, s, alpha, x, beta, y, part, done,
                                op);
  else
    launch_cplx_tv<LPR, double2>(A, reinterpret_cast<const double2*>(A->d_diag),
                                 reinterpret_cast<const double2*>(A->d_off), grid, s, alpha, x, beta, y, part, done,
                                 op);
}

int spmv_launch(dfm_mat A, double alpha, const double* x, double beta, double* y, double* dot_part,
                int grid, KrylovScalars* sc, int lanes, const SpmvOpts& o) {
  if (A->vt == DFM_COMPLEX && (o.dot_w || o.dot_part2)) return DFM_ERR_UNSUPPORTED;
  if (o.f32 && !A->d_off32) return DFM_ERR_INVALID;
  if (A->N == 0) return DFM_OK;
  cudaStream_t s = A->ctx->stream;
  if (grid <= 0) grid = spmv_grid(A);
  if (lanes <= 0) lanes = A->lanes > 0 ? A->lanes : (A->b == 3 ? 16 : 8);
  const int* done = sc ? &sc->done : nullptr;
  const int kind = o.kind >= 0 ? o.kind : A->spmv_kind;
  if (kind == 2 && A->vt == DFM_REAL) {
    switch (A->b) {
      case 1: launch_elem<1>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      case 2: launch_elem<2>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      default: launch_elem<3>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
    }
    DFM_CUDA_TRY(cudaGetLastError());
    return DFM_OK;
  }
  if (kind == 3 && A->vt == DFM_REAL) {
    cudaError_t e;
    switch (A->b) {
      case 1: e = launch_ws<1>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      case 2: e = launch_ws<2>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      default: e = launch_ws<3>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
    }
    DFM_CUDA_TRY(e);
    return DFM_OK;
  }
  if (kind == 1 && A->vt == DFM_REAL) {
    if (!A->tiles[o.f32 ? 1 : 0].valid) {
      const int rc = build_tiles(A, o.f32 ? 1 : 0);  // host set-up; normally done by the autotuner
      if (rc) return rc;
    }
    cudaError_t e;
    switch (A->b) {
      case 1: e = launch_tma<1>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      case 2: e = launch_tma<2>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      default: e = launch_tma<3>(A, lanes, grid, s, alpha, x, beta, y, dot_part, done, o); break;
    }
    DFM_CUDA_TRY(e);
    return DFM_OK;
  }
  if (A->vt == DFM_COMPLEX) {
    switch (lanes) {
      case 4: launch_cplx<4>(A, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      case 8: launch_cplx<8>(A, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      case 16: launch_cplx<16>(A, grid, s, alpha, x, beta, y, dot_part, done, o); break;
      default: launch_cplx<32>(A, grid, s, alpha, x, beta, y, dot_part, done, o); break;
    }
  } else if (A->b == 1) {
    launch_real_lpr<1>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, o);
  } else if (A->b == 2) {
    launch_real_lpr<2>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, o);
  } else {
    launch_real_lpr<3>(lanes, A, grid, s, alpha, x, beta, y, dot_part, done, o);
  }
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

__global__ void k_to_f32(size_t n, const double* __restrict__ in, float* __restrict__ out) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    out[k] = (float)in[k];
}

int to_f32(dfm_ctx c, const double* in, float* out, size_t n) {
  if (n == 0) return DFM_OK;
  const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)c->nsm * 8);
  k_to_f32<<<grid, 256, 0, c->stream>>>(n, in, out);
  DFM_CUDA_TRY(cudaGetLastError());
  return DFM_OK;
}

// FP32 copy of the values (allocated on first use, refreshed on every call).
int mat_make_f32(dfm_mat A) {
  const size_t nd = (size_t)A->N * A->vw(), no = (size_t)A->ncrs * A->vw();
  if (!A->d_diag32) {
    DFM_CUDA_TRY(cudaMalloc(&A->d_diag32, (nd + kArrayPad) * sizeof(float)));
    DFM_CUDA_TRY(cudaMalloc(&A->d_off32, (no + kArrayPad) * sizeof(float)));
  }
  int rc = to_f32(A->ctx, A->d_diag, A->d_diag32, nd);
  if (!rc) rc = to_f32(A->ctx, A->d_off, A->d_off32, no);
  if (!rc && A->vt == DFM_REAL && A->spmv_kind == 1 && !A->tiles[1].valid) rc = build_tiles(A, 1);
  return rc;
}

// Autotuner: times every lanes-per-row choice on this matrix (CUDA events on
// the context stream, best of 3 after a warm-up) and keeps the fastest.
int spmv_autotune(dfm_mat A) {
  if (A->lanes > 0) return DFM_OK;
  if (A->N == 0) { A->lanes = 8; return DFM_OK; }
  cudaStream_t s = A->ctx->stream;
  const size_t n = (size_t)A->N * A->xw();
  double *x = nullptr, *y = nullptr;
  DFM_CUDA_TRY(cudaMallocAsync(&x, n * sizeof(double), s));
  DFM_CUDA_TRY(cudaMallocAsync(&y, n * sizeof(double), s));
  DFM_CUDA_TRY(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int cand[4] = {4, 8, 16, 32};
  float best = 1e30f;
  int best_l = 8, best_k = 0;
  const bool tiles_ok = A->vt == DFM_REAL && build_tiles(A, 0) == DFM_OK;
  cudaGetLastError();
  for (int kind = 0; kind < 4; kind++)
    for (int c = 0; c < 4; c++) {
      if (kind > 0 && A->vt != DFM_REAL) break;
      if (kind == 1 && !tiles_ok) break;
      SpmvOpts o;
      o.kind = kind;
      int rc = spmv_launch(A, 1.0, x, 0.0, y, nullptr, 0, nullptr, cand[c], o);
      if (rc) return rc;
      float tmin = 1e30f;
      for (int rep = 0; rep < 3; rep++) {
        cudaEventRecord(e0, s);
        spmv_launch(A, 1.0, x, 0.0, y, nullptr, 0, nullptr, cand[c], o);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        tmin = std::min(tmin, ms);
      }
      if (tmin < best) { best = tmin; best_l = cand[c]; best_k = kind; }
    }
  A->spmv_kind = best_k;
  if (best_k == 1 && A->d_off32 && !A->tiles[1].valid) {
    const int rc = build_tiles(A, 1);
    if (rc) return rc;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(x, s);
  cudaFreeAsync(y, s);
  DFM_CUDA_TRY(cudaStreamSynchronize(s));
  A->lanes = best_l;
  return DFM_OK;
}

}  // namespace dfm
