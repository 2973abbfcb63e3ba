// Shared device helpers for the block-CRS kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dfm_b200.h"

#define DFM_DEVINL __device__ __forceinline__

// ---------------------------------------------------------------- sentinels
// Sync-free triangular sweeps write their output into a buffer pre-filled with
// a NaN payload that IEEE arithmetic never produces (operations on NaNs return
// the canonical quiet NaN), so "value != sentinel" doubles as the ready flag of
// every component.  An aligned 8-/4-byte store is single-copy atomic, so a
// reader never sees a torn value.
#define DFM_SENT64 0x7FF4DEADBEEFCAFEull
#define DFM_SENT32 0x7FA0BEEFu

template <typename T> struct Sent;
template <> struct Sent<double> {
  static DFM_DEVINL double value() { return __longlong_as_double((long long)DFM_SENT64); }
  static DFM_DEVINL bool is(double v) { return (unsigned long long)__double_as_longlong(v) == DFM_SENT64; }
};
template <> struct Sent<float> {
  static DFM_DEVINL float value() { return __uint_as_float(DFM_SENT32); }
  static DFM_DEVINL bool is(float v) { return __float_as_uint(v) == DFM_SENT32; }
};

// Loads/stores that bypass the (non-coherent) L1 so values written by other SMs
// are seen: ld/st .relaxed.gpu.
DFM_DEVINL double ld_relaxed(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
DFM_DEVINL float ld_relaxed(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
DFM_DEVINL void st_relaxed(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
DFM_DEVINL void st_relaxed(float* p, float v) {
  asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
DFM_DEVINL unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
DFM_DEVINL void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
DFM_DEVINL uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------- status word
// Device-side status shared by the kernels of one context (dfm_ctx):
//   [0] first error code raised on the device (DFM_WAIT_TIMEOUT, ...)
//   [1] number of singular ILU pivots of the last factorisation
//   [2] where a bounded wait gave up (kernel id)
struct DevStatus {
  int code;
  unsigned nsing;
  int where;
  int pad;
};

DFM_DEVINL void raise_error(DevStatus* st, int code, int where) {
  if (atomicCAS(&st->code, 0, code) == 0) st->where = where;
}

// Every spin-wait has a time limit.  When it runs out the wait records
// DFM_WAIT_TIMEOUT and gives up; the caller then stops waiting and the kernel
// drains normally, so the context stays usable.  The limit is counted with the
// SM cycle counter (a %globaltimer read costs far more than one poll and would
// sit on the critical path of every hand-off), checked every 64 polls, as
// 2 cycles per requested ns: never shorter than asked for at SM clocks up to
// 2 GHz.
DFM_DEVINL long long sm_clock() {
#ifdef __CUDA_ARCH__
  return clock64();
#else
  return 0;
#endif
}
struct SpinGuard {
  long long t0 = 0, budget = 0;
  unsigned n = 0;
  DFM_DEVINL explicit SpinGuard(uint64_t limit_ns) : t0(sm_clock()), budget((long long)(2 * limit_ns)) {}
  // true once the budget is spent (evaluated every 64th call)
  DFM_DEVINL bool expired() { return ((++n & 63u) == 0) && (sm_clock() - t0 > budget); }
};

// ---------------------------------------------------------------- reductions
template <int W, typename T>
DFM_DEVINL T group_sum(T v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic reduction of per-block partials written by the previous kernel:
// one warp sums them in a fixed order, the result is broadcast through smem.
DFM_DEVINL double reduce_partials(const double* part, int n) {
  __shared__ double s_red;
  if (threadIdx.x < 32) {
    double v = 0.0;
    for (int k = threadIdx.x; k < n; k += 32) v += part[k];
    v = group_sum<32>(v);
    if (threadIdx.x == 0) s_red = v;
  }
  __syncthreads();
  const double r = s_red;
  __syncthreads();
  return r;
}

// Block-uniform read of a device flag written by earlier kernels (or by block 0
// of the running one): every thread of the block takes the same branch.
DFM_DEVINL bool block_flag(const int* flag) {
  __shared__ int s_flag;
  __syncthreads();
  if (threadIdx.x == 0) s_flag = *(volatile const int*)flag;
  __syncthreads();
  return s_flag != 0;
}

// Block-level sum written to part[blockIdx.x] (fixed order => deterministic).
template <int NT>
DFM_DEVINL void block_partial(double v, double* part) {
  __shared__ double s_w[NT / 32];
  v = group_sum<32>(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) s_w[w] = v;
  __syncthreads();
  if (w == 0) {
    double t = (l < NT / 32) ? s_w[l] : 0.0;
    t = group_sum<32>(t);
    if (l == 0) part[blockIdx.x] = t;
  }
  __syncthreads();
}

// Exact (unfused) double ops: the reference is compiled without FMA
// contraction, so kernels that reproduce its bits use these.
DFM_DEVINL double mul_rn(double a, double b) { return __dmul_rn(a, b); }
DFM_DEVINL double add_rn(double a, double b) { return __dadd_rn(a, b); }
DFM_DEVINL double sub_rn(double a, double b) { return __dsub_rn(a, b); }
