// dfm_ilu_apply_static: the ILU(0) preconditioner application
// z = U^-1 L^-1 r without any device allocation.
//
// Some callers cannot allocate device memory when they need the
// preconditioner: code that enqueues work on a stream and must not stall it
// (cudaMalloc and cudaFree can synchronise the device), code holding a fixed
// memory budget handed out by a host framework that owns all allocations, and
// callbacks that run while an allocator lock is held.  For them this entry
// point keeps its only scratch buffer - the intermediate vector y = L^-1 r
// between the two sweeps - in a file-scope static device array of
// kNoAllocMaxDoubles doubles (4 MiB).  Every GPU that loads the library holds
// that array until the process exits.
//
// Limits and sharing:
//  * N * (doubles per block row) must not exceed kNoAllocMaxDoubles
//    (524,288 doubles: e.g. 524,288 scalar rows, 174,762 3x3 block rows or
//    262,144 complex rows); larger systems get DFM_ERR_INVALID.
//  * All calls share the one array and it keeps the last call's contents.
//    The sweeps write every entry they later read, so nothing needs clearing,
//    but calls whose kernels overlap on the GPU (different streams, or
//    different contexts on one device without ordering) race on it.
//  * The first call on a context looks up the array's device address
//    (cudaGetSymbolAddress) with the context's device current and keeps it in
//    the context; make that first call before any stream capture.
//  * The call only enqueues the two sweeps on the context's stream and
//    returns; it does not wait for them.  z is ready once the stream reaches
//    that point.  Launch errors come back as DFM_ERR_CUDA; a device-side error
//    of the sweeps is picked up later by dfm_ctx_take_error.
// It runs the one-CTA level-barrier schedule, which needs no sentinel buffers
// and no autotuning (both of which allocate on first use).
#include "dfm_internal.h"

namespace dfm {

constexpr size_t kNoAllocMaxDoubles = (size_t)1 << 19;  // 4 MiB

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxDoubles];

// Device address of the scratch array for the context's device.  In host code
// g_noalloc_scratch names a host-side stand-in, not device memory, so the
// kernels get the address cudaGetSymbolAddress reports, looked up with the
// context's device current (once per context).
static int noalloc_scratch(dfm_ctx c, double** out) {
  if (!c->noalloc_scratch) {
    int cur = 0;
    DFM_CUDA_TRY(cudaGetDevice(&cur));
    if (cur != c->device) DFM_CUDA_TRY(cudaSetDevice(c->device));
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (cur != c->device) cudaSetDevice(cur);
    if (e != cudaSuccess || !p) return cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "cudaGetSymbolAddress");
    c->noalloc_scratch = static_cast<double*>(p);
  }
  *out = c->noalloc_scratch;
  return DFM_OK;
}

}  // namespace dfm

using namespace dfm;

extern "C" int dfm_ilu_apply_static(dfm_ilu M, const double* r, double* z) {
  if (!M) return DFM_ERR_INVALID;
  const size_t n = (size_t)M->N * M->xw();
  if (n > kNoAllocMaxDoubles) return DFM_ERR_INVALID;  // beyond the static scratch
  if ((M->N && (!r || !z)) || r == z || !M->factored) return DFM_ERR_INVALID;
  if (n == 0) return DFM_OK;
  double* y = nullptr;
  int rc = noalloc_scratch(M->ctx, &y);
  if (rc) return rc;
  if ((rc = ilu_fwd_launch(M, r, y, nullptr, 2))) return rc;
  return ilu_bwd_launch(M, y, z, nullptr, nullptr, nullptr, 2);
}
