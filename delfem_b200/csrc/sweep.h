// Plan of the range-partitioned triangular sweep (sweep.cu).
#pragma once
#include <cstddef>

namespace dfm {

constexpr int kSweepThreads = 512;               // 14 consumer warps + 1 halo warp + 1 writer warp
constexpr unsigned kChunkMaxBytes = 24 * 1024;   // one chunk = one TMA bulk copy
constexpr size_t kChunkMaxRows = 448;            // at most one row per consumer thread
constexpr int kMaxStages = 8;
constexpr size_t kSweepSmemBudget = 200 * 1024;  // dynamic shared memory per CTA

// Shared memory of a CTA:  X = [range slice | halo cache, one region per stage]
// (vector elements), then the stage ring, then the mbarriers.  Every operand of
// a level is addressed by a precomputed element offset into X, so consumers
// never branch on where a dependency lives.
//
// Byte layout of a chunk in the blob and in its stage, parts 16-byte aligned:
//   [header][roff u32: row - range start][kofs u32 (nrows+1)]
//   [xoff u32 (nblk_pad): X offset of each block's operand][halo row ids u32]
//   [factor blocks][D^-1 per row (forward only)]
struct ChunkLayout {
  unsigned roff, kofs, xoff, hids, vals, dinv, bytes;
};
__host__ __device__ inline unsigned cl_al16(unsigned x) { return (x + 15u) & ~15u; }
__host__ __device__ inline ChunkLayout chunk_layout(unsigned nrows, unsigned nblk_pad, unsigned nhalo,
                                                    unsigned vblk_bytes, unsigned dinv_row_bytes) {
  ChunkLayout L;
  L.roff = 32u;                                  // uint4 row descriptors {roff, kb, ke, 0}
  L.kofs = L.roff + cl_al16(16u * nrows);        // (unused, kept for the layout's shape)
  L.xoff = L.kofs;
  L.hids = L.xoff + cl_al16(4u * nblk_pad);
  L.vals = L.hids + cl_al16(4u * nhalo);
  L.dinv = L.vals + cl_al16(vblk_bytes * nblk_pad);
  L.bytes = L.dinv + cl_al16(dinv_row_bytes * nrows);
  return L;
}

// The header carries the stage offsets of the chunk's parts and the
// offset/size of the chunk that refills the same stage (nstage chunks later
// in the CTA's list), so no thread computes a layout or touches global memory
// to keep the ring going.
struct ChunkHeader {
  unsigned nrows, xoff, vals, dinv;
  unsigned long long next_off;
  unsigned next_bytes, pad;
};

// Host/gather-side description of a chunk.
struct ChunkDesc {
  unsigned long long off;  // byte offset in the blob
  unsigned bytes;
  unsigned nrows;
  unsigned nblk_pad;       // packed blocks (multiple of 4)
  unsigned nhalo;
  unsigned blk0;           // index of the first packed block's recipe
  unsigned vals_off, dinv_off;
  unsigned row0;           // first row of the owning range
};

struct SweepPlan {
  bool valid = false;
  bool stale = true;       // values not yet gathered from the current factor
  bool fwd = true;
  int G = 0;               // CTAs (contiguous row ranges)
  int lpr = 1;             // consumer lanes per row
  bool nb = false;         // barrier-free kernel variant (rows wait on their own operands)
  bool nb_ok = false;      // its extra shared memory (row prefix per chunk) fits
  bool pipe = false;       // barrier kernel with the two-half row pipeline across levels
  unsigned max_cta_chunks = 0;
  int nstage = 0;
  int val_bytes = 8;       // 8 = FP64 factor blocks, 4 = FP32
  int vec_bytes = 8;       // 8 = FP64 vectors, 4 = FP32
  unsigned nchunks = 0;
  unsigned stage_bytes = 0;
  unsigned x_bytes = 0;    // slice + halo cache
  size_t smem = 0;
  ChunkDesc* d_chunks = nullptr;
  unsigned* d_cta_chunk = nullptr;  // G+1 chunk ranges
  unsigned* d_range = nullptr;      // G+1 ranges of row positions
  unsigned* d_rows = nullptr;       // with a row partition: the row at each position (else positions are rows)
  bool part = false;                // ranges are the parts of the ILU's row partition
  char* d_blob = nullptr;
  uint4* d_recipe = nullptr;        // per packed block: {base slot, term range, sign}
  uint4* d_terms = nullptr;         // {s1, j, s2, 0}: F[s1] (D_j^-1) (F[s2])
  bool merged = false;              // steps are pairs of levels
  // halo plans (sweep_halo.cu, schedule mode 9): compute warps read shared memory only
  bool halo = false;
  unsigned x_slice = 0;             // elements of the range slice at the start of X
  unsigned halo_stride = 0;         // elements of one stage's halo area
  int cw = 4;                       // compute warps
  int hw = 4;                       // producer warps
};

}  // namespace dfm
