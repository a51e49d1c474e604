// blocked.h -- the slice-blocked pull sweep: device layout and launchers.
//
// The reference's pull loop (src/pr_spmv.cc:46-54) gathers contrib[v] for
// every in-edge v -> u from a random place.  On the device each such gather
// that misses L1 costs one 32-byte sector request between the SM and L2, and
// those requests, not HBM bytes, bound the classic sweep (pull.cu).  This
// layout replaces them with streamed bytes (propagation blocking, Beamer,
// Asanovic and Patterson, IPDPS 2017), in two phases per sweep:
//
//   phase 1 (per source slice)  a CTA holds contrib[] of one slice of
//     slice_verts consecutive (renumbered) source ids in shared memory.  The
//     in-edges of one row from one slice form a pair; the slice's pairs are
//     stored sliced-ELL: grouped by length class into groups of 32 lanes,
//     L lanes per pair (1 to 32, chosen per run of a class), the
//     16-bit slice-local source ids of each lane's share interleaved across
//     the group in blocks of B ids (pairs of up to 8 ids: one block of 1, 2,
//     4 or 8; longer pairs: blocks of 8; padded with an id whose value is
//     zero).  All groups of one (slice, class) run have the same shape, so a
//     warp streams a contiguous block of groups as one regular array.  The
//     pair's lanes join their sums and write the partial to
//     part[dest[pair]].  Two launches: the runs of one block per pair (flat)
//     and the others.
//   phase 2 (per destination bin)  part[] is laid out bin-major: the
//     partials of one bin of consecutive rows are one contiguous block (the
//     flat launch's pairs first, each part slice-major).  A CTA copies that
//     block and the bin's positions into shared memory; each thread then
//     takes rows of the bin and sums each row's partials in slice order (a
//     16-bit position in the block per pair, rows' pairs consecutive), and
//     updates the row: new = base + d * sum, |new - old| added in FP64,
//     contrib[u] = new / out_degree(u).
//
// Every sum is a fixed tree over a fixed layout, so a sweep's result does
// not depend on scheduling.  With vertices in descending-degree order most
// edges come from the first slices, so one pair stands for many edges (at
// Kronecker scale 25, 48K-vertex slices: 0.17 pairs per edge).
//
// Stream positions and pair indices are int32 (the CSR has < 2^31 entries).
#ifndef GAPBS_B200_ENGINE_BLOCKED_H_
#define GAPBS_B200_ENGINE_BLOCKED_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "internal.h"

namespace prgpu {

// Phase 1: 1024 threads, one CTA per SM; phase 2: 256, 512 or 1024
// threads per bin (BinRowThreads).
constexpr int kSliceWarps = 32;
constexpr int kDefaultSliceVerts = 49152;  // 192 KB of contribs in shared memory
constexpr int kDefaultBinWords = 6144;     // partials per bin (pairs + rows): 24 KB + 12 KB of positions
constexpr int kLargeBinWords = 12288;      // the default where that leaves >= 64 bins per SM
constexpr int kMaxSliceVerts = 56320;      // + the zero slot, within one CTA's shared memory
constexpr int kMaxPairIds = 2048;          // longer (row, slice) pairs are cut into pieces
constexpr int kMaxBinWords = 28160;
struct SliceBlocks {
  bool ready = false;
  int32_t slice_verts = 0;   // source ids per slice
  int32_t bin_words = 0;     // shared-memory words per bin
  int32_t ndst = 0;          // rows with in-edges: [0, ndst)
  int32_t nsrc = 0;          // largest source id + 1
  int32_t nslices = 0;
  int32_t npairs = 0;        // (row, slice) pairs
  int32_t nbins = 0;
  int32_t ngroups = 0;       // phase-1 groups of 32 pair slots
  int32_t nruns = 0;         // (slice, length class) runs of groups
  int32_t nunits = 0;
  int32_t nctas = 0;         // phase-1 grid (one CTA per SM)
  int64_t m = 0;
  int64_t elems = 0;         // phase-1 stream length with padding
  int32_t part_len = 0;      // floats in part (bins + the junk slot)
  // phase 1
  uint16_t *src = nullptr;   // slice-local source ids, sliced-ELL per group
  int4 *run = nullptr;       // {first group, slice, first id, (rows << 8) | (log2 L << 4) | log2 B}
  // {run, first group, end group, 0}: pieces of runs, in run order
  int4 *seg = nullptr;
  int32_t nsegs = 0;
  // {first segment, end segment, slice, 0}: units of the flat launch, then
  // of the other, each consecutive segments of one slice; CTAs take them in
  // order from a counter
  int4 *unit = nullptr;
  int32_t nunits_flat = 0;
  int32_t *dest = nullptr;   // per pair slot (ngroups x 32): index into part
  float *part = nullptr;     // bin-major partials, one junk slot after the last bin
  // phase 2
  int32_t *binbase = nullptr;  // nbins + 1: first partial of each bin (multiple of 4)
  uint16_t *idx = nullptr;   // per pair, in (row, slice) order: position in its bin's block
  int32_t *rowq = nullptr;   // ndst + 1: the pairs of row u are idx[rowq[u] .. rowq[u + 1])
  int4 *bin = nullptr;       // {row0, row1, q0, q1}: rows and pair range
  size_t bytes = 0;          // device bytes held
};

// Builds the layout from the renumbered in-CSR of g (unweighted).  Leaves
// sb->ready false (and returns cudaSuccess) when the graph does not fit the
// layout's limits or has more than max_pairs (row, slice) pairs.
// slice_verts / bin_words: 0 for the defaults.
cudaError_t BuildSliceBlocks(const DeviceGraph &g, int slice_verts, int bin_words,
                             int64_t max_pairs, SliceBlocks *sb, cudaStream_t s,
                             std::string *err);
void FreeSliceBlocks(SliceBlocks *sb);

// Kernel-side view of one sweep of the slice-blocked path.
struct BlockedArgs {
  // phase 1
  const uint16_t *__restrict__ src;
  const int4 *__restrict__ run;
  const int4 *__restrict__ seg;
  const int4 *__restrict__ unit;
  int32_t nunits_flat;       // units [0, nunits_flat) flat, [nunits_flat, nunits) the others
  int32_t nunits;
  const int32_t *__restrict__ dest;
  int32_t slice_verts;
  int32_t nsrc;
  int32_t part_len;          // floats in part[]
  int32_t bin_words;         // shared-memory words of partials per bin
  float *part;
  // phase 2
  const int32_t *__restrict__ binbase;
  const uint16_t *__restrict__ idx;
  const int32_t *__restrict__ rowq;
  const int4 *__restrict__ bin;
  int32_t nbins;
  int32_t n;                 // vertices (rows [ndst, n) have no in-edges)
  int32_t ndst;
  int32_t zero_blocks;       // phase-2 blocks after the bins, each for 4 x threads rows
  int32_t kind;              // kKindPlain or kKindPPR
  const int32_t *__restrict__ rowoff;
  const int32_t *__restrict__ odeg;   // directed: out-degree per row; else nullptr
  const float *__restrict__ base_vec; // PPR: (1-d) t per row
  float base_scalar;
  float damping;
  float *score;
  float *contrib;            // read by phase 1, rewritten by phase 2
  // grid reduction of phase 2
  double *part1;
  double *part2;
  unsigned *tick1;
  double *trace;
  SweepCtl *ctl;
  int32_t nblocks;           // phase-2 grid
  double epsilon;
};

// Phase 1 for the runs of one block per pair (flat) or the others.
const void *SlicePartialKernel(bool flat);
const void *BinRowKernel(const SliceBlocks &sb);
int BinRowThreads(const SliceBlocks &sb);
constexpr int kSliceThreads = kSliceWarps * 32;
// Phase-2 grid: the bins, then blocks for the rows without in-edges.
int BinRowGrid(const SliceBlocks &sb, int64_t n);
size_t SliceSmemBytes(const SliceBlocks &sb);
size_t BinSmemBytes(const SliceBlocks &sb);

}  // namespace prgpu

#endif  // GAPBS_B200_ENGINE_BLOCKED_H_
