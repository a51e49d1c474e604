// blocked_prep.cu -- builds the slice-blocked layout (blocked.h) on the device,
// once per upload, from the renumbered in-CSR.
//
//  1. Every in-edge v -> u gets the key slice(v) = v / slice_verts; a stable
//     radix sort by that key puts the entries in (slice, row, original entry)
//     order.  A pair (row, slice) starts where the slice or the row changes,
//     and a pair longer than kMaxPairIds is cut into pieces of kMaxPairIds
//     (each a pair of its own); pairs are numbered in that order (k) and
//     know their first entry and length.
//  2. Rows are cut into bins of consecutive rows whose pairs plus rows fit in
//     bin_words shared-memory words (row u costs its pair count + 1): the bin
//     of u is floor(S(u) / W') with S the exclusive scan of the costs and
//     W' = bin_words - (largest row cost) - 3, so no bin overflows (its block
//     of partials is rounded up to whole float4) and none is empty.
//  3. Bin-major position of every pair: a stable sort by (bin, flat class or
//     not, slice, length class) gives each bin's block of partials: the
//     pairs of the flat classes (one block of ids per pair) slice-major,
//     then the others slice-major; blocks start on multiples of four floats.
//  4. Phase-1 order: a stable sort by (slice, length class).  Each (slice,
//     class) run is cut into groups of P = 32 / L pairs, L lanes per pair
//     (1..32, chosen per run from its pair count and its longest pair by
//     an instruction estimate, RunLogL).  A group is a matrix
//     of rows x 32 lanes of blocks of B ids (B = 1, 2, 4 or 8 by class):
//     block j of the group's pair p sits in row j / L, lane p L + j % L;
//     rows = the blocks of the run's longest pair over L, rounded up, the
//     same for every group of the run.
//     Padding ids point to the zero entry after the slice.  Pair slot
//     32 g + p of group g has dest[slot] = the pair's bin-major position
//     (a junk slot for padding).
//  5. A stable sort of the pairs by row gives the phase-2 order (row,
//     slice): per pair its position in its bin's block; row u's pairs are
//     idx[rowq[u] .. rowq[u + 1]).
//  6. Phase-1 work is cut, per launch (flat runs / the others), into
//     segments: pieces of one run of about 1 / (6 x CTAs) of the launch's
//     estimated instruction count; consecutive segments of one slice are
//     joined into units up to that size, so that short runs share one load
//     of their slice; CTAs take units in order from a counter.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <string>
#include <vector>

#include "blocked.h"

namespace prgpu {

namespace {

inline unsigned Blocks(int64_t count, int threads) {
  return static_cast<unsigned>((count + threads - 1) / threads);
}

int BitsFor(int64_t x) {  // bits needed for values in [0, x)
  int b = 1;
  while ((int64_t(1) << b) < x) b++;
  return b;
}

// Length class of a pair: lengths 1, 2, 3-4 and 5-8 (one block of 1, 2, 4
// or 8 ids: the flat classes 0, 1, 3, 7), then whole 8-id blocks 2..8,
// then four classes per doubling of the block count.  All pairs of a class
// share the block size B; every class past the flat ones has B = 8.
__host__ __device__ inline int PairClass(int len) {
  if (len <= 2) return len - 1;
  if (len <= 4) return 3;  // one block of 4 ids (a length-3 pair pads one)
  if (len <= 8) return 7;  // one block of 8 ids
  const int nb = (len + 7) >> 3;
  if (nb <= 8) return 6 + nb;
  int lg = 3;
  while ((nb >> (lg + 1)) != 0) lg++;
  return 15 + 4 * (lg - 3) + ((nb >> (lg - 2)) & 3);
}
constexpr int kClassBits = 6;

// log2 of the block size of a class
__host__ __device__ inline int ClassLogB(int cls) {
  if (cls >= 7) return 3;   // length >= 8
  if (cls >= 3) return 2;   // 4..7
  if (cls >= 1) return 1;   // 2..3
  return 0;                 // 1
}

__global__ void rowid_kernel(int32_t ndst, const int32_t *__restrict__ rowoff, int32_t *rowid) {
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= ndst) return;
  const int32_t u = static_cast<int32_t>(warp);
  for (int32_t e = rowoff[u] + lane; e < rowoff[u + 1]; e += 32) rowid[e] = u;
}

__global__ void slice_key_kernel(int64_t m, const int32_t *__restrict__ col, int32_t slice_verts,
                                 uint16_t *key, int32_t *val) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  key[i] = static_cast<uint16_t>(col[i] / slice_verts);
  val[i] = static_cast<int32_t>(i);
}

// Entry j of the (slice, row) order = CSR entry perm[j]: its slice-local
// source id and row.
__global__ void entry_kernel(int64_t m, const int32_t *__restrict__ perm,
                             const uint16_t *__restrict__ key, const int32_t *__restrict__ col,
                             const int32_t *__restrict__ rowid, int32_t slice_verts,
                             uint16_t *lid, int32_t *row_s) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int32_t e = perm[j];
  lid[j] = static_cast<uint16_t>(col[e] - static_cast<int32_t>(key[j]) * slice_verts);
  row_s[j] = rowid[e];
}

// flag[j] = 1 where entry j starts a new (slice, row) pair.
__global__ void head_flag_kernel(int64_t count, const uint16_t *__restrict__ key,
                                 const int32_t *__restrict__ row, int32_t *flag) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= count) return;
  int32_t f = j == 0;
  if (j > 0) f = (row[j] != row[j - 1]) || (key && key[j] != key[j - 1]);
  flag[j] = f;
}

// A (slice, row) pair longer than kMaxPairIds is cut into pieces of
// kMaxPairIds ids; each piece is a pair of its own (phase 2 sums all of a
// row's pairs), so that no group of phase 1 is longer than one warp's fair
// share of a CTA's work.
__global__ void piece_flag_kernel(int64_t m, const int32_t *__restrict__ incl,
                                  const int32_t *__restrict__ first, int32_t *flag) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= m || flag[j]) return;
  const int64_t e = j - first[incl[j] - 1];
  if (e % kMaxPairIds == 0) flag[j] = 1;
}

__global__ void pair_start_kernel(int64_t m, const int32_t *__restrict__ flag,
                                  const int32_t *__restrict__ incl, int32_t *first) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= m || !flag[j]) return;
  first[incl[j] - 1] = static_cast<int32_t>(j);
}

__global__ void max_row_cost_kernel(int32_t ndst, const int32_t *__restrict__ cnt, int32_t *out) {
  const int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int32_t v = u < ndst ? cnt[u] + 1 : 0;
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, v);
}

__global__ void pair_kernel(int64_t m, const int32_t *__restrict__ flag,
                            const int32_t *__restrict__ incl, const int32_t *__restrict__ row_s,
                            const uint16_t *__restrict__ key, int32_t *pair_u, int32_t *pair_c,
                            int32_t *pair_pos) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= m || !flag[j]) return;
  const int32_t k = incl[j] - 1;
  pair_u[k] = row_s[j];
  pair_c[k] = key[j];
  pair_pos[k] = static_cast<int32_t>(j);
}

__global__ void pair_len_kernel(int64_t npairs, int64_t m, const int32_t *__restrict__ pair_pos,
                                int32_t *pair_len) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  const int64_t end = k + 1 < npairs ? pair_pos[k + 1] : m;
  pair_len[k] = static_cast<int32_t>(end - pair_pos[k]);
}

__global__ void count_pairs_kernel(int64_t npairs, const int32_t *__restrict__ pair_u,
                                   int32_t *cnt) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  atomicAdd(cnt + pair_u[k], 1);
}

__global__ void row_cost_kernel(int32_t ndst, const int32_t *__restrict__ cnt, int64_t *cost) {
  const int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u >= ndst) return;
  cost[u] = static_cast<int64_t>(cnt[u]) + 1;
}

__global__ void bin_of_kernel(int32_t ndst, const int64_t *__restrict__ S, int64_t wp,
                              int32_t *binof, int32_t *bin_row0) {
  const int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u >= ndst) return;
  const int32_t b = static_cast<int32_t>(S[u] / wp);
  binof[u] = b;
  if (u == 0 || static_cast<int32_t>(S[u - 1] / wp) != b) bin_row0[b] = static_cast<int32_t>(u);
}

// Block size of bin b rounded up to whole float4; entry nbins is the junk
// slot (four floats) that padding pair slots write to.
__global__ void bin_size_kernel(int32_t nbins, const int32_t *__restrict__ bin_row0,
                                const int32_t *__restrict__ pq, int32_t *size4) {
  const int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b > nbins + 1) return;
  if (b >= nbins) {
    size4[b] = b == nbins ? 4 : 0;
    return;
  }
  const int32_t cnt = pq[bin_row0[b + 1]] - pq[bin_row0[b]];
  size4[b] = (cnt + 3) & ~3;
}

// Classes whose runs have one block of B ids per pair and one lane per pair
// (lengths 1, 2, 3-4 and 5-8): their runs are flat (FlatShape below).
__host__ __device__ inline bool ClassFlat(int cls) {
  return cls == 0 || cls == 1 || cls == 3 || cls == 7;
}

// Sort keys of the pairs: (bin, slice, class) for the bin-major order and
// (slice, class) for the phase-1 order; values: pair numbers.
__global__ void pair_keys_kernel(int64_t npairs, const int32_t *__restrict__ pair_u,
                                 const int32_t *__restrict__ pair_c,
                                 const int32_t *__restrict__ pair_len,
                                 const int32_t *__restrict__ binof, int sbits, uint64_t *key_bin,
                                 uint32_t *key_slice, int32_t *val_a, int32_t *val_b) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  const uint64_t cls = static_cast<uint64_t>(PairClass(pair_len[k]));
  const uint64_t c = static_cast<uint64_t>(pair_c[k]);
  // inside a bin: the pairs of flat classes first, then the others (each
  // slice-major), so that each phase-1 launch fills one contiguous piece of
  // every bin, in slice order
  const uint64_t other = ClassFlat(static_cast<int>(cls)) ? 0 : 1;
  key_bin[k] = (static_cast<uint64_t>(binof[pair_u[k]]) << (1 + sbits + kClassBits)) |
               (other << (sbits + kClassBits)) | (c << kClassBits) | cls;
  key_slice[k] = static_cast<uint32_t>((c << kClassBits) | cls);
  val_a[k] = static_cast<int32_t>(k);
  val_b[k] = static_cast<int32_t>(k);
}

// log2 of the lanes L that share one pair of a run, chosen per run from its
// pair count P and its longest pair (nb blocks of B ids): a group holds
// 32 / L pairs and rows = ceil(nb / L) blocks per lane, so small L pads
// fewer ids (rows round up less) but leaves pair slots of a short run empty
// and large L the reverse.  The choice minimises the estimated instructions
// of the run, per lane: groups x (rows x (4 B + 6) + 2 B + 3 log2 L + 10)
// (a block's loads and sums per row, the group's closing tree, shuffles and
// store), ties to the larger L, among the L that keep rows at most
// kMaxRunRows (or L = 32): one lane per long pair would leave few groups,
// and so few busy warps, on all but the largest graphs.  Flat classes keep
// one lane (one block per pair); for the others L = 1 still gives rows >= 2
// (their pairs have at least two blocks), so their runs never take the flat
// shape.
constexpr int kMaxRunRows = 16;
__host__ __device__ inline int RunLogL(int cls, int64_t npairs, int nb) {
  if (ClassFlat(cls)) return 0;
  const int64_t B = int64_t(1) << ClassLogB(cls);
  int best_ll = 5;
  int64_t best = -1;
  for (int ll = 0; ll <= 5; ll++) {
    const int64_t per = 32 >> ll;
    const int64_t groups = (npairs + per - 1) / per;
    const int64_t rows = (nb + (1 << ll) - 1) >> ll;
    if (rows > kMaxRunRows && ll < 5) continue;
    const int64_t c = groups * (rows * (4 * B + 6) + 2 * B + 3 * ll + 10);
    if (best < 0 || c <= best) {
      best = c;
      best_ll = ll;
    }
  }
  return best_ll;
}

// Bin-major position of the pair at sorted rank r: its bin's base plus its
// rank inside the bin (the pairs of a bin's rows are consecutive ranks,
// starting at pq[row0]).
__global__ void bin_pos_kernel(int64_t npairs, const int32_t *__restrict__ order,
                               const int32_t *__restrict__ pair_u,
                               const int32_t *__restrict__ binof,
                               const int32_t *__restrict__ bin_row0,
                               const int32_t *__restrict__ pq, const int32_t *__restrict__ binbase,
                               int32_t *ppos) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= npairs) return;
  const int32_t k = order[r];
  const int32_t b = binof[pair_u[k]];
  ppos[k] = binbase[b] + static_cast<int32_t>(r - pq[bin_row0[b]]);
}

// Runs of equal (slice, class) keys in the phase-1 order.
__global__ void run_flag_kernel(int64_t npairs, const uint32_t *__restrict__ key,
                                int32_t *flag) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= npairs) return;
  flag[i] = i == 0 || key[i] != key[i - 1];
}

__global__ void run_start_kernel(int64_t npairs, const int32_t *__restrict__ flag,
                                 const int32_t *__restrict__ run_incl, int32_t *run_start) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= npairs || !flag[i]) return;
  run_start[run_incl[i] - 1] = static_cast<int32_t>(i);
}

// Runs of one block per pair (rows 1, one lane per pair) go to the flat
// launch of phase 1.
__host__ __device__ inline bool FlatShape(int code) { return (code >> 4) == 16; }


// The longest pair of each run: the pairs of a run are consecutive in the
// phase-1 order, so the lanes of a warp that share a run join their lengths
// first and one of them updates it.
__global__ void run_max_kernel(int64_t npairs, const int32_t *__restrict__ order,
                               const int32_t *__restrict__ run_incl,
                               const int32_t *__restrict__ pair_len, int32_t *run_max) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= npairs) return;
  const int32_t r = run_incl[i] - 1;
  const unsigned peers = __match_any_sync(__activemask(), r);
  const int32_t len = __reduce_max_sync(peers, static_cast<unsigned>(pair_len[order[i]]));
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicMax(run_max + r, len);
}

// Lanes per pair of each run (RunLogL).
__global__ void run_lanes_kernel(int32_t nruns, int64_t npairs,
                                 const int32_t *__restrict__ run_start,
                                 const uint32_t *__restrict__ key,
                                 const int32_t *__restrict__ run_max, int32_t *run_ll) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  const int64_t end = r + 1 < nruns ? run_start[r + 1] : npairs;
  const int cls = static_cast<int>(key[run_start[r]] & ((1u << kClassBits) - 1));
  const int lb = ClassLogB(cls);
  const int nb = (run_max[r] + (1 << lb) - 1) >> lb;
  run_ll[r] = RunLogL(cls, end - run_start[r], nb);
}

// Groups of each (slice, class) run: its pairs, 32 / lanes to a group; a
// flat run is padded to whole blocks of 8 / B groups (32 chunks of 16 bytes).
__global__ void run_groups_kernel(int32_t nruns, int64_t npairs,
                                  const int32_t *__restrict__ run_start,
                                  const uint32_t *__restrict__ key,
                                  const int32_t *__restrict__ run_ll, int32_t *run_groups) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  const int64_t end = r + 1 < nruns ? run_start[r + 1] : npairs;
  const int cls = static_cast<int>(key[run_start[r]] & ((1u << kClassBits) - 1));
  const int per = 32 >> run_ll[r];
  int32_t groups = static_cast<int32_t>((end - run_start[r] + per - 1) / per);
  if (ClassFlat(cls)) {
    const int q = 8 >> ClassLogB(cls);
    groups = (groups + q - 1) / q * q;
  }
  run_groups[r] = groups;
}

// Slot of the pair at phase-1 rank i (group * 32 + its place in the group);
// the run of each group.
__global__ void slot_kernel(int64_t npairs, const int32_t *__restrict__ order,
                            const int32_t *__restrict__ run_incl,
                            const int32_t *__restrict__ run_start,
                            const int32_t *__restrict__ run_gbase,
                            const int32_t *__restrict__ run_ll,
                            const int32_t *__restrict__ ppos, int32_t *slot_of,
                            int32_t *group_run, int32_t *dest) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= npairs) return;
  const int32_t r = run_incl[i] - 1;
  const int per = 32 >> run_ll[r];
  const int32_t rank = static_cast<int32_t>(i - run_start[r]);
  const int32_t grp = run_gbase[r] + rank / per;
  const int32_t slot = grp * 32 + rank % per;
  const int32_t k = order[i];
  slot_of[k] = slot;
  dest[slot] = ppos[k];
  if (rank % per == 0) group_run[grp] = r;
}

// Shape of each run: 2^ll lanes per pair, blocks of 2^lb ids, rows = the
// blocks of its longest pair over the lanes; ids per group = rows x 32 x B.
__global__ void run_shape_kernel(int32_t nruns, const int32_t *__restrict__ run_start,
                                 const uint32_t *__restrict__ key,
                                 const int32_t *__restrict__ run_max,
                                 const int32_t *__restrict__ run_ll,
                                 const int32_t *__restrict__ run_groups, int32_t *run_code,
                                 int64_t *run_gsize, int64_t *run_ids) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r > nruns) return;
  if (r == nruns) {
    run_ids[r] = 0;
    return;
  }
  const int cls = static_cast<int>(key[run_start[r]] & ((1u << kClassBits) - 1));
  const int lb = ClassLogB(cls), ll = run_ll[r];
  const int nb = (run_max[r] + (1 << lb) - 1) >> lb;
  const int rows = (nb + (1 << ll) - 1) >> ll;
  run_code[r] = (rows << 8) | (ll << 4) | lb;
  run_gsize[r] = (static_cast<int64_t>(32) * rows) << lb;
  run_ids[r] = run_gsize[r] * run_groups[r];
}

__global__ void run_table_kernel(int32_t nruns, const int32_t *__restrict__ run_start,
                                 const uint32_t *__restrict__ key,
                                 const int32_t *__restrict__ run_gbase,
                                 const int64_t *__restrict__ run_ibase,
                                 const int32_t *__restrict__ run_code, int4 *run) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  run[r] = make_int4(run_gbase[r], static_cast<int32_t>(key[run_start[r]] >> kClassBits),
                     static_cast<int32_t>(run_ibase[r]), run_code[r]);
}

__global__ void fill_u16_kernel(int64_t count, uint16_t value, uint16_t *out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < count) out[i] = value;
}

__global__ void fill_i32_kernel(int64_t count, int32_t value, int32_t *out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < count) out[i] = value;
}

__global__ void iota_kernel(int64_t count, int32_t *out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < count) out[i] = static_cast<int32_t>(i);
}

// Entry j (pair k, its e-th id) of a pair of a flat run (one block of B ids
// per pair): pair P of the run sits in block P / (32 Q) of 256 ids
// (Q = 8 / B pairs per 16-byte chunk), chunk P % 32 of it, place (P / 32) % Q
// in the chunk, position e: lane c of a warp reading chunk c of a block
// holds pairs c, c + 32, ..., so the warp's stores of the pairs' partials
// and loads of their dests are lane-consecutive.  Entries of the other
// runs are placed by place_run_ids_kernel.
__global__ void scatter_ids_kernel(int64_t m, const int32_t *__restrict__ incl,
                                   const int32_t *__restrict__ pair_pos,
                                   const int32_t *__restrict__ slot_of,
                                   const int32_t *__restrict__ group_run,
                                   const int4 *__restrict__ run,
                                   const uint16_t *__restrict__ lid, uint16_t *src) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int32_t k = incl[j] - 1;
  const int32_t e = static_cast<int32_t>(j - pair_pos[k]);
  const int32_t slot = slot_of[k];
  const int32_t grp = slot >> 5;
  const int4 rd = run[group_run[grp]];
  if (!FlatShape(rd.w)) return;
  const int lb = rd.w & 15;
  const int64_t P = static_cast<int64_t>(grp - rd.x) * 32 + (slot & 31);
  const int64_t in_blk = P % (256 >> lb);
  const int64_t pos = static_cast<int64_t>(rd.z) + (P / (256 >> lb)) * 256 +
                      (in_blk & 31) * 8 + ((in_blk >> 5) << lb) + e;
  src[pos] = lid[j];
}

// The ids of a pair of a run that is not flat (blocks of 8 ids, L lanes,
// rows rows: S = 8 rows load rounds; round s = 8 row + k is the k-th id of
// every lane's block of that row, one shared-memory load of the warp).  The
// pair's ids are ordered by bank (id mod 32), rotated by the pair's first
// lane p L so that pairs of a group start on different banks, and the q-th
// id goes to round q mod S, lane p L + q / S: within a round the pair's ids
// then fall on different banks wherever its banks hold at most S ids each
// (ids in source order put ~3.5 lanes on one bank per load; this
// placement about 1.6-2.2 for the long pairs of 16 and 32 lanes).  One
// thread per pair (at most kMaxPairIds ids), a counting sort by bank.
__global__ void place_run_ids_kernel(int64_t npairs, const int32_t *__restrict__ pair_pos,
                                     const int32_t *__restrict__ pair_len,
                                     const int32_t *__restrict__ slot_of,
                                     const int32_t *__restrict__ group_run,
                                     const int4 *__restrict__ run,
                                     const int64_t *__restrict__ run_gsize,
                                     const uint16_t *__restrict__ lid, uint16_t *src) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  const int32_t slot = slot_of[k];
  const int32_t grp = slot >> 5;
  const int32_t r = group_run[grp];
  const int4 rd = run[r];
  if (FlatShape(rd.w)) return;  // placed by scatter_ids_kernel
  const int ll = (rd.w >> 4) & 15, rows = rd.w >> 8;
  const int p = slot & 31;                 // pair within the group
  const int first_lane = p << ll;
  const int S = rows * 8;
  const int32_t j0 = pair_pos[k], len = pair_len[k];
  int start[32];
#pragma unroll
  for (int b = 0; b < 32; b++) start[b] = 0;
  for (int32_t e = 0; e < len; e++) start[(lid[j0 + e] - first_lane) & 31]++;
  int acc = 0;
#pragma unroll
  for (int b = 0; b < 32; b++) {
    const int c = start[b];
    start[b] = acc;
    acc += c;
  }
  const int64_t gbase = static_cast<int64_t>(rd.z) + static_cast<int64_t>(grp - rd.x) * run_gsize[r];
  for (int32_t e = 0; e < len; e++) {
    const uint16_t v = lid[j0 + e];
    const int q = start[(v - first_lane) & 31]++;
    const int round = q % S, lane = first_lane + q / S;
    src[gbase + ((static_cast<int64_t>(round >> 3) * 32 + lane) << 3) + (round & 7)] = v;
  }
}

// Phase-2 stream element j2 = pair k2[j2] of row u2[j2]: its position in
// its bin's block.
__global__ void index_kernel(int64_t npairs, const int32_t *__restrict__ k2,
                             const int32_t *__restrict__ u2, const int32_t *__restrict__ binof,
                             const int32_t *__restrict__ binbase,
                             const int32_t *__restrict__ ppos, uint16_t *idx) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= npairs) return;
  idx[j] = static_cast<uint16_t>(ppos[k2[j]] - binbase[binof[u2[j]]]);
}

__global__ void bin_table_kernel(int32_t nbins, const int32_t *__restrict__ bin_row0,
                                 const int32_t *__restrict__ pq, int4 *bin) {
  const int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  const int32_t row0 = bin_row0[b], row1 = bin_row0[b + 1];
  bin[b] = make_int4(row0, row1, pq[row0], pq[row1]);
}


// Estimated work of one group of a run (shape code), in thread instructions
// (the kernels are bound by issue): a flat group is 32 pairs of B ids at
// about 4 B + 12 each; another group is rows x 32 lanes of items at about
// 4 B + 8 each, plus about 30 per lane to close the group.
inline int64_t GroupCost(int code, int flat) {
  const int64_t B = int64_t(1) << (code & 15), rows = code >> 8;
  return flat ? 32 * (4 * B + 12) : rows * 32 * (4 * B + 8) + 32 * 30;
}

__global__ void max_kernel(int64_t m, const int32_t *__restrict__ col, int32_t *out) {
  int32_t v = -1;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    v = max(v, col[i]);
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, v);
}

// Temporary device buffers of the build, freed together.
class Temps {
 public:
  ~Temps() { Release(); }
  template <typename T>
  cudaError_t Get(T **p, int64_t count) {
    *p = nullptr;
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * static_cast<size_t>(std::max<int64_t>(count, 1)));
    if (e == cudaSuccess) {
      ptrs_.push_back(q);
      *p = static_cast<T *>(q);
    }
    return e;
  }
  void Drop(const void *p) {
    for (auto &q : ptrs_)
      if (q == p) {
        cudaFree(q);
        q = nullptr;
      }
  }
  void Release() {
    for (void *q : ptrs_)
      if (q) cudaFree(q);
    ptrs_.clear();
  }

 private:
  std::vector<void *> ptrs_;
};

template <typename T>
cudaError_t Keep(SliceBlocks *sb, T **p, int64_t count) {
  *p = nullptr;
  const size_t bytes = sizeof(T) * static_cast<size_t>(std::max<int64_t>(count, 1));
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
  if (e == cudaSuccess) sb->bytes += bytes;
  return e;
}

// CUB scratch, grown on demand and reused.
struct CubTemp {
  Temps *tmp;
  void *ptr = nullptr;
  size_t bytes = 0;
  cudaError_t Need(size_t b) {
    if (b <= bytes) return cudaSuccess;
    if (ptr) tmp->Drop(ptr);
    char *p = nullptr;
    cudaError_t e = tmp->Get(&p, static_cast<int64_t>(b));
    ptr = p;
    bytes = e == cudaSuccess ? b : 0;
    return e;
  }
};

}  // namespace

void FreeSliceBlocks(SliceBlocks *sb) {
  void *ptrs[] = {sb->src, sb->run, sb->seg, sb->unit, sb->dest, sb->part,
                  sb->binbase, sb->idx, sb->rowq, sb->bin};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  *sb = SliceBlocks();
}

#define SB_TRY(expr)                                                \
  do {                                                              \
    cudaError_t e_ = (expr);                                        \
    if (e_ != cudaSuccess) {                                        \
      *err = std::string("slice blocks: ") + #expr + ": " + cudaGetErrorString(e_); \
      FreeSliceBlocks(sb);                                          \
      return e_;                                                    \
    }                                                               \
  } while (0)

// Radix sorts and scans through one reusable scratch buffer.
#define SB_SORT_PAIRS(K, V, N, B0, B1)                                                   \
  do {                                                                                   \
    size_t b_ = 0;                                                                       \
    SB_TRY(cub::DeviceRadixSort::SortPairs(nullptr, b_, K, V, (N), (B0), (B1), s));      \
    SB_TRY(cub_tmp.Need(b_));                                                            \
    SB_TRY(cub::DeviceRadixSort::SortPairs(cub_tmp.ptr, b_, K, V, (N), (B0), (B1), s));  \
  } while (0)
#define SB_SCAN(KIND, IN, OUT, N)                                          \
  do {                                                                     \
    size_t b_ = 0;                                                         \
    SB_TRY(cub::DeviceScan::KIND(nullptr, b_, IN, OUT, (N), s));           \
    SB_TRY(cub_tmp.Need(b_));                                              \
    SB_TRY(cub::DeviceScan::KIND(cub_tmp.ptr, b_, IN, OUT, (N), s));       \
  } while (0)

cudaError_t BuildSliceBlocks(const DeviceGraph &g, int slice_verts, int bin_words,
                             int64_t max_pairs, SliceBlocks *sb, cudaStream_t s,
                             std::string *err) {
  FreeSliceBlocks(sb);
  if (slice_verts <= 0) slice_verts = kDefaultSliceVerts;
  const bool default_bins = bin_words <= 0;
  if (default_bins) bin_words = kDefaultBinWords;
  const int64_t m = g.m;
  const int32_t ndst = static_cast<int32_t>(g.bin_row_start[kBinZero]);
  if (g.weighted || m == 0 || ndst == 0) return cudaSuccess;  // not this layout's case
  const int T = 256;
  Temps tmp;
  CubTemp cub_tmp{&tmp};
  int dev = 0, sms = 0;
  SB_TRY(cudaGetDevice(&dev));
  SB_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

  // largest source id -> number of slices
  int32_t *d_max = nullptr;
  SB_TRY(tmp.Get(&d_max, 1));
  SB_TRY(cudaMemsetAsync(d_max, 0xff, sizeof(int32_t), s));
  max_kernel<<<std::min<unsigned>(Blocks(m, T), 4 * sms), T, 0, s>>>(m, g.col, d_max);
  int32_t hmax = -1;
  SB_TRY(cudaMemcpyAsync(&hmax, d_max, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SB_TRY(cudaStreamSynchronize(s));
  const int64_t nsrc = static_cast<int64_t>(hmax) + 1;
  const int64_t nslices = (nsrc + slice_verts - 1) / slice_verts;
  // slice ids and classes must fit the sort keys
  if (nslices > 65535) return cudaSuccess;
  const int sbits = BitsFor(nslices);

  // 1. entries in (slice, row) order; pairs
  int32_t *rowid = nullptr, *vals[2] = {nullptr, nullptr}, *row_s = nullptr;
  uint16_t *keys[2] = {nullptr, nullptr}, *lid = nullptr;
  SB_TRY(tmp.Get(&rowid, m));
  SB_TRY(tmp.Get(&keys[0], m));
  SB_TRY(tmp.Get(&keys[1], m));
  SB_TRY(tmp.Get(&vals[0], m));
  SB_TRY(tmp.Get(&vals[1], m));
  rowid_kernel<<<Blocks(static_cast<int64_t>(ndst) * 32, T), T, 0, s>>>(ndst, g.rowoff, rowid);
  slice_key_kernel<<<Blocks(m, T), T, 0, s>>>(m, g.col, slice_verts, keys[0], vals[0]);
  SB_TRY(cudaGetLastError());
  cub::DoubleBuffer<uint16_t> kb(keys[0], keys[1]);
  cub::DoubleBuffer<int32_t> vb(vals[0], vals[1]);
  SB_SORT_PAIRS(kb, vb, static_cast<int>(m), 0, sbits);
  const uint16_t *key = kb.Current();
  const int32_t *perm = vb.Current();
  SB_TRY(tmp.Get(&lid, m));
  SB_TRY(tmp.Get(&row_s, m));
  entry_kernel<<<Blocks(m, T), T, 0, s>>>(m, perm, key, g.col, rowid, slice_verts, lid, row_s);
  SB_TRY(cudaGetLastError());
  tmp.Drop(rowid);
  tmp.Drop(vb.Alternate());
  tmp.Drop(kb.Alternate());
  tmp.Drop(vb.Current());
  int32_t *hf = nullptr, *incl = nullptr;
  SB_TRY(tmp.Get(&hf, m));
  SB_TRY(tmp.Get(&incl, m));
  head_flag_kernel<<<Blocks(m, T), T, 0, s>>>(m, key, row_s, hf);
  SB_SCAN(InclusiveSum, hf, incl, static_cast<int>(m));
  {
    // cut long pairs into pieces: flags at every kMaxPairIds-th id of a pair
    int32_t npairs0 = 0, *first = nullptr;
    SB_TRY(cudaMemcpyAsync(&npairs0, incl + (m - 1), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SB_TRY(cudaStreamSynchronize(s));
    SB_TRY(tmp.Get(&first, npairs0));
    pair_start_kernel<<<Blocks(m, T), T, 0, s>>>(m, hf, incl, first);
    piece_flag_kernel<<<Blocks(m, T), T, 0, s>>>(m, incl, first, hf);
    SB_TRY(cudaGetLastError());
    SB_SCAN(InclusiveSum, hf, incl, static_cast<int>(m));
    tmp.Drop(first);
  }
  int32_t npairs = 0;
  SB_TRY(cudaMemcpyAsync(&npairs, incl + (m - 1), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SB_TRY(cudaStreamSynchronize(s));
  if (npairs > max_pairs) return cudaSuccess;  // the caller keeps the gather sweep
  // large graphs: bins twice as large while that still leaves at least 64
  // bins per SM (fewer, longer runs of each slice's partials in every bin;
  // measured at Kronecker scale 25: 1.77 against 1.82 ms per sweep)
  if (default_bins &&
      static_cast<int64_t>(npairs) + ndst >= int64_t(64) * sms * kLargeBinWords)
    bin_words = kLargeBinWords;
  int32_t *pair_u = nullptr, *pair_c = nullptr, *pair_pos = nullptr, *pair_len = nullptr;
  SB_TRY(tmp.Get(&pair_u, npairs));
  SB_TRY(tmp.Get(&pair_c, npairs));
  SB_TRY(tmp.Get(&pair_pos, npairs));
  SB_TRY(tmp.Get(&pair_len, npairs));
  pair_kernel<<<Blocks(m, T), T, 0, s>>>(m, hf, incl, row_s, key, pair_u, pair_c, pair_pos);
  pair_len_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, m, pair_pos, pair_len);
  SB_TRY(cudaGetLastError());
  tmp.Drop(row_s);
  tmp.Drop(hf);

  // 2. bins
  int32_t *cnt = nullptr, *pq = nullptr, *binof = nullptr, *bin_row0 = nullptr;
  int64_t *cost = nullptr, *S = nullptr;
  SB_TRY(tmp.Get(&cnt, ndst + 1));
  SB_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (ndst + 1), s));
  count_pairs_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, pair_u, cnt);
  SB_TRY(tmp.Get(&cost, ndst));
  SB_TRY(tmp.Get(&S, ndst));
  SB_TRY(tmp.Get(&pq, ndst + 1));
  row_cost_kernel<<<Blocks(ndst, T), T, 0, s>>>(ndst, cnt, cost);
  // the largest row cost (its pairs + 1, its bin block rounded to float4)
  // must leave room in a bin
  int32_t *d_maxc = nullptr, maxc = 0;
  SB_TRY(tmp.Get(&d_maxc, 1));
  SB_TRY(cudaMemsetAsync(d_maxc, 0, sizeof(int32_t), s));
  max_row_cost_kernel<<<Blocks(ndst, T), T, 0, s>>>(ndst, cnt, d_maxc);
  SB_TRY(cudaMemcpyAsync(&maxc, d_maxc, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SB_TRY(cudaStreamSynchronize(s));
  if (maxc + 3 > bin_words / 2) {
    FreeSliceBlocks(sb);
    return cudaSuccess;
  }
  const int64_t wp = bin_words - maxc - 3;
  SB_SCAN(ExclusiveSum, cost, S, ndst);
  SB_SCAN(ExclusiveSum, cnt, pq, ndst + 1);  // pq[ndst] = npairs
  int64_t last_S = 0;
  SB_TRY(cudaMemcpyAsync(&last_S, S + (ndst - 1), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SB_TRY(cudaStreamSynchronize(s));
  const int32_t nbins = static_cast<int32_t>(last_S / wp) + 1;
  SB_TRY(tmp.Get(&binof, ndst));
  SB_TRY(tmp.Get(&bin_row0, nbins + 1));
  bin_of_kernel<<<Blocks(ndst, T), T, 0, s>>>(ndst, S, wp, binof, bin_row0);
  SB_TRY(cudaMemcpyAsync(bin_row0 + nbins, &ndst, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  SB_TRY(cudaGetLastError());
  tmp.Drop(cost);
  tmp.Drop(S);

  // 3. bin-major positions
  int32_t *size4 = nullptr, *ppos = nullptr;
  SB_TRY(tmp.Get(&size4, nbins + 2));
  bin_size_kernel<<<Blocks(nbins + 2, T), T, 0, s>>>(nbins, bin_row0, pq, size4);
  SB_TRY(Keep(sb, &sb->binbase, nbins + 2));
  SB_SCAN(ExclusiveSum, size4, sb->binbase, nbins + 2);  // binbase[nbins] = junk slot
  int32_t part_len = 0;
  SB_TRY(cudaMemcpyAsync(&part_len, sb->binbase + nbins + 1, sizeof(int32_t),
                         cudaMemcpyDeviceToHost, s));
  uint64_t *kbin[2] = {nullptr, nullptr};
  uint32_t *kslice[2] = {nullptr, nullptr};
  int32_t *va[2] = {nullptr, nullptr}, *vs[2] = {nullptr, nullptr};
  SB_TRY(tmp.Get(&kbin[0], npairs));
  SB_TRY(tmp.Get(&kbin[1], npairs));
  SB_TRY(tmp.Get(&kslice[0], npairs));
  SB_TRY(tmp.Get(&kslice[1], npairs));
  SB_TRY(tmp.Get(&va[0], npairs));
  SB_TRY(tmp.Get(&va[1], npairs));
  SB_TRY(tmp.Get(&vs[0], npairs));
  SB_TRY(tmp.Get(&vs[1], npairs));
  pair_keys_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, pair_u, pair_c, pair_len, binof, sbits,
                                                   kbin[0], kslice[0], va[0], vs[0]);
  SB_TRY(cudaGetLastError());
  cub::DoubleBuffer<uint64_t> kbb(kbin[0], kbin[1]);
  cub::DoubleBuffer<int32_t> vab(va[0], va[1]);
  SB_SORT_PAIRS(kbb, vab, npairs, 0, BitsFor(nbins) + 1 + sbits + kClassBits);
  SB_TRY(tmp.Get(&ppos, npairs));
  bin_pos_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, vab.Current(), pair_u, binof, bin_row0,
                                                 pq, sb->binbase, ppos);
  SB_TRY(cudaGetLastError());
  tmp.Drop(kbin[0]);
  tmp.Drop(kbin[1]);
  tmp.Drop(va[0]);
  tmp.Drop(va[1]);

  // 4. phase-1 order, slots, groups
  cub::DoubleBuffer<uint32_t> ksb(kslice[0], kslice[1]);
  cub::DoubleBuffer<int32_t> vsb(vs[0], vs[1]);
  SB_SORT_PAIRS(ksb, vsb, npairs, 0, sbits + kClassBits);
  const uint32_t *key1 = ksb.Current();
  const int32_t *order1 = vsb.Current();
  int32_t *rflag = nullptr, *rincl = nullptr;
  SB_TRY(tmp.Get(&rflag, npairs));
  SB_TRY(tmp.Get(&rincl, npairs));
  run_flag_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, key1, rflag);
  SB_SCAN(InclusiveSum, rflag, rincl, npairs);
  int32_t nruns = 0;
  SB_TRY(cudaMemcpyAsync(&nruns, rincl + (npairs - 1), sizeof(int32_t), cudaMemcpyDeviceToHost,
                         s));
  SB_TRY(cudaStreamSynchronize(s));
  int32_t *run_start = nullptr, *run_groups = nullptr, *run_gbase = nullptr;
  SB_TRY(tmp.Get(&run_start, nruns));
  SB_TRY(tmp.Get(&run_groups, nruns + 1));
  SB_TRY(tmp.Get(&run_gbase, nruns + 1));
  run_start_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, rflag, rincl, run_start);
  int32_t *run_max = nullptr, *run_ll = nullptr;
  SB_TRY(tmp.Get(&run_max, nruns));
  SB_TRY(tmp.Get(&run_ll, nruns));
  SB_TRY(cudaMemsetAsync(run_max, 0, sizeof(int32_t) * nruns, s));
  run_max_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, order1, rincl, pair_len, run_max);
  run_lanes_kernel<<<Blocks(nruns, T), T, 0, s>>>(nruns, npairs, run_start, key1, run_max,
                                                   run_ll);
  run_groups_kernel<<<Blocks(nruns, T), T, 0, s>>>(nruns, npairs, run_start, key1, run_ll,
                                                   run_groups);
  SB_TRY(cudaMemsetAsync(run_groups + nruns, 0, sizeof(int32_t), s));
  SB_SCAN(ExclusiveSum, run_groups, run_gbase, nruns + 1);
  int32_t ngroups = 0;
  SB_TRY(cudaMemcpyAsync(&ngroups, run_gbase + nruns, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SB_TRY(cudaStreamSynchronize(s));
  if (static_cast<int64_t>(ngroups) * 32 > 0x7fffffffLL) {  // slots are int32
    FreeSliceBlocks(sb);
    return cudaSuccess;
  }
  const int32_t nslots = ngroups * 32;
  int32_t *slot_of = nullptr, *group_run = nullptr, *run_code = nullptr;
  int64_t *run_gsize = nullptr, *run_ids = nullptr, *run_ibase = nullptr;
  SB_TRY(tmp.Get(&slot_of, npairs));
  SB_TRY(tmp.Get(&group_run, ngroups));
  SB_TRY(tmp.Get(&run_code, nruns));
  SB_TRY(tmp.Get(&run_gsize, nruns));
  SB_TRY(tmp.Get(&run_ids, nruns + 1));
  SB_TRY(tmp.Get(&run_ibase, nruns + 1));
  SB_TRY(Keep(sb, &sb->dest, nslots));
  fill_i32_kernel<<<Blocks(nslots, T), T, 0, s>>>(nslots, part_len - 4, sb->dest);  // junk slot
  slot_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, order1, rincl, run_start, run_gbase, run_ll,
                                              ppos, slot_of, group_run, sb->dest);
  run_shape_kernel<<<Blocks(nruns + 1, T), T, 0, s>>>(nruns, run_start, key1, run_max, run_ll,
                                                      run_groups, run_code, run_gsize, run_ids);
  SB_TRY(cudaGetLastError());
  SB_SCAN(ExclusiveSum, run_ids, run_ibase, nruns + 1);
  int64_t elems = 0;
  SB_TRY(cudaMemcpyAsync(&elems, run_ibase + nruns, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SB_TRY(cudaStreamSynchronize(s));
  if (elems > 0x7fffffffLL - 64) {  // id offsets are int32
    FreeSliceBlocks(sb);
    return cudaSuccess;
  }
  SB_TRY(Keep(sb, &sb->run, nruns));
  run_table_kernel<<<Blocks(nruns, T), T, 0, s>>>(nruns, run_start, key1, run_gbase, run_ibase,
                                                  run_code, sb->run);
  SB_TRY(Keep(sb, &sb->src, elems + 64));
  fill_u16_kernel<<<Blocks(elems + 64, T), T, 0, s>>>(elems + 64,
                                                      static_cast<uint16_t>(slice_verts), sb->src);
  scatter_ids_kernel<<<Blocks(m, T), T, 0, s>>>(m, incl, pair_pos, slot_of, group_run, sb->run,
                                                lid, sb->src);
  place_run_ids_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, pair_pos, pair_len, slot_of,
                                                       group_run, sb->run, run_gsize, lid,
                                                       sb->src);
  SB_TRY(Keep(sb, &sb->part, part_len));
  SB_TRY(cudaMemsetAsync(sb->part, 0, sizeof(float) * part_len, s));
  SB_TRY(cudaGetLastError());

  // 5. phase-2 stream: pairs in (row, slice) order
  int32_t *ku[2] = {nullptr, nullptr}, *kk[2] = {nullptr, nullptr};
  SB_TRY(tmp.Get(&ku[0], npairs));
  SB_TRY(tmp.Get(&ku[1], npairs));
  SB_TRY(tmp.Get(&kk[0], npairs));
  SB_TRY(tmp.Get(&kk[1], npairs));
  SB_TRY(cudaMemcpyAsync(ku[0], pair_u, sizeof(int32_t) * npairs, cudaMemcpyDeviceToDevice, s));
  iota_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, kk[0]);
  cub::DoubleBuffer<int32_t> ub(ku[0], ku[1]), pb(kk[0], kk[1]);
  SB_SORT_PAIRS(ub, pb, npairs, 0, BitsFor(ndst));
  const int32_t *u2 = ub.Current(), *k2 = pb.Current();
  SB_TRY(Keep(sb, &sb->idx, npairs + 16));  // read in whole 16-byte words
  SB_TRY(cudaMemsetAsync(sb->idx, 0, sizeof(uint16_t) * (npairs + 16), s));
  index_kernel<<<Blocks(npairs, T), T, 0, s>>>(npairs, k2, u2, binof, sb->binbase, ppos, sb->idx);
  SB_TRY(Keep(sb, &sb->rowq, ndst + 1));
  SB_TRY(cudaMemcpyAsync(sb->rowq, pq, sizeof(int32_t) * (ndst + 1), cudaMemcpyDeviceToDevice, s));
  SB_TRY(Keep(sb, &sb->bin, nbins));
  bin_table_kernel<<<Blocks(nbins, T), T, 0, s>>>(nbins, bin_row0, pq, sb->bin);
  SB_TRY(cudaGetLastError());

  // 6. phase-1 work: each run cut into segments of about 1 / (6 G) of its
  //    launch's estimated work; consecutive segments of one slice joined
  //    into units up to that size (so short runs share one slice load);
  //    CTAs take units from a counter
  const int G = sms;
  std::vector<int32_t> rgb(nruns + 1);
  std::vector<int4> rtab(nruns);
  SB_TRY(cudaMemcpyAsync(rgb.data(), run_gbase, sizeof(int32_t) * (nruns + 1),
                         cudaMemcpyDeviceToHost, s));
  SB_TRY(cudaMemcpyAsync(rtab.data(), sb->run, sizeof(int4) * nruns, cudaMemcpyDeviceToHost, s));
  SB_TRY(cudaStreamSynchronize(s));
  std::vector<int4> segs, units;
  int32_t nunits_flat = 0;
  for (int flat = 1; flat >= 0; flat--) {
    double total = 0;
    for (int64_t r = 0; r < nruns; r++)
      if (FlatShape(rtab[r].w) == (flat != 0))
        total += static_cast<double>(GroupCost(rtab[r].w, flat)) * (rgb[r + 1] - rgb[r]);
    const double target = std::max(1.0, total / (6.0 * G));
    double unit_cost = 0;
    for (int64_t r = 0; r < nruns; r++) {
      if (FlatShape(rtab[r].w) != (flat != 0)) continue;
      const int32_t g0 = rgb[r], g1 = rgb[r + 1];
      const double gc = static_cast<double>(GroupCost(rtab[r].w, flat));
      // flat segments hold whole blocks of 8 / B groups
      const int64_t q = flat ? 8 >> (rtab[r].w & 15) : 1;
      int64_t per = std::max<int64_t>(1, static_cast<int64_t>(target / gc));
      per = (per + q - 1) / q * q;
      for (int64_t g = g0; g < g1; g += per) {
        const int32_t ge = static_cast<int32_t>(std::min<int64_t>(g1, g + per));
        const double c = gc * (ge - g);
        const bool join = !units.empty() && units.back().z == rtab[r].y &&
                          units.back().y == static_cast<int32_t>(segs.size()) &&
                          static_cast<int32_t>(units.size()) > (flat ? 0 : nunits_flat) &&
                          unit_cost + c <= target;
        segs.push_back(make_int4(static_cast<int32_t>(r), static_cast<int32_t>(g), ge, 0));
        if (join) {
          units.back().y++;
          unit_cost += c;
        } else {
          const int32_t sg = static_cast<int32_t>(segs.size()) - 1;
          units.push_back(make_int4(sg, sg + 1, rtab[r].y, 0));
          unit_cost = c;
        }
      }
    }
    if (flat) nunits_flat = static_cast<int32_t>(units.size());
  }
  const int32_t nunits = static_cast<int32_t>(units.size());
  const int32_t nsegs = static_cast<int32_t>(segs.size());
  SB_TRY(Keep(sb, &sb->seg, nsegs));
  SB_TRY(Keep(sb, &sb->unit, nunits));
  if (nsegs)
    SB_TRY(cudaMemcpyAsync(sb->seg, segs.data(), sizeof(int4) * nsegs, cudaMemcpyHostToDevice, s));
  if (nunits)
    SB_TRY(cudaMemcpyAsync(sb->unit, units.data(), sizeof(int4) * nunits, cudaMemcpyHostToDevice,
                           s));
  SB_TRY(cudaStreamSynchronize(s));  // the host vectors above feed async copies
  sb->nsegs = nsegs;

  sb->slice_verts = slice_verts;
  sb->bin_words = bin_words;
  sb->ndst = ndst;
  sb->nsrc = static_cast<int32_t>(nsrc);
  sb->nslices = static_cast<int32_t>(nslices);
  sb->npairs = npairs;
  sb->nbins = nbins;
  sb->ngroups = ngroups;
  sb->nruns = nruns;
  sb->nunits = nunits;
  sb->nunits_flat = nunits_flat;
  sb->nctas = G;
  sb->m = m;
  sb->elems = elems;
  sb->part_len = part_len;
  sb->ready = true;
  return cudaSuccess;
}

#undef SB_SCAN
#undef SB_SORT_PAIRS
#undef SB_TRY

}  // namespace prgpu
