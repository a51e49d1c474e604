// blocked.cu -- the two kernels of a slice-blocked pull sweep (see blocked.h).
//
// The replaced loop is src/pr_spmv.cc:46-54: for every row u, the float sum
// of contrib[v] over its in-neighbours, then new = base + d * sum, the FP64
// L1 change and (src/pr_spmv.cc:43-45) the next contrib = new / out_degree.
// Phase 1 (slice_partial_kernel) forms, per (row, source slice) pair, the
// float sum of that slice's contribs; phase 2 (bin_row_kernel) sums each
// row's pair partials in slice order and updates the row.  Every sum is a
// fixed tree over a fixed layout, so two runs give identical bits.
#include <cuda_runtime.h>

#include "blocked.h"
#include "common.cuh"
#include "sweep_reduce.cuh"

namespace prgpu {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint4 ld_stream_u4(const uint4 *p, uint64_t pol) {
  uint4 r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p), "l"(pol));
  return r;
}

// Shared-memory float at byte address base + 4 i (32-bit shared-window
// address), so that the compiler issues a shared load with 32-bit address
// arithmetic whatever it can prove about the pointer it came from.
__device__ __forceinline__ unsigned lds_u16(unsigned base, unsigned i) {
  unsigned short v;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(base + (i << 1)));
  return v;
}

__device__ __forceinline__ float lds_f32(unsigned base, unsigned i) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(base + (i << 2)));
  return v;
}

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Asynchronous global -> shared copies (cp.async): the issuing thread does
// not wait for the data, so many copies are in flight at once; completion is
// awaited with cp_async_wait_all() and then a barrier.
__device__ __forceinline__ void cp_async_4(float *smem_dst, const float *gmem_src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_16(float4 *smem_dst, const float4 *gmem_src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}



// The block of B ids a lane reads for one row of a group (B = 8, the block
// size of every run that is not flat), and its ids.
template <int B> struct IdBlock;
template <> struct IdBlock<8> {
  uint4 q;
  __device__ __forceinline__ void load(const uint16_t *p, uint64_t pol) {
    q = ld_stream_u4(reinterpret_cast<const uint4 *>(p), pol);
  }
  __device__ __forceinline__ unsigned id(int k) const {
    const unsigned w = k < 2 ? q.x : (k < 4 ? q.y : (k < 6 ? q.z : q.w));
    return (k & 1) ? (w >> 16) : (w & 0xffffu);
  }
};

// A warp's contiguous block of ng groups of one run (all of one shape: rows
// rows of 32 lanes x B ids, 2^ll lanes per pair) is one regular array: item
// i (row i % rows of group i / rows) of lane l sits at base + (32 i + l) B.
// Each lane streams its column with U items (64 bytes) in flight,
// keeps B running sums (one per position in a block), and at the end of
// each group joins them by a fixed tree, then across the pair's lanes by an
// xor tree; the pair's first lane writes the partial to part[dest[32 g + p]].
// dest is fetched one group ahead.
template <int B>
__device__ __forceinline__ void warp_run_groups(const BlockedArgs &a, const uint16_t *base,
                                                int g, int ng, int rows, int ll, unsigned svb,
                                                uint64_t pol) {
  constexpr int U = B >= 4 ? 32 / B : 8;
  const int lane = threadIdx.x & 31;
  const int p = lane >> ll;
  const int nitems = ng * rows;
  const int gend = g + ng;
  int d_next = ld_stream_s32(a.dest + static_cast<int64_t>(g) * 32 + p, pol);
  float acc[B];
#pragma unroll
  for (int k = 0; k < B; k++) acc[k] = 0.f;
  int row = 0;
  const uint16_t *col = base + lane * B;
  for (int i = 0; i < nitems; i += U) {
    IdBlock<B> q[U];
#pragma unroll
    for (int t = 0; t < U; t++)
      if (i + t < nitems) q[t].load(col + static_cast<int64_t>(i + t) * 32 * B, pol);
#pragma unroll
    for (int t = 0; t < U; t++) {
      if (i + t >= nitems) break;
#pragma unroll
      for (int k = 0; k < B; k++) acc[k] = __fadd_rn(acc[k], lds_f32(svb, q[t].id(k)));
      if (++row == rows) {
        // the group is complete
#pragma unroll
        for (int h = B / 2; h > 0; h >>= 1)
#pragma unroll
          for (int k = 0; k < h; k++) acc[k] = __fadd_rn(acc[k], acc[k + h]);
        float sum = acc[0];
        for (int o = (1 << ll) >> 1; o > 0; o >>= 1)
          sum = __fadd_rn(sum, __shfl_xor_sync(kFull, sum, o));
        const int d = d_next;
        if (g + 1 < gend) d_next = ld_stream_s32(a.dest + static_cast<int64_t>(g + 1) * 32 + p, pol);
        // d is a position in part[] by construction; the range check keeps a
        // layout fault from writing outside it
        if ((lane & ((1 << ll) - 1)) == 0 &&
            static_cast<unsigned>(d) < static_cast<unsigned>(a.part_len))
          st_hint_f32(a.part + d, sum, pol);
#pragma unroll
        for (int k = 0; k < B; k++) acc[k] = 0.f;
        row = 0;
        g++;
      }
    }
  }
}

// A warp's share of a flat run: blocks of 32 chunks of 16 bytes (8 ids),
// chunk c holding pairs c, c + 32, ... (8 / B pairs of B ids) of the block.
// Two blocks per step: every lane loads its chunk and the dests of its
// pairs (one coalesced load per pair place), sums each pair's B ids and
// stores the partials, each store lane-consecutive over the block's pairs.
__device__ __forceinline__ void warp_flat_pairs(const BlockedArgs &a, const uint16_t *base,
                                                int g, int ng, int lb, unsigned svb,
                                                uint64_t pol) {
  const int lane = threadIdx.x & 31;
  const int pp = 8 >> lb;      // pairs per chunk
  const int nblk = ng / pp;    // a block is pp groups (whole by the layout)
  const uint4 *c4 = reinterpret_cast<const uint4 *>(base);
  const int32_t *dst = a.dest + static_cast<int64_t>(g) * 32;
  for (int b0 = 0; b0 < nblk; b0 += 2) {
    uint4 q[2];
    int d[2][8];
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const int bk = b0 + t;
      if (bk < nblk) {
        q[t] = ld_stream_u4(c4 + bk * 32 + lane, pol);
        const int32_t *dp = dst + bk * 32 * pp + lane;
#pragma unroll
        for (int k = 0; k < 8; k++)
          if (k < pp) d[t][k] = ld_stream_s32(dp + 32 * k, pol);
      }
    }
#pragma unroll
    for (int t = 0; t < 2; t++) {
      if (b0 + t >= nblk) break;
      const unsigned w[4] = {q[t].x, q[t].y, q[t].z, q[t].w};
      float v[8];
#pragma unroll
      for (int k = 0; k < 8; k++)
        v[k] = lds_f32(svb, (k & 1) ? (w[k >> 1] >> 16) : (w[k >> 1] & 0xffffu));
      // pairwise tree: after level h, v[j << h] holds the sum of ids
      // [j 2^h, (j + 1) 2^h)
#pragma unroll
      for (int h = 0; h < 3; h++) {
        if (h >= lb) break;
#pragma unroll
        for (int j = 0; j < 8; j += 2 << h) v[j] = __fadd_rn(v[j], v[j + (1 << h)]);
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        if (j >= pp) break;
        const int dj = d[t][j];
        // v[(j << lb) & 7], selected without indexing registers at run time
        const float x = lb == 0 ? v[j] : (lb == 1 ? v[(2 * j) & 7] : (lb == 2 ? v[(4 * j) & 7] : v[0]));
        if (static_cast<unsigned>(dj) < static_cast<unsigned>(a.part_len))
          st_hint_f32(a.part + dj, x, pol);
      }
    }
  }
}

// Groups in one chunk of a phase-1 segment of the given run shape: flat
// runs two blocks of 32 chunks of 16 bytes (2 x 8 / B groups); the others
// enough groups for about 16 rows of items per lane.
template <bool FLAT>
__device__ __forceinline__ int ChunkGroups(int code) {
  if (FLAT) return 2 * (8 >> (code & 15));
  const int rows = code >> 8;
  return rows >= 16 ? 1 : 16 / rows;
}

// Phase 1: one CTA per SM takes units (consecutive segments of one slice,
// each segment a range of the groups of one (slice, class) run) in order
// from a counter until none is left: the runs of one
// block per pair (FLAT) or the others, the two kinds being two launches so
// that each is compiled for its own paths.  When the slice changes the CTA
// loads the slice's contribs into shared memory (plus a zero at index
// slice_verts, the id of padding entries); its warps take chunks of the
// unit from a shared counter, so that they finish the unit together.
template <bool FLAT>
__global__ void __launch_bounds__(kSliceThreads, 1)
slice_partial_kernel(const BlockedArgs a) {
  if (*reinterpret_cast<volatile const int *>(&a.ctl->loop.done)) return;
  extern __shared__ __align__(16) float sv[];
  __shared__ int s_unit;
  __shared__ int s_chunk;  // next chunk of the current unit
  const uint64_t ps = policy_evict_first();
  int cur_slice = -1;
  const int ubase = FLAT ? 0 : a.nunits_flat;
  const int ucount = FLAT ? a.nunits_flat : a.nunits - a.nunits_flat;
  int *next = &a.ctl->unit_next[FLAT ? 0 : 1];
  for (;;) {
    if (threadIdx.x == 0) s_unit = atomicAdd(next, 1);
    __syncthreads();  // also: every warp is done with the previous unit
    const int k = s_unit;
    if (k >= ucount) break;
    // no warp takes chunks of the previous unit any more: restart the count
    // (read only after the barrier below)
    if (threadIdx.x == 0) s_chunk = 0;
    const int4 un = a.unit[ubase + k];  // first segment, end segment, slice
    if (un.z != cur_slice) {
      const int v0 = un.z * a.slice_verts;
      const int cnt = min(a.slice_verts, a.nsrc - v0);
      const int n4 = cnt >> 2;
      const float4 *c4 = reinterpret_cast<const float4 *>(a.contrib + v0);
      float4 *sv4 = reinterpret_cast<float4 *>(sv);
      for (int i = threadIdx.x; i < n4; i += kSliceThreads) cp_async_16(sv4 + i, c4 + i);
      for (int i = (n4 << 2) + threadIdx.x; i < cnt; i += kSliceThreads)
        cp_async_4(sv + i, a.contrib + v0 + i);
      if (threadIdx.x == 0) sv[a.slice_verts] = 0.f;
      cp_async_wait_all();
      cur_slice = un.z;
    }
    __syncthreads();  // the slice is in place; s_unit may be overwritten next
    const unsigned svb = smem_addr(sv);
    // warps take chunks of the unit from a shared counter until none is
    // left: a chunk is a few groups of one segment (flat segments: whole
    // blocks of 8 / B groups), found by walking the unit's segments
    const int lane = threadIdx.x & 31;
    for (;;) {
      int c = 0;
      if (lane == 0) c = atomicAdd(&s_chunk, 1);
      c = __shfl_sync(kFull, c, 0);
      int sg = un.x, gw0 = 0, gw1 = 0;
      int4 rd = make_int4(0, 0, 0, 0);
      for (; sg < un.y; sg++) {
        const int4 seg = a.seg[sg];  // run, first group, end group
        rd = a.run[seg.x];           // first group, slice, first id, shape
        const int cg = ChunkGroups<FLAT>(rd.w);
        const int nch = (seg.z - seg.y + cg - 1) / cg;
        if (c < nch) {
          gw0 = seg.y + c * cg;
          gw1 = min(seg.z, gw0 + cg);
          break;
        }
        c -= nch;
      }
      if (sg >= un.y) break;
      const int rows = rd.w >> 8, ll = (rd.w >> 4) & 15, lb = rd.w & 15;
      const uint16_t *base =
          a.src + rd.z + (static_cast<int64_t>(gw0 - rd.x) * rows * 32 << lb);
      if (FLAT) {
        warp_flat_pairs(a, base, gw0, gw1 - gw0, lb, svb, ps);
      } else {
        // every run that is not flat has blocks of 8 ids (the layout's classes)
        warp_run_groups<8>(a, base, gw0, gw1 - gw0, rows, ll, svb, ps);
      }
    }
  }
}

// Phase 2: one CTA per bin of rows (then blocks for the rows without
// in-edges, on the first sweep only).  The bin's partials, one contiguous
// block of part[], and the bin's stretch of idx[] (per pair of its rows, in
// row order, the pair's position in the block) are copied into shared
// memory; then each thread takes rows u = row0 + t, + kBinThreads, ...: it
// sums the row's partials in slice order (positions idx[rowq[u] ..
// rowq[u + 1])) and updates the row, the next row's own data fetched
// before this one is written.
template <int kBinThreads>
__global__ void __launch_bounds__(kBinThreads)
bin_row_kernel(const BlockedArgs a) {
  constexpr int kBinWarps = kBinThreads / 32;
  constexpr int kZeroRowsPerBlock = kBinThreads * 4;
  if (*reinterpret_cast<volatile const int *>(&a.ctl->loop.done)) return;
  const int it = *reinterpret_cast<volatile const int *>(&a.ctl->loop.loops);
  extern __shared__ __align__(16) float sm[];
  __shared__ double sred[kBinWarps];
  const uint64_t ps = policy_evict_first();
  const uint64_t pl = policy_evict_last();
  double err = 0.0;  // every |new - old| added in FP64 (src/pr_spmv.cc:42,53)
  const int b = blockIdx.x;
  // both phase-1 launches of this sweep are complete: their unit counters
  // start again from zero for the next sweep
  if (b == 0 && threadIdx.x == 0) a.ctl->unit_next[0] = a.ctl->unit_next[1] = 0;
  if (b < a.nbins) {
    const int4 bn = a.bin[b];
    const int row0 = bn.x, row1 = bn.y, q0 = bn.z, q1 = bn.w;
    const int np4 = (q1 - q0 + 3) >> 2;  // the block is padded to whole float4
    const float4 *src4 = reinterpret_cast<const float4 *>(a.part + a.binbase[b]);
    float4 *sm4 = reinterpret_cast<float4 *>(sm);
    for (int i = threadIdx.x; i < np4; i += kBinThreads) cp_async_16(sm4 + i, src4 + i);
    // the bin's positions idx[q0 .. q1) follow the partials in shared
    // memory, copied in 16-byte words from the one holding idx[q0]
    const int e0 = q0 & ~7;
    const int nq = (q1 - e0 + 7) >> 3;
    uint16_t *sx = reinterpret_cast<uint16_t *>(sm + ((a.bin_words + 3) & ~3));
    const float4 *idx4 = reinterpret_cast<const float4 *>(a.idx + e0);
    for (int i = threadIdx.x; i < nq; i += kBinThreads)
      cp_async_16(reinterpret_cast<float4 *>(sx) + i, idx4 + i);
    // the first row's own data is fetched while the copies arrive
    int u = row0 + threadIdx.x;
    int s0 = 0, s1 = 0, deg = 1;
    float old = 0.f;
    if (u < row1) {
      s0 = a.rowq[u] - e0;
      s1 = a.rowq[u + 1] - e0;
      old = ld_score(a.score + u, ps);
      deg = a.odeg ? a.odeg[u] : a.rowoff[u + 1] - a.rowoff[u];
    }
    cp_async_wait_all();
    __syncthreads();
    const unsigned smb = smem_addr(sm);
    const unsigned sxb = smem_addr(sx);
    while (u < row1) {
      float sum = 0.f;
      int j = s0;
      for (; j + 3 < s1; j += 4) {
        const unsigned i0 = lds_u16(sxb, j), i1 = lds_u16(sxb, j + 1);
        const unsigned i2 = lds_u16(sxb, j + 2), i3 = lds_u16(sxb, j + 3);
        sum = __fadd_rn(sum, lds_f32(smb, i0));
        sum = __fadd_rn(sum, lds_f32(smb, i1));
        sum = __fadd_rn(sum, lds_f32(smb, i2));
        sum = __fadd_rn(sum, lds_f32(smb, i3));
      }
      for (; j < s1; j++) sum = __fadd_rn(sum, lds_f32(smb, lds_u16(sxb, j)));
      const int un = u + kBinThreads;
      int n0 = 0, n1 = 0, ndeg = 1;
      float nold = 0.f;
      if (un < row1) {  // the next row's data, fetched before this row is written
        n0 = a.rowq[un] - e0;
        n1 = a.rowq[un + 1] - e0;
        nold = ld_score(a.score + un, ps);
        ndeg = a.odeg ? a.odeg[un] : a.rowoff[un + 1] - a.rowoff[un];
      }
      const float base = a.kind == kKindPPR ? a.base_vec[u] : a.base_scalar;
      // the reference's update: base + d * sum, two roundings (src/pr_spmv.cc:51)
      const float nw = __fadd_rn(base, __fmul_rn(a.damping, sum));
      st_hint_f32(a.score + u, nw, ps);
      st_hint_f32(a.contrib + u, __fdiv_rn(nw, __int2float_rn(deg)), pl);
      err += static_cast<double>(fabsf(__fsub_rn(nw, old)));
      u = un;
      s0 = n0;
      s1 = n1;
      old = nold;
      deg = ndeg;
    }
  } else if (it == 0) {
    // rows without in-neighbours: new = base from the first sweep on
    const int lo = a.ndst + (b - a.nbins) * kZeroRowsPerBlock;
    const int hi = min(a.n, lo + kZeroRowsPerBlock);
    for (int u = lo + threadIdx.x; u < hi; u += kBinThreads) {
      const float base = a.kind == kKindPPR ? a.base_vec[u] : a.base_scalar;
      const float nw = __fadd_rn(base, __fmul_rn(a.damping, 0.f));
      const float old = ld_score(a.score + u, ps);
      st_hint_f32(a.score + u, nw, ps);
      // in a directed graph such a row can still have out-edges
      if (a.odeg) st_hint_f32(a.contrib + u, __fdiv_rn(nw, __int2float_rn(a.odeg[u])), pl);
      err += static_cast<double>(fabsf(__fsub_rn(nw, old)));
    }
  }
  const double block_err = block_sum_d<kBinThreads>(err, sred);
  const SweepReduce red{a.part1, a.part2, a.tick1, a.trace, a.ctl, a.nblocks, a.epsilon};
  sweep_grid_finish<kBinThreads>(red, it, block_err, sred);
}

}  // namespace

const void *SlicePartialKernel(bool flat) {
  return flat ? reinterpret_cast<const void *>(slice_partial_kernel<true>)
              : reinterpret_cast<const void *>(slice_partial_kernel<false>);
}
// Larger bins get more threads per CTA (about one per 24 words), so that
// the fewer, larger CTAs still fill the SMs (measured at Kronecker scale 25
// with 12288-word bins: 0.47 ms for 512 threads against 0.53 for 256).
int BinRowThreads(const SliceBlocks &sb) {
  return sb.bin_words >= 2 * kLargeBinWords ? 1024 : (sb.bin_words >= kLargeBinWords ? 512 : 256);
}

const void *BinRowKernel(const SliceBlocks &sb) {
  switch (BinRowThreads(sb)) {
    case 1024: return reinterpret_cast<const void *>(bin_row_kernel<1024>);
    case 512: return reinterpret_cast<const void *>(bin_row_kernel<512>);
    default: return reinterpret_cast<const void *>(bin_row_kernel<256>);
  }
}

int BinRowGrid(const SliceBlocks &sb, int64_t n) {
  const int64_t zero_rows = int64_t(4) * BinRowThreads(sb);
  return sb.nbins + static_cast<int>((n - sb.ndst + zero_rows - 1) / zero_rows);
}

// contribs + the zero slot, rounded to whole float4
size_t SliceSmemBytes(const SliceBlocks &sb) { return sizeof(float) * (sb.slice_verts + 4); }
// the bin's partials, then its positions (16-byte words from the one
// holding its first position)
size_t BinSmemBytes(const SliceBlocks &sb) {
  return sizeof(float) * ((sb.bin_words + 3) & ~3) + sizeof(uint16_t) * (sb.bin_words + 16);
}

}  // namespace prgpu
