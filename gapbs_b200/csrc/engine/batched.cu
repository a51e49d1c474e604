// batched.cu -- batched personalized PageRank: one launch per sweep updates an
// N x Bp block of scores (a tile of up to 64 teleport vectors) as a CSR x
// dense-block product,
//   S'[u, c] = (1-d) t[u, c] + d * sum_{v in in(u)} S[v, c] / S_v,
// with a per-column FP64 L1 change and per-column retirement: a column whose
// change drops below epsilon stops updating (its scores are final) while the
// others continue.
//
// Layout: the block is vertex-major (row u holds its Bp columns
// contiguously, Bp in {8, 16, 32, 64}).  A lane owns four consecutive
// columns and loads them with one 16-byte load, so L = Bp/4 lanes cover one
// neighbour row and one warp instruction gathers 32/L neighbour rows, each a
// whole number of 32-byte sectors.  Four such instructions are in flight per
// lane before their sums are formed.  The CSR is streamed once per sweep for
// all Bp columns.  A lane whose four columns have all retired issues no
// gather, so a sector is skipped once its eight columns have retired.
//
// Work split (rows renumbered by descending in-degree, as for the plain
// sweep): a persistent grid (SMs x resident blocks) first takes the hub-row
// segments block-cooperatively (the row's last segment block sums the
// segment partials in segment order), then every warp takes whole rows,
// interleaved across the grid, and finally the short rows (fewer in-entries
// than two rounds of a warp's gathers) go one row per lane group, 32/L rows
// per warp at once, so the per-row work (offsets, old score, update, stores)
// of the many short rows runs in parallel instead of one row at a time.
//
// Cache policy: contrib rows are written and gathered evict-last in L2 (the
// index and score streams are evict-first); the first l1_rows rows (the
// highest in-degree vertices, gathered most often) are gathered through L1,
// all others bypass it so they cannot evict the hubs.
//
// Occupancy: the sweep is bound by the latency of its gathers, not by L2 or
// HBM bandwidth (a 64-column sweep moves ~7 TB/s from L2, a fifth of what the
// L2-to-SM path carries), so the kernel is compiled for 8 resident blocks per
// SM (6 for weighted graphs) even though that spills a few registers to L1:
// more warps in flight beat the spill traffic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "batched.h"
#include "common.cuh"

namespace prgpu {

namespace {

constexpr int kBT = 256;       // threads per block
constexpr int kBW = kBT / 32;  // warps per block
constexpr int kUnroll = 4;     // gather instructions in flight per lane
constexpr int64_t kL1GatherBytes = 96 * 1024;  // L1 budget for hub rows per SM

struct BatchArgs {
  int32_t n;
  int32_t Bp;  // padded tile width
  const int32_t *__restrict__ rowoff;
  const int32_t *__restrict__ col;
  const float *__restrict__ win;
  const int32_t *__restrict__ odeg;
  const float *__restrict__ rsum;
  const float *__restrict__ base;
  const uint8_t *__restrict__ tflag;  // row has a nonzero base entry
  float damping;
  float *S;
  float *C0;  // contrib ping-pong: sweep k gathers C[k & 1], writes C[(k + 1) & 1]
  float *C1;
  int32_t nseg;
  int32_t hub_rows;
  int32_t zero_start;
  const int32_t *__restrict__ seg_row;
  const int32_t *__restrict__ seg_first;
  unsigned *hub_ticket;
  float *seg_partial;
  double *part1;
  double *part2;
  unsigned *tick1;
  BatchCtl *ctl;
  double *trace;
  int32_t *sweeps;
  int32_t nblocks;
  int32_t stop_at;  // stop for a repack once at most this many columns iterate
  int32_t zero_final_sweep;  // first sweep that may skip rows without in-neighbours
  int32_t l1_rows;  // rows [0, l1_rows) (the hubs) are gathered through L1; the
                    // rest bypass it so they cannot evict the hubs
  int32_t short_start;  // rows [short_start, n) go one row per lane group
  double epsilon;
};

// Tile column c -> caller column (or source column of a repack).
struct ColMap {
  int32_t c[kMaxTile];
};

template <bool W, bool DIR>
__device__ __forceinline__ float bdenom(const BatchArgs &a, int u) {
  if (W) return a.rsum[u];
  if (DIR) return __int2float_rn(a.odeg[u]);
  return __int2float_rn(a.rowoff[u + 1] - a.rowoff[u]);
}

__device__ __forceinline__ float4 f4add(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// Loads columns 4*gl .. 4*gl+3 of contrib row v (through L1 for hub rows).
// The offset is counted in float4 units in 32 bits: the host keeps
// n * L below 2^32 (MaxTileFor).
template <int L>
__device__ __forceinline__ float4 gather_row4(const BatchArgs &a, const float *Cin, int v, int gl,
                                              uint64_t pg) {
  const float4 *src = reinterpret_cast<const float4 *>(Cin) +
                      (static_cast<uint32_t>(v) * static_cast<uint32_t>(L) + static_cast<uint32_t>(gl));
  return v < a.l1_rows ? ld_gather_v4(src, pg) : ld_gather_v4_cold(src, pg);
}

// Sum over entries [s, e) of w_e * Cin[v_e, 4*gl .. 4*gl+3], where lane group
// grp = lane / L takes every (32/L)-th entry; the caller reduces across
// groups.  Indices (and weights) are loaded 32 at a time and broadcast.
template <int L, bool W>
__device__ __forceinline__ float4 row_accumulate(const BatchArgs &a, const float *Cin, int s, int e,
                                                 int lane, bool gather, uint64_t ps, uint64_t pg,
                                                 bool have_first = false, int idx_first = 0,
                                                 float w_first = 0.f) {
  constexpr int NPW = 32 / L;
  const int grp = lane / L, gl = lane % L;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int j0 = s; j0 < e; j0 += 32) {
    const int cnt = min(32, e - j0);
    int idx = 0;
    float w = 0.f;
    if (have_first && j0 == s) {
      idx = idx_first;
      w = w_first;
    } else if (lane < cnt) {
      idx = ld_stream_s32(a.col + j0 + lane, ps);
      if (W) w = ld_stream_f32(a.win + j0 + lane, ps);
    }
    for (int k = 0; k < cnt; k += NPW * kUnroll) {
      float4 x[kUnroll];
      float wk[kUnroll];
#pragma unroll
      for (int q = 0; q < kUnroll; q++) {
        const int kk = k + q * NPW + grp;
        const int v = __shfl_sync(0xffffffffu, idx, kk & 31);
        wk[q] = W ? __shfl_sync(0xffffffffu, w, kk & 31) : 1.f;
        x[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gather && kk < cnt) x[q] = gather_row4<L>(a, Cin, v, gl, pg);
      }
#pragma unroll
      for (int q = 0; q < kUnroll; q++) {
        if (W) {
          acc.x = __fmaf_rn(wk[q], x[q].x, acc.x);
          acc.y = __fmaf_rn(wk[q], x[q].y, acc.y);
          acc.z = __fmaf_rn(wk[q], x[q].z, acc.z);
          acc.w = __fmaf_rn(wk[q], x[q].w, acc.w);
        } else {
          acc = f4add(acc, x[q]);
        }
      }
    }
  }
  // combine the lane groups (fixed xor order: deterministic)
#pragma unroll
  for (int o = L; o < 32; o <<= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
    acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
    acc.w += __shfl_xor_sync(0xffffffffu, acc.w, o);
  }
  return acc;
}

// Short rows: lane group grp = lane / L owns one row (entries [s, s + len),
// len may differ between groups) and sums w_e * Cin[v_e, 4*gl .. 4*gl+3]
// over it, kUnroll gathers in flight per group.  Each lane loads CH / L of
// every CH consecutive indices of its group's row; the loop runs to the
// longest row of the warp (warp-uniform trip count, shuffles stay converged).
template <int L, bool W>
__device__ __forceinline__ float4 group_accumulate(const BatchArgs &a, const float *Cin, int s,
                                                   int len, int lane, bool gather, uint64_t ps,
                                                   uint64_t pg) {
  constexpr int CH = L > kUnroll ? L : kUnroll;
  constexpr int R = CH / L;
  const int grp = lane / L, gl = lane % L;
  int maxlen = len;
#pragma unroll
  for (int o = L; o < 32; o <<= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int j0 = 0; j0 < maxlen; j0 += CH) {
    int idx[R];
    float w[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int j = j0 + r * L + gl;
      idx[r] = 0;
      w[r] = 0.f;
      if (j < len) {
        idx[r] = ld_stream_s32(a.col + s + j, ps);
        if (W) w[r] = ld_stream_f32(a.win + s + j, ps);
      }
    }
#pragma unroll
    for (int k = 0; k < CH; k += kUnroll) {
      if (j0 + k < maxlen) {  // warp-uniform
        float4 x[kUnroll];
        float wk[kUnroll];
#pragma unroll
        for (int q = 0; q < kUnroll; q++) {
          const int kk = k + q;
          const int srcl = grp * L + (kk % L);
          const int v = __shfl_sync(0xffffffffu, idx[kk / L], srcl);
          wk[q] = W ? __shfl_sync(0xffffffffu, w[kk / L], srcl) : 1.f;
          x[q] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (gather && j0 + kk < len) x[q] = gather_row4<L>(a, Cin, v, gl, pg);
        }
#pragma unroll
        for (int q = 0; q < kUnroll; q++) {
          if (W) {
            acc.x = __fmaf_rn(wk[q], x[q].x, acc.x);
            acc.y = __fmaf_rn(wk[q], x[q].y, acc.y);
            acc.z = __fmaf_rn(wk[q], x[q].z, acc.z);
            acc.w = __fmaf_rn(wk[q], x[q].w, acc.w);
          } else {
            acc = f4add(acc, x[q]);
          }
        }
      }
    }
  }
  return acc;
}

__device__ __forceinline__ float comp(const float4 &v, int c) {
  return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}

// Updates the four columns 4*gl.. of row u from their sums (active columns
// only); adds |new - old| per column to err[].
template <bool W, bool DIR>
__device__ __forceinline__ void finish4(const BatchArgs &a, float *Cout, int u, int gl,
                                        unsigned active4, float4 sum, float4 old, float4 bs,
                                        float den, double *err, uint64_t ps, uint64_t pl) {
  const int64_t i = static_cast<int64_t>(u) * a.Bp + 4 * gl;
  float nw[4], cv[4];
  // one division per row; contrib = new * (1 / S_v) is within an ulp of new / S_v
  const float inv = __frcp_rn(den);
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const float o = comp(old, c);
    const bool act = (active4 >> c) & 1u;
    nw[c] = act ? __fadd_rn(comp(bs, c), __fmul_rn(a.damping, comp(sum, c))) : o;
    cv[c] = __fmul_rn(nw[c], inv);
    if (act) err[c * kBT] += static_cast<double>(fabsf(__fsub_rn(nw[c], o)));
  }
  st_hint_v4(reinterpret_cast<float4 *>(a.S + i), make_float4(nw[0], nw[1], nw[2], nw[3]), ps);
  st_hint_v4(reinterpret_cast<float4 *>(Cout + i), make_float4(cv[0], cv[1], cv[2], cv[3]), pl);
}

template <int L, bool W, bool DIR>
__global__ void __launch_bounds__(kBT, W ? 6 : 8) batch_sweep_kernel(const BatchArgs a) {
  if (*reinterpret_cast<volatile const int *>(&a.ctl->loop.done)) return;
  const int it = *reinterpret_cast<volatile const int *>(&a.ctl->loop.loops);
  const float *Cin = (it & 1) ? a.C1 : a.C0;
  float *Cout = (it & 1) ? a.C0 : a.C1;
  __shared__ double serr[kBW][kMaxTile];
  __shared__ double scol[kMaxTile];
  __shared__ float sacc[kBW][kMaxTile];
  __shared__ int s_last;
  const uint64_t ps = policy_evict_first();
  const uint64_t pg = policy_evict_last();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int gl = lane % L;
  const int Bp = a.Bp;
  const unsigned long long active =
      *reinterpret_cast<volatile const unsigned long long *>(&a.ctl->active);
  const unsigned active4 = static_cast<unsigned>((active >> (4 * gl)) & 0xFull);
  const bool gather = active4 != 0u;
  // per-thread FP64 error of its four columns, in shared memory (column c of
  // thread t at s_err[c][t]) to keep registers for gathers in flight
  __shared__ double s_err[4][kBT];
  double *err = &s_err[0][threadIdx.x];
#pragma unroll
  for (int c = 0; c < 4; c++) err[c * kBT] = 0.0;
  if (threadIdx.x < kMaxTile) scol[threadIdx.x] = 0;

  // ---- hub segments, block-cooperative
  for (int seg = blockIdx.x; seg < a.nseg; seg += gridDim.x) {
    const int u = a.seg_row[seg];
    const int first = a.seg_first[u];
    const int nseg = a.seg_first[u + 1] - first;
    const int rs = a.rowoff[u], re = a.rowoff[u + 1];
    const int s = rs + (seg - first) * kSegEntries;
    const int e = min(re, s + kSegEntries);
    const int per = (e - s + kBW - 1) / kBW;
    const int ws = min(e, s + wid * per), we = min(e, ws + per);
    const float4 acc = row_accumulate<L, W>(a, Cin, ws, we, lane, gather, ps, pg);
    if (lane < L) {
      sacc[wid][4 * gl + 0] = acc.x;
      sacc[wid][4 * gl + 1] = acc.y;
      sacc[wid][4 * gl + 2] = acc.z;
      sacc[wid][4 * gl + 3] = acc.w;
    }
    __syncthreads();
    if (threadIdx.x < Bp) {
      float p = 0.f;
      for (int w = 0; w < kBW; w++) p += sacc[w][threadIdx.x];
      a.seg_partial[static_cast<int64_t>(seg) * Bp + threadIdx.x] = p;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned t = atomicAdd(a.hub_ticket + u, 1u);
      s_last = (t == static_cast<unsigned>(nseg - 1));
    }
    __syncthreads();
    if (s_last) {
      // the row's last segment block finishes the row: thread c owns column c
      __threadfence();
      const int c = threadIdx.x;
      if (c < Bp && ((active >> c) & 1ull)) {
        float sum = 0.f;
        for (int k = 0; k < nseg; k++)
          sum = __fadd_rn(sum, __ldcg(a.seg_partial + static_cast<int64_t>(first + k) * Bp + c));
        const int64_t i = static_cast<int64_t>(u) * Bp + c;
        const float old = ld_score(a.S + i, ps);
        const float b0 = a.tflag[u] ? a.base[i] : 0.f;
        const float nw = __fadd_rn(b0, __fmul_rn(a.damping, sum));
        st_hint_f32(a.S + i, nw, ps);
        st_hint_f32(Cout + i, __fdiv_rn(nw, bdenom<W, DIR>(a, u)), pg);
        scol[c] += static_cast<double>(fabsf(__fsub_rn(nw, old)));
      }
      if (threadIdx.x == 0) a.hub_ticket[u] = 0;
    }
    __syncthreads();
  }

  // ---- every other row: one warp per row, interleaved across the grid
  const int gw = blockIdx.x * kBW + wid;
  const int nw = gridDim.x * kBW;
  // Rows without in-neighbours hold new = base from the first sweep on; their
  // contrib is final once both ping-pong buffers hold it (after the second
  // sweep; an undirected graph never gathers it at all).  Later sweeps skip
  // them: their scores cannot change and their L1 change is exactly zero.
  const int row_end = (it >= a.zero_final_sweep) ? a.zero_start : a.n;
  const int warp_end = min(max(a.short_start, a.hub_rows), row_end);
  for (int u = a.hub_rows + gw; u < warp_end; u += nw) {
    float4 old = make_float4(0.f, 0.f, 0.f, 0.f), bs = old;
    const int64_t i = static_cast<int64_t>(u) * Bp + 4 * gl;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (u < a.zero_start)
      acc = row_accumulate<L, W>(a, Cin, a.rowoff[u], a.rowoff[u + 1], lane, gather, ps, pg);
    if (lane < L && gather) {
      old = ld_score_v4(reinterpret_cast<const float4 *>(a.S + i), ps);
      if (__ldg(a.tflag + u)) bs = ld_stream_v4f(reinterpret_cast<const float4 *>(a.base + i), ps);
      finish4<W, DIR>(a, Cout, u, gl, active4, acc, old, bs, bdenom<W, DIR>(a, u), err, ps,
                      pg);
    }
  }
  {
    constexpr int NPW = 32 / L;
    const int grp = lane / L;
    const int sbeg = max(warp_end, a.hub_rows);
    for (int u0 = sbeg + gw * NPW; u0 < row_end; u0 += nw * NPW) {
      const int u = u0 + grp;
      const bool valid = u < row_end;
      int s = 0, len = 0;
      if (valid && u < a.zero_start) {
        s = a.rowoff[u];
        len = a.rowoff[u + 1] - s;
      }
      float4 old = make_float4(0.f, 0.f, 0.f, 0.f), bs = old;
      const int64_t i = static_cast<int64_t>(u) * Bp + 4 * gl;
      const float4 acc = group_accumulate<L, W>(a, Cin, s, len, lane, gather, ps, pg);
      if (valid && gather) {
        old = ld_score_v4(reinterpret_cast<const float4 *>(a.S + i), ps);
        if (__ldg(a.tflag + u)) bs = ld_stream_v4f(reinterpret_cast<const float4 *>(a.base + i), ps);
        finish4<W, DIR>(a, Cout, u, gl, active4, acc, old, bs, bdenom<W, DIR>(a, u), err, ps,
                        pg);
      }
    }
  }
  // lane groups hold partial errors of the same columns: combine them
  double errc[4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    errc[c] = err[c * kBT];
#pragma unroll
    for (int o = L; o < 32; o <<= 1) errc[c] += __shfl_xor_sync(0xffffffffu, errc[c], o);
  }

  // ---- per-column block partial, then two-stage grid reduction per column
  if (lane < L) {
#pragma unroll
    for (int c = 0; c < 4; c++) serr[wid][4 * gl + c] = errc[c];
  }
  __syncthreads();
  const int b = blockIdx.x;
  if (threadIdx.x < Bp) {
    double p = scol[threadIdx.x];
    for (int w = 0; w < kBW; w++) p += serr[w][threadIdx.x];
    a.part1[static_cast<int64_t>(b) * Bp + threadIdx.x] = p;
  }
  __threadfence();
  __syncthreads();
  const int g = b / kReduceGroup;
  const int gsize = min(kReduceGroup, a.nblocks - g * kReduceGroup);
  const int ngroups = (a.nblocks + kReduceGroup - 1) / kReduceGroup;
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(a.tick1 + g, 1u);
    s_last = (t == static_cast<unsigned>(gsize - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x < Bp) {
    double p = 0;
    for (int i = 0; i < gsize; i++)
      p += __ldcg(a.part1 + static_cast<int64_t>(g * kReduceGroup + i) * Bp + threadIdx.x);
    a.part2[static_cast<int64_t>(g) * Bp + threadIdx.x] = p;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    a.tick1[g] = 0;
    const unsigned t2 = atomicAdd(&a.ctl->tick2, 1u);
    s_last = (t2 == static_cast<unsigned>(ngroups - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  __shared__ unsigned long long s_retire;
  if (threadIdx.x == 0) s_retire = 0ull;
  __syncthreads();
  if (threadIdx.x < Bp && ((active >> threadIdx.x) & 1ull)) {
    double tot = 0;
    for (int i = 0; i < ngroups; i++)
      tot += __ldcg(a.part2 + static_cast<int64_t>(i) * Bp + threadIdx.x);
    a.trace[static_cast<int64_t>(it) * Bp + threadIdx.x] = tot;
    a.sweeps[threadIdx.x] = it + 1;
    if (tot < a.epsilon) atomicOr(&s_retire, 1ull << threadIdx.x);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long next = active & ~s_retire;
    a.ctl->active = next;
    a.ctl->tick2 = 0;
    if (next == 0ull) {
      a.ctl->loop.done = 1;
    } else if (__popcll(next) <= a.stop_at) {
      // few enough survivors to repack them into a narrower tile
      a.ctl->compact = 1;
      a.ctl->loop.done = 1;
    }
    __threadfence();
  }
}

// The per-tile copy kernels below run on a grid of kCopyBlocksPerSM blocks
// per SM and stride over their cells, four independent cells in flight per
// thread: launching one short-lived thread per cell (hundreds of millions of
// them for a 64-column tile) would be bound by block launch, not by HBM.
// Cells are (row, column) with 2^lb column slots per row; the grid's thread
// count is a multiple of 2^lb, so a thread keeps one column for all its
// cells and reads its entry of the column tables (kernel parameters) once:
// 32 different parameter-array entries per warp instruction would be
// serialised by the constant cache on every cell.
constexpr int kCopyBlocksPerSM = 8;
constexpr int kCopyThreads = 256;

// Copies the surviving columns map.c[j] (j < nact) of a width-Bo tile into
// columns j of a width-2^lbn tile (padding columns zero); base is copied on
// flagged rows only.
__global__ void __launch_bounds__(kCopyThreads)
    batch_repack_kernel(int32_t n, int Bo, int lbn, int nact, ColMap map,
                        const uint8_t *__restrict__ tflag, const float *__restrict__ So,
                        const float *__restrict__ bo, const float *__restrict__ Co,
                        float *__restrict__ Sn, float *__restrict__ bn, float *__restrict__ Cn) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int j = static_cast<int>(t & ((1 << lbn) - 1));
  const int64_t ustride = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> lbn;
  const bool real = j < nact;
  const int sc = real ? map.c[j] : 0;
  for (int64_t u0 = t >> lbn; u0 < n; u0 += 4 * ustride) {
    float sv[4], cv[4], bv[4];
    bool fl[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int64_t u = u0 + r * ustride;
      sv[r] = cv[r] = bv[r] = 0.f;
      fl[r] = false;
      if (u < n) {
        fl[r] = tflag[u] != 0;
        if (real) {
          const int64_t src = u * Bo + sc;
          sv[r] = So[src];
          cv[r] = Co[src];
          if (fl[r]) bv[r] = bo[src];
        }
      }
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int64_t u = u0 + r * ustride;
      if (u < n) {
        const int64_t i = (u << lbn) + j;
        Sn[i] = sv[r];
        Cn[i] = cv[r];
        if (fl[r]) bn[i] = bv[r];
      }
    }
  }
}

// Tile init, one thread per four columns of a row: S = t, C = t / S_v,
// base = (1-d) t (written only on rows with a nonzero teleport entry, which
// tflag marks); padding columns are zero.  Cell i is row u = i >> lq,
// columns 4 * (i & (Bp/4 - 1)) ..; a row's cells are consecutive lanes of
// one warp (Bp/4 <= 16), and whole warps stride together so the row-wide
// ballot always has all 32 lanes.
template <bool W, bool DIR>
__global__ void __launch_bounds__(kCopyThreads)
    batch_init_kernel(int32_t n, int B, int lq, int K, int c0, const int32_t *__restrict__ perm,
                      const int32_t *__restrict__ rowoff, const int32_t *__restrict__ odeg,
                      const float *__restrict__ rsum, const float *__restrict__ tele_old,
                      float uniform, float one_minus_d, float *__restrict__ S,
                      float *__restrict__ C, float *__restrict__ base, uint8_t *__restrict__ tflag) {
  const int64_t total = static_cast<int64_t>(n) << lq;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int lane = threadIdx.x & 31;
  const int w = 1 << lq;
  const unsigned grp_mask = (w >= 32 ? 0xffffffffu : ((1u << w) - 1u)) << (lane & ~(w - 1));
  for (int64_t wb = static_cast<int64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31);
       wb < total; wb += stride) {
    const int64_t i = wb + lane;
    const int64_t u = i >> lq;
    const bool live = i < total;
    const int q = static_cast<int>(i & (w - 1));
    float t[4] = {0.f, 0.f, 0.f, 0.f};
    bool nz = false;
    float denom = 1.f;
    if (live) {
      const int64_t row = tele_old ? static_cast<int64_t>(perm[u]) * K + c0 : 0;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int col = 4 * q + c;
        if (col < B) t[c] = tele_old ? tele_old[row + col] : uniform;
        nz |= t[c] != 0.f;
      }
      if (W) denom = rsum[u];
      else if (DIR) denom = __int2float_rn(odeg[u]);
      else denom = __int2float_rn(rowoff[u + 1] - rowoff[u]);
    }
    // any nonzero teleport entry in the row: OR over the row's w lanes
    const bool row_nz = (__ballot_sync(0xffffffffu, nz) & grp_mask) != 0u;
    if (live) {
      const int64_t o = 4 * i;  // = u * Bp + 4 * q
      *reinterpret_cast<float4 *>(S + o) = make_float4(t[0], t[1], t[2], t[3]);
      *reinterpret_cast<float4 *>(C + o) =
          make_float4(__fdiv_rn(t[0], denom), __fdiv_rn(t[1], denom), __fdiv_rn(t[2], denom),
                      __fdiv_rn(t[3], denom));
      if (row_nz)
        *reinterpret_cast<float4 *>(base + o) =
            make_float4(__fmul_rn(one_minus_d, t[0]), __fmul_rn(one_minus_d, t[1]),
                        __fmul_rn(one_minus_d, t[2]), __fmul_rn(one_minus_d, t[3]));
      if (q == 0) tflag[u] = row_nz ? 1 : 0;
    }
  }
}

// Where each tile column's final scores are: block `phase[c]` of the score
// arena (width W[phase]), column j[c].
struct OutSrc {
  const float *S[4];
  int32_t W[4];
  int32_t j[kMaxTile];
  int8_t phase[kMaxTile];
};

// The tile's write-back: caller column c0 + c of original vertex perm[u]
// takes tile column c of renumbered row u.  Rows are read in order and every
// output row is written as one contiguous run of B floats.
__global__ void __launch_bounds__(kCopyThreads)
    batch_out_kernel(int32_t n, int B, int lb, int K, int c0, const int32_t *__restrict__ perm,
                     OutSrc src, float *__restrict__ out_old) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int c = static_cast<int>(t & ((1 << lb) - 1));
  if (c >= B) return;  // whole-thread exit: no collective below
  const int64_t ustride = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> lb;
  const int p = src.phase[c];
  const float *__restrict__ Sp = src.S[p];
  const int64_t Wp = src.W[p];
  const int jc = src.j[c];
  for (int64_t u0 = t >> lb; u0 < n; u0 += 4 * ustride) {
    float x[4];
    int64_t o[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int64_t u = u0 + r * ustride;
      o[r] = -1;
      if (u < n) {
        x[r] = Sp[u * Wp + jc];
        o[r] = static_cast<int64_t>(perm[u]) * K + c0 + c;
      }
    }
#pragma unroll
    for (int r = 0; r < 4; r++)
      if (o[r] >= 0) out_old[o[r]] = x[r];
  }
}

// Resets the control block, tickets, sweep counts and trace of a phase.
__global__ void batch_phase_begin_kernel(BatchCtl *ctl, unsigned long long active, int loops,
                                         int done, unsigned *tick1, int ngroups, int32_t *sweeps,
                                         double *trace, int64_t trace_len) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  if (t == 0) {
    ctl->loop.done = done;
    ctl->loop.loops = loops;
    ctl->loop.halted = done;
    ctl->tick2 = 0;
    ctl->compact = 0;
    ctl->active = active;
  }
  for (int64_t k = t; k <= ngroups; k += stride) tick1[k] = 0;
  for (int64_t k = t; k < kMaxTile; k += stride) sweeps[k] = 0;
  for (int64_t k = t; k < trace_len; k += stride) trace[k] = 0.0;
}

// Blocks for a copy kernel over `cells` cells: the persistent grid, or fewer
// when the copy is small.
unsigned CopyGrid(int64_t cells) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t need = (cells + kCopyThreads - 1) / kCopyThreads;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(need, sms * kCopyBlocksPerSM)));
}

int Log2(int x) {
  int l = 0;
  while ((1 << l) < x) l++;
  return l;
}

template <typename T>
cudaError_t GrowB(T **p, int64_t *cap, int64_t need) {
  if (*p && *cap >= need) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<int64_t>(need, 1));
  if (e == cudaSuccess) *cap = need;
  return e;
}

// Widest tile whose contrib block has fewer than 2^32 float4 cells (the
// gather's 32-bit offset): 64 up to 2^26 vertices, 8 for any int32 graph.
int MaxTileFor(int64_t n) {
  for (int i = 3; i > 0; i--)
    if (n * (kTileWidths[i] / 4) <= int64_t(0xffffffffLL)) return kTileWidths[i];
  return kTileWidths[0];
}

BatchSchedule DefaultSchedule(int Bp) {
  BatchSchedule d;
  d.short_len = std::max(kShortLens[0], std::min(kShortLens[4], 1024 / Bp));
  d.l1_kb = static_cast<int>(kL1GatherBytes / 1024);
  return d;
}

int PadWidth(int b) {
  for (int w : kTileWidths)
    if (b <= w) return w;
  return kMaxTile;
}

template <int L>
const void *SweepFor(const DeviceGraph &g) {
  if (g.weighted) return reinterpret_cast<const void *>(batch_sweep_kernel<L, true, false>);
  if (g.directed) return reinterpret_cast<const void *>(batch_sweep_kernel<L, false, true>);
  return reinterpret_cast<const void *>(batch_sweep_kernel<L, false, false>);
}

const void *BatchSweepKernel(const DeviceGraph &g, int Bp) {
  switch (Bp) {
    case 8: return SweepFor<2>(g);
    case 16: return SweepFor<4>(g);
    case 32: return SweepFor<8>(g);
    default: return SweepFor<16>(g);
  }
}

int GridFor(const void *fn) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBT, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return sms * per_sm;
}

#define PB_TRY(expr)                                                   \
  do {                                                                 \
    cudaError_t e_ = (expr);                                           \
    if (e_ != cudaSuccess) {                                           \
      *err = std::string(#expr) + ": " + cudaGetErrorString(e_);       \
      return e_;                                                       \
    }                                                                  \
  } while (0)

// Pinned read-back area: control block, per-column sweeps, trace.
constexpr int64_t kHostSweepsOff = 64;
constexpr int64_t kHostTraceOff = kHostSweepsOff + sizeof(int32_t) * kMaxTile;
static_assert(sizeof(BatchCtl) <= kHostSweepsOff, "control block fits its slot");
int64_t HostBytes(int iters) {
  return kHostTraceOff + sizeof(double) * static_cast<int64_t>(std::max(iters, 1)) * kMaxTile;
}

// Buffers for tiles up to kMaxTile columns and a grid of up to nblocks.
cudaError_t EnsureBatchBuffers(const DeviceGraph &g, BatchScratch &bs, int nblocks, int iters,
                               std::string *err) {
  const int64_t n = g.n;
  const int64_t cells = n * kMaxTile;
  if (!bs.S || bs.cap_cells < cells) {
    int64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (float **p : {&bs.S, &bs.C[0], &bs.C[1], &bs.base, &bs.base2}) {
      if (*p) cudaFree(*p);
      *p = nullptr;
    }
    bs.cap_cells = bs.cap_cells2 = 0;
    PB_TRY(GrowB(&bs.S, &c0, 2 * cells));
    PB_TRY(GrowB(&bs.C[0], &c1, cells));
    PB_TRY(GrowB(&bs.C[1], &c2, cells));
    PB_TRY(GrowB(&bs.base, &c3, cells));
    bs.cap_cells = cells;
  }
  const int ngroups = (nblocks + kReduceGroup - 1) / kReduceGroup;
  PB_TRY(GrowB(&bs.part1, &bs.cap_part, static_cast<int64_t>(nblocks) * kMaxTile));
  if (!bs.part2 || bs.cap_groups < ngroups + 1) {
    int64_t c = 0;
    if (bs.part2) cudaFree(bs.part2), bs.part2 = nullptr;
    if (bs.tick1) cudaFree(bs.tick1), bs.tick1 = nullptr;
    PB_TRY(GrowB(&bs.part2, &c, static_cast<int64_t>(ngroups + 1) * kMaxTile));
    c = 0;
    PB_TRY(GrowB(&bs.tick1, &c, ngroups + 1));
    bs.cap_groups = ngroups + 1;
  }
  PB_TRY(GrowB(&bs.trace, &bs.cap_trace, static_cast<int64_t>(std::max(iters, 1)) * kMaxTile));
  if (!bs.sweeps) PB_TRY(cudaMalloc(&bs.sweeps, sizeof(int32_t) * kMaxTile));
  PB_TRY(GrowB(&bs.seg_partial, &bs.cap_seg, std::max<int64_t>(g.num_segments, 1) * kMaxTile));
  PB_TRY(GrowB(&bs.tflag, &bs.cap_flag, n));
  if (!bs.ctl) PB_TRY(cudaMalloc(&bs.ctl, sizeof(BatchCtl)));
  const int64_t host_need = HostBytes(iters);
  if (!bs.host || bs.cap_host < host_need) {
    if (bs.host) cudaFreeHost(bs.host);
    bs.host = nullptr;
    bs.cap_host = 0;
    PB_TRY(cudaMallocHost(reinterpret_cast<void **>(&bs.host), host_need));
    bs.cap_host = host_need;
  }
  for (cudaEvent_t &e : bs.ev)
    if (!e) PB_TRY(cudaEventCreate(&e));
  return cudaSuccess;
}

int WidthIndex(int Bp) { return Bp == 8 ? 0 : Bp == 16 ? 1 : Bp == 32 ? 2 : 3; }

// One tile: columns [c0, c0 + B) of the caller's N x K teleport block.
// The tile iterates in phases: whenever the columns still iterating fit in
// half the tile width, the loop stops, the survivors are repacked into the
// narrowest tile that holds them, and sweeping resumes there (retired
// columns' scores are written out at the end of the phase they retired in).
cudaError_t SolveTile(const DeviceGraph &g, BatchScratch &bs, cudaStream_t s, int max_iters,
                      double epsilon, float damping, int K, int c0, int B, int Bp,
                      const BatchSchedule &sched, const float *tele_old, float *out_old,
                      int32_t *sweeps_tile, double *trace_tile, float *sweep_ms,
                      int64_t *launches, std::string *err) {
  const int64_t n = g.n;
  const void *fn0 = BatchSweepKernel(g, Bp);
  const int nblocks0 = GridFor(fn0);
  PB_TRY(EnsureBatchBuffers(g, bs, nblocks0, max_iters, err));
  const int lq = Log2(Bp / 4);
  const unsigned ib = CopyGrid(n << lq);
  const float uniform = 1.0f / static_cast<float>(n);
  const float omd = 1.0f - damping;
  if (g.weighted)
    batch_init_kernel<true, false><<<ib, kCopyThreads, 0, s>>>(static_cast<int32_t>(n), B, lq, K, c0, g.perm, g.rowoff, g.odeg, g.rsum, tele_old, uniform, omd, bs.S, bs.C[0], bs.base, bs.tflag);
  else if (g.directed)
    batch_init_kernel<false, true><<<ib, kCopyThreads, 0, s>>>(static_cast<int32_t>(n), B, lq, K, c0, g.perm, g.rowoff, g.odeg, g.rsum, tele_old, uniform, omd, bs.S, bs.C[0], bs.base, bs.tflag);
  else
    batch_init_kernel<false, false><<<ib, kCopyThreads, 0, s>>>(static_cast<int32_t>(n), B, lq, K, c0, g.perm, g.rowoff, g.odeg, g.rsum, tele_old, uniform, omd, bs.S, bs.C[0], bs.base, bs.tflag);
  PB_TRY(cudaGetLastError());
  *launches += 1;

  // tile column -> caller column
  ColMap map;
  for (int j = 0; j < kMaxTile; j++) map.c[j] = j < B ? c0 + j : 0;
  int nact = B;                 // columns of the current tile (all iterate at phase start)
  float *S = bs.S, *base = bs.base;
  int64_t s_off = 0;            // this phase's score block within the arena
  OutSrc osrc;
  std::memset(&osrc, 0, sizeof(osrc));
  int phase = 0;
  float *Cpair[2] = {bs.C[0], bs.C[1]};  // Cpair[k & 1] is gathered by sweep k
  int loops = 0;
  for (int j = 0; j < B; j++) sweeps_tile[j] = 0;
  BatchCtl ctl;
  const int32_t *sw = reinterpret_cast<const int32_t *>(bs.host + kHostSweepsOff);
  const double *tr = reinterpret_cast<const double *>(bs.host + kHostTraceOff);
  *sweep_ms = 0;
  cudaEvent_t e0 = bs.ev[0], e1 = bs.ev[1];
  int tile_bp = Bp;
  while (true) {
    const void *fn = BatchSweepKernel(g, tile_bp);
    const int nblocks = GridFor(fn);
    PB_TRY(EnsureBatchBuffers(g, bs, nblocks, max_iters, err));
    const int ngroups = (nblocks + kReduceGroup - 1) / kReduceGroup;
    const unsigned long long active0 = (nact == 64) ? ~0ull : ((1ull << nact) - 1ull);
    batch_phase_begin_kernel<<<8, 256, 0, s>>>(bs.ctl, active0, loops, loops >= max_iters ? 1 : 0,
                                               bs.tick1, ngroups, bs.sweeps, bs.trace,
                                               static_cast<int64_t>(max_iters) * kMaxTile);
    PB_TRY(cudaGetLastError());
    *launches += 1;
    BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = static_cast<int32_t>(n);
    a.Bp = tile_bp;
    a.rowoff = g.rowoff;
    a.col = g.col;
    a.win = g.weighted ? g.win : nullptr;
    a.odeg = g.odeg;
    a.rsum = g.rsum;
    a.base = base;
    a.tflag = bs.tflag;
    a.damping = damping;
    a.S = S;
    a.C0 = Cpair[0];
    a.C1 = Cpair[1];
    a.nseg = static_cast<int32_t>(g.num_segments);
    a.hub_rows = static_cast<int32_t>(g.num_hub_rows);
    a.zero_start = static_cast<int32_t>(g.bin_row_start[kBinZero]);
    a.seg_row = g.seg_row;
    a.seg_first = g.seg_first;
    a.hub_ticket = g.hub_ticket;
    a.seg_partial = bs.seg_partial;
    a.part1 = bs.part1;
    a.part2 = bs.part2;
    a.tick1 = bs.tick1;
    a.ctl = bs.ctl;
    a.trace = bs.trace;
    a.sweeps = bs.sweeps;
    a.nblocks = nblocks;
    a.stop_at = tile_bp > 8 ? tile_bp / 2 : 0;
    // Directed graphs gather the contribs of rows without in-neighbours, so
    // both ping-pong buffers must hold them in this phase's layout: those rows
    // are processed in the phase's first two sweeps.  Undirected graphs never
    // gather them (no in-neighbour means no out-neighbour).
    a.zero_final_sweep = g.directed ? loops + 2 : 1;
    // the schedule of this phase's width (a repack narrows the tile)
    const BatchSchedule ph = tile_bp == Bp ? sched : ResolveSchedule(bs, tile_bp);
    a.l1_rows = static_cast<int32_t>(
        std::min<int64_t>(n, int64_t(1024) * ph.l1_kb / (4 * tile_bp)));
    // rows shorter than ph.short_len go one per lane group: the degree bin
    // whose lower bound is short_len starts there
    {
      int b = 1;
      while (b < kBinZero && g.bins.min_len[b - 1] > ph.short_len) b++;
      a.short_start = static_cast<int32_t>(g.bin_row_start[b]);
    }
    a.epsilon = epsilon;
    PB_TRY(cudaEventRecord(e0, s));
    PB_TRY(bs.loop[WidthIndex(tile_bp)].Launch(fn, dim3(nblocks), dim3(kBT), &a, sizeof(a),
                                               &bs.ctl->loop, max_iters, s));
    PB_TRY(cudaEventRecord(e1, s));
    PB_TRY(cudaMemcpyAsync(bs.host, bs.ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
    PB_TRY(cudaMemcpyAsync(bs.host + kHostSweepsOff, bs.sweeps, sizeof(int32_t) * nact,
                           cudaMemcpyDeviceToHost, s));
    if (max_iters && trace_tile)
      PB_TRY(cudaMemcpyAsync(bs.host + kHostTraceOff, bs.trace,
                             sizeof(double) * static_cast<int64_t>(max_iters) * tile_bp,
                             cudaMemcpyDeviceToHost, s));
    PB_TRY(cudaStreamSynchronize(s));
    std::memcpy(&ctl, bs.host, sizeof(ctl));
    // every column of this phase has its latest scores in this phase's block
    osrc.S[phase] = S;
    osrc.W[phase] = tile_bp;
    for (int j = 0; j < nact; j++) {
      const int lc = map.c[j] - c0;
      osrc.phase[lc] = static_cast<int8_t>(phase);
      osrc.j[lc] = j;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    *sweep_ms += ms;
    const int phase_loops = ctl.loop.loops;  // sweeps issued so far (all phases)
    *launches += 2 * static_cast<int64_t>(phase_loops - loops);
    for (int j = 0; j < nact; j++) {
      const int lc = map.c[j] - c0;       // column within the tile
      if (sw[j] > 0) sweeps_tile[lc] = sw[j];
      if (trace_tile)
        for (int it = loops; it < std::min(phase_loops, max_iters); it++)
          trace_tile[static_cast<int64_t>(it) * kMaxTile + lc] = tr[static_cast<int64_t>(it) * tile_bp + j];
    }
    loops = phase_loops;
    if (!ctl.compact || loops >= max_iters) break;
    // repack the survivors into the narrowest tile that holds them
    ColMap src, next_map;
    int m2 = 0;
    for (int j = 0; j < nact; j++)
      if ((ctl.active >> j) & 1ull) {
        src.c[m2] = j;
        next_map.c[m2] = map.c[j];
        m2++;
      }
    for (int j = m2; j < kMaxTile; j++) src.c[j] = next_map.c[j] = 0;
    const int bn = PadWidth(m2);
    if (!bs.base2 || bs.cap_cells2 < n * kMaxTile) {
      if (bs.base2) cudaFree(bs.base2);
      bs.base2 = nullptr;
      int64_t c2b = 0;
      PB_TRY(GrowB(&bs.base2, &c2b, n * kMaxTile));
      bs.cap_cells2 = n * kMaxTile;
    }
    const int64_t s_off_new = s_off + n * tile_bp;
    if (s_off_new + n * bn > 2 * n * kMaxTile || phase + 1 >= 4) {
      *err = "batched solve: phase blocks exceed the score arena";
      return cudaErrorInvalidValue;
    }
    float *S_new = bs.S + s_off_new;
    float *b_new = (base == bs.base) ? bs.base2 : bs.base;
    float *C_cur = Cpair[loops & 1];
    float *C_new = Cpair[(loops + 1) & 1];  // free: holds contribs two sweeps old
    batch_repack_kernel<<<CopyGrid(n * bn), kCopyThreads, 0, s>>>(
        static_cast<int32_t>(n), tile_bp, Log2(bn), m2, src, bs.tflag, S, base, C_cur, S_new,
        b_new, C_new);
    PB_TRY(cudaGetLastError());
    *launches += 1;
    S = S_new;
    s_off = s_off_new;
    phase++;
    base = b_new;
    Cpair[loops & 1] = C_new;
    Cpair[(loops + 1) & 1] = C_cur;
    map = next_map;
    nact = m2;
    tile_bp = bn;
  }
  // one write-back of all B columns, each from the block it finished in
  if (out_old) {
    const int lb = Log2(B);
    batch_out_kernel<<<CopyGrid(n << lb), kCopyThreads, 0, s>>>(static_cast<int32_t>(n), B, lb, K,
                                                                  c0, g.perm, osrc, out_old);
    PB_TRY(cudaGetLastError());
    *launches += 1;
  }
  return cudaSuccess;
}

// Autotuner: times sweeps of the first tile (one warm sweep that builds the
// loop graph, then two timed ones) at each supported width with the
// default schedule and keeps the width with the lowest time per
// column-sweep; then, at that width, tries half and twice the default
// short-row length and L1 budgets of 64 and 160 KB, one knob after the
// other, keeping a change only when it is faster.
cudaError_t TuneTile(const DeviceGraph &g, BatchScratch &bs, cudaStream_t s, float damping,
                     int ncols, const float *tele_old, std::string *err) {
  std::vector<int32_t> sw(kMaxTile);
  auto time_one = [&](int w, const BatchSchedule &sch, double *per_col_sweep) {
    const int B = std::min(w, ncols);
    float ms = 0;
    int64_t nl = 0;
    cudaError_t e = SolveTile(g, bs, s, 1, 0.0, damping, ncols, 0, B, w, sch, tele_old, nullptr,
                              sw.data(), nullptr, &ms, &nl, err);
    if (e != cudaSuccess) return e;
    e = SolveTile(g, bs, s, 2, 0.0, damping, ncols, 0, B, w, sch, tele_old, nullptr, sw.data(),
                  nullptr, &ms, &nl, err);
    if (e != cudaSuccess) return e;
    *per_col_sweep = ms / (2.0 * B);
    return cudaSuccess;
  };
  double best = 1e300;
  int best_w = kMaxTile;
  for (int w : kTileWidths) {
    if (PadWidth(std::min(w, ncols)) != w) continue;  // would waste a wider tile
    if (w > MaxTileFor(g.n)) continue;                // beyond the gather's 32-bit offsets
    double t = 0;
    cudaError_t e = time_one(w, DefaultSchedule(w), &t);
    if (e != cudaSuccess) return e;
    if (t < best) {
      best = t;
      best_w = w;
    }
  }
  BatchSchedule cur = DefaultSchedule(best_w);
  for (int k = 0; k < 2; k++) {
    const int len = k == 0 ? cur.short_len / 2 : cur.short_len * 2;
    if (len < kShortLens[0] || len > kShortLens[4]) continue;
    BatchSchedule c = cur;
    c.short_len = len;
    double t = 0;
    cudaError_t e = time_one(best_w, c, &t);
    if (e != cudaSuccess) return e;
    if (t < best) {
      best = t;
      cur = c;
    }
  }
  const BatchSchedule by_len = cur;
  for (int kb : {64, 160}) {
    BatchSchedule c = by_len;
    c.l1_kb = kb;
    double t = 0;
    cudaError_t e = time_one(best_w, c, &t);
    if (e != cudaSuccess) return e;
    if (t < best) {
      best = t;
      cur = c;
    }
  }
  bs.tuned_tile = best_w;
  bs.tuned_sched = cur;
  bs.tuned_ncols = ncols;
  bs.tuned_graph = g.rowoff;
  return cudaSuccess;
}

}  // namespace

BatchSchedule ResolveSchedule(const BatchScratch &bs, int Bp) {
  BatchSchedule r = DefaultSchedule(Bp);
  if (bs.tuned_tile == Bp && bs.tuned_sched.short_len) r = bs.tuned_sched;
  if (bs.sched.short_len) r.short_len = bs.sched.short_len;
  if (bs.sched.l1_kb) r.l1_kb = bs.sched.l1_kb;
  return r;
}

void FreeBatchScratch(BatchScratch *b) {
  for (auto &l : b->loop) l.Reset();
  float **fp[] = {&b->S, &b->C[0], &b->C[1], &b->base, &b->base2, &b->seg_partial};
  for (float **p : fp) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  double **dp[] = {&b->part1, &b->part2, &b->trace};
  for (double **p : dp) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (b->tick1) cudaFree(b->tick1);
  if (b->sweeps) cudaFree(b->sweeps);
  if (b->ctl) cudaFree(b->ctl);
  if (b->tflag) cudaFree(b->tflag);
  if (b->host) cudaFreeHost(b->host);
  for (cudaEvent_t &e : b->ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  b->tick1 = nullptr;
  b->sweeps = nullptr;
  b->ctl = nullptr;
  b->tflag = nullptr;
  b->host = nullptr;
  b->cap_flag = b->cap_host = 0;
  b->cap_cells = b->cap_cells2 = b->cap_part = b->cap_groups = b->cap_trace = b->cap_seg = 0;
  b->tuned_tile = b->tuned_ncols = 0;
  b->tuned_sched = BatchSchedule();
  b->tuned_graph = nullptr;
}

cudaError_t SolveBatched(const DeviceGraph &g, BatchScratch &bs, cudaStream_t s,
                         int max_iters, double epsilon, float damping, int ncols,
                         const float *tele_old, float *out_old, int32_t *sweeps_out,
                         double *err_trace, double *ms_sweep, double *ms_total,
                         int64_t *launches, std::string *err) {
  int tile = bs.tile;
  if (tile == 0) {
    if (bs.tuned_graph != g.rowoff || bs.tuned_ncols != ncols || bs.tuned_tile == 0) {
      cudaError_t e = TuneTile(g, bs, s, damping, ncols, tele_old, err);
      if (e != cudaSuccess) return e;
    }
    tile = bs.tuned_tile;
  }
  tile = PadWidth(std::max(1, std::min(std::min(tile, kMaxTile), MaxTileFor(g.n))));
  cudaEvent_t t0, t1;
  PB_TRY(cudaEventCreate(&t0));
  PB_TRY(cudaEventCreate(&t1));
  PB_TRY(cudaEventRecord(t0, s));
  std::vector<double> trace_tile(static_cast<size_t>(std::max(max_iters, 1)) * kMaxTile);
  std::vector<int32_t> sweeps_tile(kMaxTile);
  double sweep_total = 0;
  int64_t nl = 0;
  for (int c0 = 0; c0 < ncols; c0 += tile) {
    const int B = std::min(tile, ncols - c0);
    const int Bp = PadWidth(B);
    std::fill(trace_tile.begin(), trace_tile.end(), 0.0);
    float ms = 0;
    cudaError_t e = SolveTile(g, bs, s, max_iters, epsilon, damping, ncols, c0, B, Bp,
                              ResolveSchedule(bs, Bp), tele_old,
                              out_old, sweeps_tile.data(), trace_tile.data(), &ms, &nl, err);
    if (e != cudaSuccess) return e;
    sweep_total += ms;
    for (int c = 0; c < B; c++) {
      if (sweeps_out) sweeps_out[c0 + c] = sweeps_tile[c];
      if (err_trace)
        for (int it = 0; it < max_iters; it++)
          err_trace[static_cast<int64_t>(it) * ncols + c0 + c] =
              trace_tile[static_cast<int64_t>(it) * kMaxTile + c];
    }
  }
  PB_TRY(cudaEventRecord(t1, s));
  PB_TRY(cudaEventSynchronize(t1));
  float tot = 0;
  cudaEventElapsedTime(&tot, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  *ms_sweep = sweep_total;
  *ms_total = tot;
  *launches = nl;
  return cudaSuccess;
}

#undef PB_TRY

}  // namespace prgpu
