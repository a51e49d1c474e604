// batched.cu -- batched personalized PageRank: one launch per sweep updates an
// N x B block of scores (B <= 64 teleport vectors) as a CSR x dense-block
// product,
//   S'[u, c] = (1-d) t[u, c] + d * sum_{v in in(u)} S[v, c] / S_v,
// with a per-column FP64 L1 change and per-column retirement: a column whose
// change drops below epsilon stops updating (its scores are final) while the
// others continue.  The block is vertex-major (row u holds its B columns
// contiguously), so one gathered neighbour row is one or two 128-byte lines
// and the CSR is streamed once per sweep for all columns.
//
// Work split: hub rows (>= the hub threshold of the plain sweep) are cut into
// segments, one block per segment, combined by the row's last block in
// segment order; every other row is handled by one warp whose lanes own
// columns (lane, lane + 32), round-robin over the degree-sorted rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "batched.h"
#include "common.cuh"

namespace prgpu {

namespace {

constexpr int kBT = 256;                 // threads per block
constexpr int kBW = kBT / 32;            // warps per block
constexpr int kWarpBlocksPerSM = 8;

struct BatchArgs {
  int32_t n;
  int32_t B;
  const int32_t *__restrict__ rowoff;
  const int32_t *__restrict__ col;
  const float *__restrict__ win;
  const int32_t *__restrict__ odeg;
  const float *__restrict__ rsum;
  const float *__restrict__ base;
  float damping;
  float *S;
  float *C0;   // contrib ping-pong: sweep k gathers C[k & 1], writes C[(k + 1) & 1]
  float *C1;
  int32_t nseg;
  int32_t hub_rows;
  int32_t zero_start;
  int32_t warp_blocks;
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
  double epsilon;
};

template <bool W, bool DIR>
__device__ __forceinline__ float bdenom(const BatchArgs &a, int u) {
  if (W) return a.rsum[u];
  if (DIR) return __int2float_rn(a.odeg[u]);
  return __int2float_rn(a.rowoff[u + 1] - a.rowoff[u]);
}

// Warp accumulates sum over entries [s, e) of w_e * Cin[v_e, c] for its two
// columns; indices are loaded 32 at a time and broadcast by shuffle.
template <bool W>
__device__ __forceinline__ void warp_accumulate(const BatchArgs &a, const float *Cin, int s, int e,
                                                int lane, bool a0, bool a1, float &acc0,
                                                float &acc1, uint64_t ps, uint64_t pg) {
  const int B = a.B;
  for (int j0 = s; j0 < e; j0 += 32) {
    const int j = j0 + lane;
    int idx = 0;
    float w = 0.f;
    if (j < e) {
      idx = ld_stream_s32(a.col + j, ps);
      if (W) w = ld_stream_f32(a.win + j, ps);
    }
    const int cnt = min(32, e - j0);
    int k = 0;
    for (; k + 4 <= cnt; k += 4) {
      const int v0 = __shfl_sync(0xffffffffu, idx, k);
      const int v1 = __shfl_sync(0xffffffffu, idx, k + 1);
      const int v2 = __shfl_sync(0xffffffffu, idx, k + 2);
      const int v3 = __shfl_sync(0xffffffffu, idx, k + 3);
      float w0 = 1.f, w1 = 1.f, w2 = 1.f, w3 = 1.f;
      if (W) {
        w0 = __shfl_sync(0xffffffffu, w, k);
        w1 = __shfl_sync(0xffffffffu, w, k + 1);
        w2 = __shfl_sync(0xffffffffu, w, k + 2);
        w3 = __shfl_sync(0xffffffffu, w, k + 3);
      }
      if (a0) {
        const float x0 = ld_gather(Cin + static_cast<int64_t>(v0) * B + lane, pg);
        const float x1 = ld_gather(Cin + static_cast<int64_t>(v1) * B + lane, pg);
        const float x2 = ld_gather(Cin + static_cast<int64_t>(v2) * B + lane, pg);
        const float x3 = ld_gather(Cin + static_cast<int64_t>(v3) * B + lane, pg);
        if (W) {
          acc0 = __fmaf_rn(w0, x0, acc0); acc0 = __fmaf_rn(w1, x1, acc0);
          acc0 = __fmaf_rn(w2, x2, acc0); acc0 = __fmaf_rn(w3, x3, acc0);
        } else {
          acc0 += x0; acc0 += x1; acc0 += x2; acc0 += x3;
        }
      }
      if (a1) {
        const float x0 = ld_gather(Cin + static_cast<int64_t>(v0) * B + 32 + lane, pg);
        const float x1 = ld_gather(Cin + static_cast<int64_t>(v1) * B + 32 + lane, pg);
        const float x2 = ld_gather(Cin + static_cast<int64_t>(v2) * B + 32 + lane, pg);
        const float x3 = ld_gather(Cin + static_cast<int64_t>(v3) * B + 32 + lane, pg);
        if (W) {
          acc1 = __fmaf_rn(w0, x0, acc1); acc1 = __fmaf_rn(w1, x1, acc1);
          acc1 = __fmaf_rn(w2, x2, acc1); acc1 = __fmaf_rn(w3, x3, acc1);
        } else {
          acc1 += x0; acc1 += x1; acc1 += x2; acc1 += x3;
        }
      }
    }
    for (; k < cnt; k++) {
      const int v = __shfl_sync(0xffffffffu, idx, k);
      const float wk = W ? __shfl_sync(0xffffffffu, w, k) : 1.f;
      if (a0) {
        const float x = ld_gather(Cin + static_cast<int64_t>(v) * B + lane, pg);
        acc0 = W ? __fmaf_rn(wk, x, acc0) : acc0 + x;
      }
      if (a1) {
        const float x = ld_gather(Cin + static_cast<int64_t>(v) * B + 32 + lane, pg);
        acc1 = W ? __fmaf_rn(wk, x, acc1) : acc1 + x;
      }
    }
  }
}

// Updates column c of row u; returns |new - old|.
template <bool W, bool DIR>
__device__ __forceinline__ double bfinish(const BatchArgs &a, float *Cout, int u, int c, float sum,
                                          float denom, uint64_t ps, uint64_t pl) {
  const int64_t i = static_cast<int64_t>(u) * a.B + c;
  const float old = ld_score(a.S + i, ps);
  const float nw = __fadd_rn(a.base[i], __fmul_rn(a.damping, sum));
  st_hint_f32(a.S + i, nw, ps);
  st_hint_f32(Cout + i, __fdiv_rn(nw, denom), pl);
  return static_cast<double>(fabsf(__fsub_rn(nw, old)));
}

template <bool W, bool DIR>
__global__ void __launch_bounds__(kBT) batch_sweep_kernel(const BatchArgs a) {
  if (*reinterpret_cast<volatile const int *>(&a.ctl->loop.done)) return;
  const int it = *reinterpret_cast<volatile const int *>(&a.ctl->loop.loops);
  const float *Cin = (it & 1) ? a.C1 : a.C0;
  float *Cout = (it & 1) ? a.C0 : a.C1;
  __shared__ double serr[kBW][kMaxTile];
  __shared__ float sacc[kBW][kMaxTile];
  __shared__ int s_last;
  const uint64_t ps = policy_evict_first();
  const uint64_t pg = policy_evict_last();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned long long active = *reinterpret_cast<volatile const unsigned long long *>(&a.ctl->active);
  const bool a0 = lane < a.B && ((active >> lane) & 1ull);
  const bool a1 = lane + 32 < a.B && ((active >> (lane + 32)) & 1ull);
  double e0 = 0, e1 = 0;
  if (static_cast<int>(blockIdx.x) < a.nseg) {
    // ---- hub segment: 8 warps split the segment, combine in smem
    const int seg = blockIdx.x;
    const int u = a.seg_row[seg];
    const int first = a.seg_first[u];
    const int nseg = a.seg_first[u + 1] - first;
    const int rs = a.rowoff[u], re = a.rowoff[u + 1];
    const int s = rs + (seg - first) * kSegEntries;
    const int e = min(re, s + kSegEntries);
    const int per = (e - s + kBW - 1) / kBW;
    const int ws = min(e, s + wid * per), we = min(e, ws + per);
    float acc0 = 0.f, acc1 = 0.f;
    warp_accumulate<W>(a, Cin, ws, we, lane, a0, a1, acc0, acc1, ps, pg);
    sacc[wid][lane] = acc0;
    sacc[wid][lane + 32] = acc1;
    __syncthreads();
    if (threadIdx.x < a.B) {
      float p = 0.f;
      for (int w = 0; w < kBW; w++) p += sacc[w][threadIdx.x];
      a.seg_partial[static_cast<int64_t>(seg) * a.B + threadIdx.x] = p;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned t = atomicAdd(a.hub_ticket + u, 1u);
      s_last = (t == static_cast<unsigned>(nseg - 1));
    }
    __syncthreads();
    // The row's last segment block finishes the row: thread c owns column c.
    double dcol = 0;
    if (s_last) {
      __threadfence();
      const int c = threadIdx.x;
      if (c < a.B && ((active >> c) & 1ull)) {
        float sum = 0.f;
        for (int k = 0; k < nseg; k++)
          sum = __fadd_rn(sum, __ldcg(a.seg_partial + static_cast<int64_t>(first + k) * a.B + c));
        dcol = bfinish<W, DIR>(a, Cout, u, c, sum, bdenom<W, DIR>(a, u), ps, pg);
      }
      if (threadIdx.x == 0) a.hub_ticket[u] = 0;
    }
    for (int i = threadIdx.x; i < kBW * kMaxTile; i += kBT) (&serr[0][0])[i] = 0;
    __syncthreads();
    if (threadIdx.x < kMaxTile) serr[0][threadIdx.x] = dcol;
    __syncthreads();
  } else {
    // ---- warp per row, round-robin over the non-hub rows
    const int gw = (blockIdx.x - a.nseg) * kBW + wid;
    const int W_all = a.warp_blocks * kBW;
    for (int u = a.hub_rows + gw; u < a.n; u += W_all) {
      float acc0 = 0.f, acc1 = 0.f;
      if (u < a.zero_start)
        warp_accumulate<W>(a, Cin, a.rowoff[u], a.rowoff[u + 1], lane, a0, a1, acc0, acc1, ps, pg);
      const float den = bdenom<W, DIR>(a, u);
      if (a0) e0 += bfinish<W, DIR>(a, Cout, u, lane, acc0, den, ps, pg);
      if (a1) e1 += bfinish<W, DIR>(a, Cout, u, lane + 32, acc1, den, ps, pg);
    }
    serr[wid][lane] = e0;
    serr[wid][lane + 32] = e1;
    __syncthreads();
  }
  // ---- per-column block partial, then two-stage grid reduction per column
  const int B = a.B;
  const int b = blockIdx.x;
  if (threadIdx.x < B) {
    double p = 0;
    for (int w = 0; w < kBW; w++) p += serr[w][threadIdx.x];
    a.part1[static_cast<int64_t>(b) * B + threadIdx.x] = p;
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
  if (threadIdx.x < B) {
    double p = 0;
    for (int i = 0; i < gsize; i++)
      p += __ldcg(a.part1 + static_cast<int64_t>(g * kReduceGroup + i) * B + threadIdx.x);
    a.part2[static_cast<int64_t>(g) * B + threadIdx.x] = p;
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
  if (threadIdx.x < B && ((active >> threadIdx.x) & 1ull)) {
    double tot = 0;
    for (int i = 0; i < ngroups; i++) tot += __ldcg(a.part2 + static_cast<int64_t>(i) * B + threadIdx.x);
    a.trace[static_cast<int64_t>(it) * B + threadIdx.x] = tot;
    a.sweeps[threadIdx.x] = it + 1;
    if (tot < a.epsilon) atomicOr(&s_retire, 1ull << threadIdx.x);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long next = active & ~s_retire;
    a.ctl->active = next;
    a.ctl->tick2 = 0;
    if (next == 0ull) a.ctl->loop.done = 1;
    __threadfence();
  }
}

template <bool W, bool DIR>
__global__ void batch_init_kernel(int32_t n, int B, int K, int c0, const int32_t *__restrict__ perm,
                                  const int32_t *__restrict__ rowoff, const int32_t *__restrict__ odeg,
                                  const float *__restrict__ rsum, const float *__restrict__ tele_old,
                                  float uniform, float one_minus_d, float *S, float *C, float *base) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<int64_t>(n) * B) return;
  const int64_t u = i / B;
  const int c = static_cast<int>(i - u * B);
  const float t = tele_old ? tele_old[static_cast<int64_t>(perm[u]) * K + c0 + c] : uniform;
  float denom;
  if (W) denom = rsum[u];
  else if (DIR) denom = __int2float_rn(odeg[u]);
  else denom = __int2float_rn(rowoff[u + 1] - rowoff[u]);
  S[i] = t;
  base[i] = __fmul_rn(one_minus_d, t);
  C[i] = __fdiv_rn(t, denom);
}

__global__ void batch_out_kernel(int32_t n, int B, int K, int c0, const int32_t *__restrict__ inv,
                                 const float *__restrict__ S, float *out_old) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<int64_t>(n) * B) return;
  const int64_t v = i / B;
  const int c = static_cast<int>(i - v * B);
  out_old[v * K + c0 + c] = S[static_cast<int64_t>(inv[v]) * B + c];
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

}  // namespace

void FreeBatchScratch(BatchScratch *b) {
  b->loop.Reset();
  float **fp[] = {&b->S, &b->C[0], &b->C[1], &b->base, &b->seg_partial};
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
  b->tick1 = nullptr;
  b->sweeps = nullptr;
  b->ctl = nullptr;
  b->cap_cells = b->cap_part = b->cap_trace = b->cap_seg = 0;
}

#define PB_TRY(expr)                                                   \
  do {                                                                 \
    cudaError_t e_ = (expr);                                           \
    if (e_ != cudaSuccess) {                                           \
      *err = std::string(#expr) + ": " + cudaGetErrorString(e_);       \
      return e_;                                                       \
    }                                                                  \
  } while (0)

cudaError_t SolveBatched(const DeviceGraph &g, BatchScratch &bs, cudaStream_t s,
                         int max_iters, double epsilon, float damping, int ncols,
                         const float *tele_old, float *out_old, int32_t *sweeps_out,
                         double *err_trace, double *ms_sweep, double *ms_total,
                         int64_t *launches, std::string *err) {
  const int tile = bs.tile > 0 ? std::min(bs.tile, kMaxTile) : kMaxTile;
  const int64_t n = g.n;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int nseg = static_cast<int>(g.num_segments);
  const int warp_blocks = sms * kWarpBlocksPerSM;
  const int nblocks = nseg + warp_blocks;
  const int ngroups = (nblocks + kReduceGroup - 1) / kReduceGroup;
  const int Bmax = std::min(tile, ncols);
  PB_TRY(GrowB(&bs.S, &bs.cap_cells, n * Bmax));
  {
    int64_t c1 = 0, c2 = 0, c3 = 0;
    if (bs.C[0]) cudaFree(bs.C[0]), bs.C[0] = nullptr;
    if (bs.C[1]) cudaFree(bs.C[1]), bs.C[1] = nullptr;
    if (bs.base) cudaFree(bs.base), bs.base = nullptr;
    PB_TRY(GrowB(&bs.C[0], &c1, n * Bmax));
    PB_TRY(GrowB(&bs.C[1], &c2, n * Bmax));
    PB_TRY(GrowB(&bs.base, &c3, n * Bmax));
  }
  {
    int64_t c1 = 0, c2 = 0, c3 = 0;
    if (bs.part1) cudaFree(bs.part1), bs.part1 = nullptr;
    if (bs.part2) cudaFree(bs.part2), bs.part2 = nullptr;
    if (bs.tick1) cudaFree(bs.tick1), bs.tick1 = nullptr;
    PB_TRY(GrowB(&bs.part1, &c1, static_cast<int64_t>(nblocks) * Bmax));
    PB_TRY(GrowB(&bs.part2, &c2, static_cast<int64_t>(ngroups) * Bmax));
    PB_TRY(GrowB(&bs.tick1, &c3, ngroups + 1));
    bs.cap_part = nblocks;
  }
  PB_TRY(GrowB(&bs.trace, &bs.cap_trace, static_cast<int64_t>(std::max(max_iters, 1)) * Bmax));
  {
    int64_t c = 0;
    if (bs.sweeps) cudaFree(bs.sweeps), bs.sweeps = nullptr;
    PB_TRY(GrowB(&bs.sweeps, &c, kMaxTile));
  }
  PB_TRY(GrowB(&bs.seg_partial, &bs.cap_seg, std::max<int64_t>(nseg, 1) * Bmax));
  if (!bs.ctl) PB_TRY(cudaMalloc(&bs.ctl, sizeof(BatchCtl)));

  cudaEvent_t ev[4];
  for (auto &e : ev) PB_TRY(cudaEventCreate(&e));
  float sweep_total = 0;
  int64_t nl = 0;
  PB_TRY(cudaEventRecord(ev[0], s));
  const float uniform = 1.0f / static_cast<float>(n);
  const float omd = 1.0f - damping;
  std::vector<double> trace_tile(static_cast<size_t>(std::max(max_iters, 1)) * Bmax);
  std::vector<int32_t> sweeps_tile(kMaxTile);
  for (int c0 = 0; c0 < ncols; c0 += tile) {
    const int B = std::min(tile, ncols - c0);
    const int T = 256;
    const unsigned ib = static_cast<unsigned>((n * B + T - 1) / T);
    if (g.weighted)
      batch_init_kernel<true, false><<<ib, T, 0, s>>>(static_cast<int32_t>(n), B, ncols, c0, g.perm, g.rowoff, g.odeg, g.rsum, tele_old, uniform, omd, bs.S, bs.C[0], bs.base);
    else if (g.directed)
      batch_init_kernel<false, true><<<ib, T, 0, s>>>(static_cast<int32_t>(n), B, ncols, c0, g.perm, g.rowoff, g.odeg, g.rsum, tele_old, uniform, omd, bs.S, bs.C[0], bs.base);
    else
      batch_init_kernel<false, false><<<ib, T, 0, s>>>(static_cast<int32_t>(n), B, ncols, c0, g.perm, g.rowoff, g.odeg, g.rsum, tele_old, uniform, omd, bs.S, bs.C[0], bs.base);
    nl++;
    BatchCtl ctl0;
    std::memset(&ctl0, 0, sizeof(ctl0));
    ctl0.active = (B == 64) ? ~0ull : ((1ull << B) - 1ull);
    ctl0.loop.done = max_iters == 0 ? 1 : 0;
    PB_TRY(cudaMemcpyAsync(bs.ctl, &ctl0, sizeof(ctl0), cudaMemcpyHostToDevice, s));
    PB_TRY(cudaMemsetAsync(bs.tick1, 0, sizeof(unsigned) * (ngroups + 1), s));
    PB_TRY(cudaMemsetAsync(bs.sweeps, 0, sizeof(int32_t) * kMaxTile, s));
    if (max_iters)
      PB_TRY(cudaMemsetAsync(bs.trace, 0, sizeof(double) * static_cast<int64_t>(max_iters) * B, s));
    BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = static_cast<int32_t>(n);
    a.B = B;
    a.rowoff = g.rowoff;
    a.col = g.col;
    a.win = g.weighted ? g.win : nullptr;
    a.odeg = g.odeg;
    a.rsum = g.rsum;
    a.base = bs.base;
    a.damping = damping;
    a.S = bs.S;
    a.nseg = nseg;
    a.hub_rows = static_cast<int32_t>(g.num_hub_rows);
    a.zero_start = static_cast<int32_t>(g.bin_row_start[kBinZero]);
    a.warp_blocks = warp_blocks;
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
    a.epsilon = epsilon;
    a.C0 = bs.C[0];
    a.C1 = bs.C[1];
    const void *fn = g.weighted ? reinterpret_cast<const void *>(batch_sweep_kernel<true, false>)
                   : g.directed ? reinterpret_cast<const void *>(batch_sweep_kernel<false, true>)
                                : reinterpret_cast<const void *>(batch_sweep_kernel<false, false>);
    PB_TRY(cudaEventRecord(ev[1], s));
    PB_TRY(bs.loop.Launch(fn, dim3(nblocks), dim3(kBT), &a, sizeof(a), &bs.ctl->loop, max_iters, s));
    PB_TRY(cudaEventRecord(ev[2], s));
    batch_out_kernel<<<ib, T, 0, s>>>(static_cast<int32_t>(n), B, ncols, c0, g.inv, bs.S, out_old);
    nl++;
    PB_TRY(cudaGetLastError());
    PB_TRY(cudaMemcpyAsync(sweeps_tile.data(), bs.sweeps, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, s));
    if (max_iters)
      PB_TRY(cudaMemcpyAsync(trace_tile.data(), bs.trace, sizeof(double) * static_cast<int64_t>(max_iters) * B,
                             cudaMemcpyDeviceToHost, s));
    PB_TRY(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[1], ev[2]);
    sweep_total += ms;
    int tile_loops = 0;
    for (int c = 0; c < B; c++) tile_loops = std::max(tile_loops, sweeps_tile[c]);
    nl += 2 * tile_loops;  // sweep + decide kernel per executed sweep
    for (int c = 0; c < B; c++) {
      if (sweeps_out) sweeps_out[c0 + c] = sweeps_tile[c];
      if (err_trace)
        for (int it = 0; it < max_iters; it++)
          err_trace[static_cast<int64_t>(it) * ncols + c0 + c] = trace_tile[static_cast<int64_t>(it) * B + c];
    }
  }
  PB_TRY(cudaEventRecord(ev[3], s));
  PB_TRY(cudaEventSynchronize(ev[3]));
  float tot = 0;
  cudaEventElapsedTime(&tot, ev[0], ev[3]);
  for (auto &e : ev) cudaEventDestroy(e);
  *ms_sweep = sweep_total;
  *ms_total = tot;
  *launches = nl;
  return cudaSuccess;
}

#undef PB_TRY

}  // namespace prgpu
