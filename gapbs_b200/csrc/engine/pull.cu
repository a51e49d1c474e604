// pull.cu -- the fused pull-direction Jacobi sweep (one launch per sweep).
//
// One launch performs, for every vertex u, what the reference does in two
// OpenMP loops plus a reduction (src/pr_spmv.cc:43-54):
//   sum   = sum over in-neighbours v of contrib[v]
//   new   = base + d * sum                      (float, two roundings)
//   err  += |new - old|                          (float difference, FP64 sum)
//   contrib'[u] = new / out_degree(u)            (next sweep's input)
// and then decides convergence on the device (error < epsilon, :57-58), so a
// whole solve is max_iters back-to-back launches with no host round trip; a
// launch that finds the solve converged returns immediately.
//
// Work split (rows are renumbered by descending in-degree, so each bin is a
// contiguous row range):
//   HUB   one block per kSegEntries-entry segment of a long row; the block
//         that finishes a row's last segment (per-row ticket) sums the
//         segment partials in segment order and updates the row;
//   G=32..1  lane groups of G threads per row, 128-bit neighbour loads (each
//         lane reads whole aligned 4-entry chunks and masks entries outside
//         its row), two chunks in flight per lane, xor-tree group sum;
//   ZERO  rows without in-neighbours: new = base.
// Every |new - old| is added to an FP64 per-thread sum (the reference adds
// each to a double, src/pr_spmv.cc:42,53), then reduced with a deterministic
// two-stage tree (per-block partials -> per-512-block group -> total).
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "sweep_reduce.cuh"

namespace prgpu {

// The reference's float update: base + d * sum with two roundings (no FMA).
__device__ __forceinline__ float pr_update(float base, float d, float sum) {
  return __fadd_rn(base, __fmul_rn(d, sum));
}

__device__ __forceinline__ float ld_contrib(const float *cin, int v, int l1_rows, uint64_t pg) {
  return v < l1_rows ? ld_gather(cin + v, pg) : ld_gather_cold(cin + v, pg);
}

template <bool W>
__device__ __forceinline__ float gather_chunk(float acc, const int4 q, const float4 w,
                                              int b, int s, int e, const float *cin,
                                              int l1_rows, uint64_t pg) {
  const bool i0 = (b >= s) & (b < e);
  const bool i1 = (b + 1 >= s) & (b + 1 < e);
  const bool i2 = (b + 2 >= s) & (b + 2 < e);
  const bool i3 = (b + 3 >= s) & (b + 3 < e);
  float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
  if (i0) v0 = ld_contrib(cin, q.x, l1_rows, pg);
  if (i1) v1 = ld_contrib(cin, q.y, l1_rows, pg);
  if (i2) v2 = ld_contrib(cin, q.z, l1_rows, pg);
  if (i3) v3 = ld_contrib(cin, q.w, l1_rows, pg);
  if (W) {
    if (i0) acc = __fmaf_rn(w.x, v0, acc);
    if (i1) acc = __fmaf_rn(w.y, v1, acc);
    if (i2) acc = __fmaf_rn(w.z, v2, acc);
    if (i3) acc = __fmaf_rn(w.w, v3, acc);
  } else {
    if (i0) acc = __fadd_rn(acc, v0);
    if (i1) acc = __fadd_rn(acc, v1);
    if (i2) acc = __fadd_rn(acc, v2);
    if (i3) acc = __fadd_rn(acc, v3);
  }
  return acc;
}

// Sum over entries [s, e) by the calling lane of a G-lane group: the lane
// takes aligned 4-entry chunks (s/4 + lane), (s/4 + lane + G), ...; up to four
// chunk loads are in flight before their gathers are issued.
template <int G, bool W>
__device__ __forceinline__ float lane_partial(const PullArgs &a, const float *cin, int s, int e,
                                              int lane, uint64_t ps, uint64_t pg) {
  const int4 *col4 = reinterpret_cast<const int4 *>(a.col);
  const float4 *w4 = reinterpret_cast<const float4 *>(a.win);
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const int4 zi = make_int4(0, 0, 0, 0);
  float acc = 0.f;
  const int c1 = (e + 3) >> 2;
  int c = (s >> 2) + lane;
  for (; c + 3 * G < c1; c += 4 * G) {
    const int4 q0 = ld_stream_v4(col4 + c, ps);
    const int4 q1 = ld_stream_v4(col4 + c + G, ps);
    const int4 q2 = ld_stream_v4(col4 + c + 2 * G, ps);
    const int4 q3 = ld_stream_v4(col4 + c + 3 * G, ps);
    float4 w0 = z4, w1 = z4, w2 = z4, w3 = z4;
    if (W) {
      w0 = ld_stream_v4f(w4 + c, ps);
      w1 = ld_stream_v4f(w4 + c + G, ps);
      w2 = ld_stream_v4f(w4 + c + 2 * G, ps);
      w3 = ld_stream_v4f(w4 + c + 3 * G, ps);
    }
    acc = gather_chunk<W>(acc, q0, w0, c << 2, s, e, cin, a.l1_rows, pg);
    acc = gather_chunk<W>(acc, q1, w1, (c + G) << 2, s, e, cin, a.l1_rows, pg);
    acc = gather_chunk<W>(acc, q2, w2, (c + 2 * G) << 2, s, e, cin, a.l1_rows, pg);
    acc = gather_chunk<W>(acc, q3, w3, (c + 3 * G) << 2, s, e, cin, a.l1_rows, pg);
  }
  if (c < c1) {
    // up to three remaining chunks, loads predicated on the row's last chunk
    const bool h1 = c + G < c1, h2 = c + 2 * G < c1;
    const int4 q0 = ld_stream_v4(col4 + c, ps);
    const int4 q1 = h1 ? ld_stream_v4(col4 + c + G, ps) : zi;
    const int4 q2 = h2 ? ld_stream_v4(col4 + c + 2 * G, ps) : zi;
    float4 w0 = z4, w1 = z4, w2 = z4;
    if (W) {
      w0 = ld_stream_v4f(w4 + c, ps);
      if (h1) w1 = ld_stream_v4f(w4 + c + G, ps);
      if (h2) w2 = ld_stream_v4f(w4 + c + 2 * G, ps);
    }
    acc = gather_chunk<W>(acc, q0, w0, c << 2, s, e, cin, a.l1_rows, pg);
    if (h1) acc = gather_chunk<W>(acc, q1, w1, (c + G) << 2, s, e, cin, a.l1_rows, pg);
    if (h2) acc = gather_chunk<W>(acc, q2, w2, (c + 2 * G) << 2, s, e, cin, a.l1_rows, pg);
  }
  return acc;
}

template <bool W, bool DIR>
__device__ __forceinline__ float denom_of(const PullArgs &a, int u, int s, int e) {
  if (W) return a.rsum[u];
  if (DIR) return __int2float_rn(a.odeg[u]);
  return __int2float_rn(e - s);
}

// Updates row u from its gathered sum; returns |new - old| (as float).
template <bool W, bool DIR, int KIND>
__device__ __forceinline__ float finish_row(const PullArgs &a, float *cout, int u, int s, int e,
                                            float sum, float old, uint64_t ps, uint64_t pl) {
  const float base = KIND != kKindPlain ? a.base_vec[u] : a.base_scalar;
  if (KIND == kKindAdjoint) {
    // lambda[v] = w[v] + d * (sum_u w(v->u) lambda[u]) / S_v; lambda itself
    // is what the next sweep gathers.
    // A vertex without out-edges has no row in P: (P lambda)[v] = 0.
    const float den = denom_of<W, DIR>(a, u, s, e);
    const float nw = pr_update(base, a.damping, den > 0.f ? __fdiv_rn(sum, den) : 0.f);
    st_hint_f32(a.score + u, nw, ps);
    st_hint_f32(cout + u, nw, pl);
    return fabsf(__fsub_rn(nw, old));
  }
  const float nw = pr_update(base, a.damping, sum);
  st_hint_f32(a.score + u, nw, ps);
  st_hint_f32(cout + u, __fdiv_rn(nw, denom_of<W, DIR>(a, u, s, e)), pl);
  return fabsf(__fsub_rn(nw, old));
}

// Deterministic two-stage FP64 grid reduction of the block errors; the last
// block records the sweep's error and the convergence decision.
__device__ __forceinline__ void grid_finish(const PullArgs &a, int it, double block_err,
                                            double *sred) {
  const SweepReduce r{a.part1, a.part2, a.tick1, a.trace, a.ctl, a.nblocks, a.epsilon};
  sweep_grid_finish<kSweepThreads>(r, it, block_err, sred);
}

// One warp task of a G-lane-group bin: rows bin_row[bin] + task * (32 / G)
// + lane / G, one row per group.  The group leader's old-score load is issued
// before the gather so the two latencies overlap.
template <int G, bool W, bool DIR, int KIND>
__device__ __forceinline__ float warp_task(const PullArgs &a, const float *cin, float *cout,
                                           int bin, int task, int lane32, uint64_t ps,
                                           uint64_t pg, uint64_t pl) {
  constexpr int kRowsPerTask = 32 / G;
  const int lane = lane32 % G;
  const int u = a.bin_row[bin] + task * kRowsPerTask + lane32 / G;
  const bool valid = u < a.bin_row[bin + 1];
  int s = 0, e = 0;
  float old = 0.f;
  if (valid) {
    s = a.rowoff[u];
    e = a.rowoff[u + 1];
    if (lane == 0) old = ld_score(a.score + u, ps);
  }
  float acc = lane_partial<G, W>(a, cin, s, e, lane, ps, pg);
  acc = group_sum<G>(acc);
  float err = 0.f;
  if (valid && lane == 0) err = finish_row<W, DIR, KIND>(a, cout, u, s, e, acc, old, ps, pl);
  return err;
}

// One hub segment, processed by the whole block; the block that completes a
// row's last segment (per-row ticket) sums the row's segment partials in
// segment order and updates the row.  Called block-uniformly.
template <bool W, bool DIR, int KIND>
__device__ __forceinline__ float hub_segment(const PullArgs &a, const float *cin, float *cout,
                                             float *sredf, int seg, uint64_t ps, uint64_t pg,
                                             uint64_t pl) {
  __shared__ int s_fin;
  const int u = a.seg_row[seg];
  const int first = a.seg_first[u];
  const int nseg = a.seg_first[u + 1] - first;
  const int rs = a.rowoff[u], re = a.rowoff[u + 1];
  const int s = rs + (seg - first) * kSegEntries;
  const int e = min(re, s + kSegEntries);
  float acc = lane_partial<kSweepThreads, W>(a, cin, s, e, threadIdx.x, ps, pg);
  const float part = block_sum_f<kSweepThreads>(acc, sredf);
  if (threadIdx.x == 0) {
    a.seg_partial[seg] = part;
    __threadfence();
    const unsigned t = atomicAdd(a.hub_ticket + u, 1u);
    s_fin = (t == static_cast<unsigned>(nseg - 1));
  }
  __syncthreads();
  float err = 0.f;
  if (s_fin && threadIdx.x == 0) {
    __threadfence();
    float sum = 0.f;
    for (int k = 0; k < nseg; k++) sum = __fadd_rn(sum, __ldcg(a.seg_partial + first + k));
    a.hub_ticket[u] = 0;
    err = finish_row<W, DIR, KIND>(a, cout, u, rs, re, sum, ld_score(a.score + u, ps), ps, pl);
  }
  return err;
}

// One warp task of the ZERO bin: 32 * kZeroRowsPerThread rows without
// in-neighbours (new = base).
template <bool W, bool DIR, int KIND>
__device__ __forceinline__ double zero_task(const PullArgs &a, float *cout, int task, int lane32,
                                           uint64_t ps, uint64_t pl) {
  constexpr int kRows = 32 * kZeroRowsPerThread;
  const int row0 = a.bin_row[kBinZero] + task * kRows;
  const int end = a.bin_row[kBinZero + 1];
  float old[kZeroRowsPerThread];
#pragma unroll
  for (int i = 0; i < kZeroRowsPerThread; i++) {
    const int u = row0 + i * 32 + lane32;
    old[i] = u < end ? ld_score(a.score + u, ps) : 0.f;
  }
  double err = 0.0;
#pragma unroll
  for (int i = 0; i < kZeroRowsPerThread; i++) {
    const int u = row0 + i * 32 + lane32;
    if (u < end) {
      const float base = KIND != kKindPlain ? a.base_vec[u] : a.base_scalar;
      const float nw = pr_update(base, a.damping, 0.f);
      st_hint_f32(a.score + u, nw, ps);
      // A row without in-neighbours can still have out-neighbours in a
      // directed graph; its contrib is then read by the next sweep.
      if (KIND == kKindAdjoint) st_hint_f32(cout + u, nw, pl);
      else if (W || DIR) st_hint_f32(cout + u, __fdiv_rn(nw, denom_of<W, DIR>(a, u, 0, 0)), pl);
      err += static_cast<double>(fabsf(__fsub_rn(nw, old[i])));
    }
  }
  return err;
}

// Persistent sweep: every block first takes hub segments (block-cooperative,
// round-robin), then every warp takes row tasks of bins 1..7 interleaved
// across all warps of the grid.  Rows are sorted by length, so interleaving
// hands every warp an even share of each length class.  One block reduction
// and one grid reduction per sweep.
template <bool W, bool DIR, int KIND>
__global__ void __launch_bounds__(kSweepThreads)
pull_sweep_kernel(const PullArgs a) {
  if (*reinterpret_cast<volatile const int *>(&a.ctl->loop.done)) return;
  const int it = *reinterpret_cast<volatile const int *>(&a.ctl->loop.loops);
  const float *cin = (it & 1) ? a.c1 : a.c0;
  float *cout = (it & 1) ? a.c0 : a.c1;
  __shared__ double sred[kSweepThreads / 32];
  __shared__ float sredf[kSweepThreads / 32];
  const uint64_t ps = policy_evict_first();
  const uint64_t pg = policy_evict_last();
  const uint64_t pl = pg;
  // every |new - old| is added in FP64, as the reference adds it to a double
  double err = 0.0;
  for (int seg = blockIdx.x; seg < a.nseg; seg += gridDim.x)
    err += hub_segment<W, DIR, KIND>(a, cin, cout, sredf, seg, ps, pg, pl);
  const int lane32 = threadIdx.x & 31;
  const int gw = blockIdx.x * (kSweepThreads / 32) + (threadIdx.x >> 5);
  const int nw = gridDim.x * (kSweepThreads / 32);
  // rows without in-neighbours (the last bin) are final after their first
  // sweep (their second for a directed graph, whose contribs they supply)
  const int ntasks = (it >= a.zero_final_sweep) ? a.task_start[kBinZero] : a.task_start[kNumBins];
  for (int t = gw; t < ntasks; t += nw) {
    int bin = 1;
#pragma unroll
    for (int i = 2; i < kNumBins; i++) bin += (t >= a.task_start[i]);
    const int k = t - a.task_start[bin];
    switch (bin) {
      case 1: err += warp_task<32, W, DIR, KIND>(a, cin, cout, 1, k, lane32, ps, pg, pl); break;
      case 2: err += warp_task<16, W, DIR, KIND>(a, cin, cout, 2, k, lane32, ps, pg, pl); break;
      case 3: err += warp_task<8, W, DIR, KIND>(a, cin, cout, 3, k, lane32, ps, pg, pl); break;
      case 4: err += warp_task<4, W, DIR, KIND>(a, cin, cout, 4, k, lane32, ps, pg, pl); break;
      case 5: err += warp_task<2, W, DIR, KIND>(a, cin, cout, 5, k, lane32, ps, pg, pl); break;
      case 6: err += warp_task<1, W, DIR, KIND>(a, cin, cout, 6, k, lane32, ps, pg, pl); break;
      default: err += zero_task<W, DIR, KIND>(a, cout, k, lane32, ps, pl); break;
    }
  }
  const double block_err = block_sum_d<kSweepThreads>(err, sred);
  grid_finish(a, it, block_err, sred);
}

// ---- generic warp-per-row sweep (unsorted CSR, grid-stride) ----------------

template <bool W, int KIND>
__global__ void __launch_bounds__(kSweepThreads)
pull_generic_kernel(const PullArgs a) {
  if (*reinterpret_cast<volatile const int *>(&a.ctl->loop.done)) return;
  const int it = *reinterpret_cast<volatile const int *>(&a.ctl->loop.loops);
  const float *cin = (it & 1) ? a.c1 : a.c0;
  float *cout = (it & 1) ? a.c0 : a.c1;
  __shared__ double sred[kSweepThreads / 32];
  const uint64_t ps = policy_evict_first();
  const uint64_t pg = policy_evict_last();
  const int lane = threadIdx.x & 31;
  const int warps = a.nblocks * (kSweepThreads / 32);
  double err = 0.0;
  for (int u = blockIdx.x * (kSweepThreads / 32) + (threadIdx.x >> 5); u < a.n; u += warps) {
    const int s = a.rowoff[u], e = a.rowoff[u + 1];
    float acc = lane_partial<32, W>(a, cin, s, e, lane, ps, pg);
    acc = group_sum<32>(acc);
    if (lane == 0)
      err += finish_row<W, false, KIND>(a, cout, u, s, e, acc, ld_score(a.score + u, ps), ps, pg);
  }
  const double block_err = block_sum_d<kSweepThreads>(err, sred);
  grid_finish(a, it, block_err, sred);
}

const void *PullGenericKernel(const PullArgs &a) {
  const bool W = a.win != nullptr;
  if (a.kind == kKindAdjoint)
    return W ? reinterpret_cast<const void *>(pull_generic_kernel<true, kKindAdjoint>)
             : reinterpret_cast<const void *>(pull_generic_kernel<false, kKindAdjoint>);
  return W ? reinterpret_cast<const void *>(pull_generic_kernel<true, kKindPPR>)
           : reinterpret_cast<const void *>(pull_generic_kernel<false, kKindPPR>);
}

// ---- adjoint gradients ---------------------------------------------------------

// One warp per renumbered out-row v:
//   (P lambda)[v] = sum_e w_e lambda[u_e] / S_v
//   grad_ew[orig position of e] = d s[v] / S_v (lambda[u_e] - (P lambda)[v])
__global__ void adjoint_edge_grad_kernel(int32_t n, const int32_t *__restrict__ orow,
                                         const int32_t *__restrict__ ocol,
                                         const float *__restrict__ wout,
                                         const float *__restrict__ rsum,
                                         const int32_t *__restrict__ perm,
                                         const int32_t *__restrict__ orig_off,
                                         const float *__restrict__ lam,
                                         const float *__restrict__ sv, float damping,
                                         float *grad_ew) {
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int v = static_cast<int>(warp);
  const int s = orow[v], e = orow[v + 1];
  if (s == e) return;
  double acc = 0;
  for (int j = s + lane; j < e; j += 32)
    acc += static_cast<double>(wout ? wout[j] : 1.f) * lam[ocol[j]];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const double S = rsum ? static_cast<double>(rsum[v]) : static_cast<double>(e - s);
  const double plam = acc / S;
  const double coef = static_cast<double>(damping) * sv[v] / S;
  const int64_t base = orig_off[perm[v]];
  for (int j = s + lane; j < e; j += 32)
    grad_ew[base + (j - s)] = static_cast<float>(coef * (lam[ocol[j]] - plam));
}

__global__ void adjoint_teleport_grad_kernel(int32_t n, const int32_t *__restrict__ inv,
                                             const float *__restrict__ lam, float omd,
                                             float *grad_t) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= n) return;
  grad_t[v] = __fmul_rn(omd, lam[inv[v]]);
}

cudaError_t LaunchAdjointGrads(const DeviceGraph &g, const int32_t *orow, const int32_t *ocol,
                               const float *wout, const float *lam_new, const float *s_new,
                               float damping, float *grad_ew, float *grad_t_old,
                               cudaStream_t s) {
  const int n = static_cast<int>(g.n);
  if (grad_ew) {
    adjoint_edge_grad_kernel<<<static_cast<unsigned>((static_cast<int64_t>(n) * 32 + 255) / 256), 256, 0, s>>>(
        n, orow, ocol, wout, g.weighted ? g.rsum : nullptr, g.perm, g.orig_out_off, lam_new, s_new,
        damping, grad_ew);
  }
  if (grad_t_old)
    adjoint_teleport_grad_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, g.inv, lam_new, 1.0f - damping,
                                                                 grad_t_old);
  return cudaGetLastError();
}

// Deterministic sum_i |x_i| in double: one block, fixed stride order.
__global__ void l1_norm_kernel(const float *__restrict__ x, int64_t n, double *out) {
  __shared__ double sred[32];
  double v = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) v += fabs(static_cast<double>(x[i]));
  const double t = block_sum_d<1024>(v, sred);
  if (threadIdx.x == 0) *out = t;
}

cudaError_t LaunchL1Norm(const float *x, int64_t n, double *out, cudaStream_t s) {
  l1_norm_kernel<<<1, 1024, 0, s>>>(x, n, out);
  return cudaGetLastError();
}

// ---- init / permutation kernels ---------------------------------------------

template <bool W, bool DIR>
__global__ void pull_init_kernel(int32_t n, const int32_t *__restrict__ rowoff,
                                 const int32_t *__restrict__ odeg,
                                 const float *__restrict__ rsum,
                                 const float *__restrict__ tele_new, float init_scalar,
                                 float one_minus_d, float *score, float *contrib,
                                 float *base) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const float t = tele_new ? tele_new[u] : init_scalar;
  score[u] = t;
  if (tele_new) base[u] = __fmul_rn(one_minus_d, t);
  float denom;
  if (W) denom = rsum[u];
  else if (DIR) denom = __int2float_rn(odeg[u]);
  else denom = __int2float_rn(rowoff[u + 1] - rowoff[u]);
  contrib[u] = __fdiv_rn(t, denom);
}

__global__ void gather_out_kernel(int32_t n, int ncols, const int32_t *__restrict__ inv,
                                  const float *__restrict__ src_new, float *dst_old) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<int64_t>(n) * ncols) return;
  const int64_t v = i / ncols;
  const int c = static_cast<int>(i - v * ncols);
  dst_old[i] = src_new[static_cast<int64_t>(inv[v]) * ncols + c];
}

__global__ void gather_in_kernel(int32_t n, int ncols, const int32_t *__restrict__ perm,
                                 const float *__restrict__ src_old, float *dst_new) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<int64_t>(n) * ncols) return;
  const int64_t u = i / ncols;
  const int c = static_cast<int>(i - u * ncols);
  dst_new[i] = src_old[static_cast<int64_t>(perm[u]) * ncols + c];
}

// ---- launchers ---------------------------------------------------------------

int PullTasks(const DeviceGraph &g, int32_t task_start[kNumBins + 1]) {
  int64_t tasks = 0;
  task_start[0] = 0;
  for (int b = 1; b < kNumBins; b++) {
    task_start[b] = static_cast<int32_t>(tasks);
    const int64_t rows = g.bin_row_start[b + 1] - g.bin_row_start[b];
    const int64_t per = (b == kBinZero) ? 32 * kZeroRowsPerThread : 32 / kBinGroup[b];
    tasks += (rows + per - 1) / per;
  }
  task_start[kNumBins] = static_cast<int32_t>(tasks);
  return static_cast<int>(tasks);
}

int PullGrid(const void *kernel) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSweepThreads, 0) !=
          cudaSuccess || per_sm < 1)
    per_sm = 1;
  return sms * per_sm;
}

template <bool W, bool DIR>
const void *SweepForKind(int kind) {
  if (kind == kKindPlain) return reinterpret_cast<const void *>(pull_sweep_kernel<W, DIR, kKindPlain>);
  if (kind == kKindPPR) return reinterpret_cast<const void *>(pull_sweep_kernel<W, DIR, kKindPPR>);
  return reinterpret_cast<const void *>(pull_sweep_kernel<W, DIR, kKindAdjoint>);
}

const void *PullSweepKernel(const PullArgs &a) {
  if (a.win != nullptr) return SweepForKind<true, false>(a.kind);
  if (a.odeg != nullptr) return SweepForKind<false, true>(a.kind);
  return SweepForKind<false, false>(a.kind);
}

cudaError_t LaunchPullInit(const DeviceGraph &g, Scratch &sc, const float *tele_new,
                           float init_scalar, float damping, cudaStream_t s) {
  const int n = static_cast<int>(g.n);
  if (n == 0) return cudaSuccess;
  const int threads = 256;
  const int blocks = (n + threads - 1) / threads;
  const float omd = 1.0f - damping;
  if (g.weighted)
    pull_init_kernel<true, false><<<blocks, threads, 0, s>>>(
        n, g.rowoff, g.odeg, g.rsum, tele_new, init_scalar, omd, sc.score, sc.contrib[0], sc.base);
  else if (g.directed)
    pull_init_kernel<false, true><<<blocks, threads, 0, s>>>(
        n, g.rowoff, g.odeg, g.rsum, tele_new, init_scalar, omd, sc.score, sc.contrib[0], sc.base);
  else
    pull_init_kernel<false, false><<<blocks, threads, 0, s>>>(
        n, g.rowoff, g.odeg, g.rsum, tele_new, init_scalar, omd, sc.score, sc.contrib[0], sc.base);
  return cudaGetLastError();
}

cudaError_t LaunchGatherOut(const DeviceGraph &g, const float *src_new, float *dst_old,
                            int ncols, cudaStream_t s) {
  const int64_t total = g.n * ncols;
  if (total == 0) return cudaSuccess;
  const int threads = 256;
  const int64_t blocks = (total + threads - 1) / threads;
  gather_out_kernel<<<static_cast<unsigned>(blocks), threads, 0, s>>>(
      static_cast<int32_t>(g.n), ncols, g.inv, src_new, dst_old);
  return cudaGetLastError();
}

cudaError_t LaunchScatterIn(const DeviceGraph &g, const float *src_old, float *dst_new,
                            int ncols, cudaStream_t s) {
  const int64_t total = g.n * ncols;
  if (total == 0) return cudaSuccess;
  const int threads = 256;
  const int64_t blocks = (total + threads - 1) / threads;
  gather_in_kernel<<<static_cast<unsigned>(blocks), threads, 0, s>>>(
      static_cast<int32_t>(g.n), ncols, g.perm, src_old, dst_new);
  return cudaGetLastError();
}

cudaError_t LaunchResetCtl(Scratch &sc, int nblocks, int iters, cudaStream_t s) {
  const int ngroups = (nblocks + kReduceGroup - 1) / kReduceGroup;
  cudaError_t e = cudaMemsetAsync(sc.ctl, 0, sizeof(SweepCtl), s);
  if (e != cudaSuccess) return e;
  if (ngroups) e = cudaMemsetAsync(sc.tick1, 0, sizeof(unsigned) * ngroups, s);
  if (e != cudaSuccess) return e;
  if (iters) e = cudaMemsetAsync(sc.trace, 0, sizeof(double) * iters, s);
  return e;
}

}  // namespace prgpu
