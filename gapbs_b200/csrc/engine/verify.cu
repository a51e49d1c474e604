// verify.cu -- the reference's PRVerifier (src/pr_spmv.cc:78-94) on the device.
//
// The reference pushes contrib[u] = score[u] / out_degree(u) along the
// out-edges of u = 0, 1, 2, ... in turn, so incoming[v] is the float sum of
// v's in-neighbours' contribs in ascending source order, and the check is
// error = sum over n of |base + d * incoming[n] - score[n]| (float
// arithmetic per vertex, added in double in vertex order).
//
// The renumbered in-CSR keeps every row in the caller's order, and the
// reference's builder sorts each row by source id (src/builder.h:154-156), so
// adding a row's contribs one at a time in row order gives incoming[v] bit for
// bit.  Rows are in descending-length order: a warp takes each of the long
// rows (its lanes fetch 32 contribs at once, so the gathers are in flight
// together, then add them in row order, each term broadcast to the warp), and
// a thread takes each of the short ones (adding its row in order, four loads
// issued ahead).  Either way the sum keeps its sequential rounding.  The
// residual of each row is written at the vertex's original id; the host adds
// them in double in id order, which is the reference's own L1 sum.  Nothing
// here shares code with the sweep kernels, so the check does not inherit a
// fault of theirs.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace prgpu {

namespace {

constexpr int kVerifyThreads = 256;
constexpr int kLongRow = 32;  // rows of at least this many entries get a warp
constexpr unsigned kFull = 0xffffffffu;

// contrib[v] = score[perm[v]] / out_degree(v) over new ids: the float score
// divided by the degree converted to float (src/pr_spmv.cc:83).  A vertex
// without out-edges gets inf or NaN, as in the reference; no row reads it.
__global__ void verify_contrib_kernel(int64_t n, const float *__restrict__ score_orig,
                                      const int32_t *__restrict__ perm,
                                      const int32_t *__restrict__ rowoff,
                                      const int32_t *__restrict__ odeg, float *contrib) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int32_t deg = odeg ? odeg[v] : rowoff[v + 1] - rowoff[v];
  contrib[v] = __fdiv_rn(score_orig[perm[v]], __int2float_rn(deg));
}

// resid_orig[perm[u]] = |base + d * sum - score|, each operation rounded on
// its own (src/pr_spmv.cc:89).
__device__ __forceinline__ void write_residual(int64_t u, float sum,
                                               const float *__restrict__ score_orig,
                                               const int32_t *__restrict__ perm, float base,
                                               float damping, float *resid_orig) {
  const int32_t v = perm[u];
  const float r = __fsub_rn(__fadd_rn(base, __fmul_rn(damping, sum)), score_orig[v]);
  resid_orig[v] = fabsf(r);
}

// One warp per row of [0, nrows) (grid-stride over rows): the row's contribs
// are fetched 32 at a time, the next 32 while the current ones are added;
// every lane keeps the same running sum.  A full chunk's 32 broadcasts are
// unrolled, so they are issued ahead of their adds.  The longest rows bound
// the kernel: each is one warp's sequential sum, fetched one chunk ahead, so
// the longest row at Kronecker scale 25 (639,467 entries) waits on memory
// about 20,000 times in turn.
__global__ void __launch_bounds__(kVerifyThreads, 4)
verify_long_rows_kernel(int64_t nrows, const int32_t *__restrict__ rowoff,
                        const int32_t *__restrict__ col, const float *__restrict__ contrib,
                        const float *__restrict__ score_orig, const int32_t *__restrict__ perm,
                        float base, float damping, float *resid_orig) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kVerifyThreads / 32);
  for (int64_t u = (static_cast<int64_t>(blockIdx.x) * kVerifyThreads + threadIdx.x) >> 5;
       u < nrows; u += warps) {
    const int32_t lo = rowoff[u], hi = rowoff[u + 1];
    float sum = 0.f;
    float c = lo + lane < hi ? contrib[col[lo + lane]] : 0.f;
    for (int32_t j = lo; j < hi; j += 32) {
      const int cnt = min(32, hi - j);
      const int32_t jn = j + 32 + lane;
      const float cn = jn < hi ? contrib[col[jn]] : 0.f;
      if (cnt == 32) {
#pragma unroll
        for (int k = 0; k < 32; k++) sum = __fadd_rn(sum, __shfl_sync(kFull, c, k));
      } else {
        for (int k = 0; k < cnt; k++) sum = __fadd_rn(sum, __shfl_sync(kFull, c, k));
      }
      c = cn;
    }
    if (lane == 0) write_residual(u, sum, score_orig, perm, base, damping, resid_orig);
  }
}

// One thread per row of [r0, n): the thread adds its row's contribs in row
// order, the loads of four entries issued before their adds.
__global__ void __launch_bounds__(kVerifyThreads)
verify_short_rows_kernel(int64_t r0, int64_t n, const int32_t *__restrict__ rowoff,
                         const int32_t *__restrict__ col, const float *__restrict__ contrib,
                         const float *__restrict__ score_orig, const int32_t *__restrict__ perm,
                         float base, float damping, float *resid_orig) {
  const int64_t u = r0 + static_cast<int64_t>(blockIdx.x) * kVerifyThreads + threadIdx.x;
  if (u >= n) return;
  const int32_t lo = rowoff[u], hi = rowoff[u + 1];
  float sum = 0.f;
  int32_t j = lo;
  for (; j + 3 < hi; j += 4) {
    const float c0 = contrib[col[j]], c1 = contrib[col[j + 1]];
    const float c2 = contrib[col[j + 2]], c3 = contrib[col[j + 3]];
    sum = __fadd_rn(sum, c0);
    sum = __fadd_rn(sum, c1);
    sum = __fadd_rn(sum, c2);
    sum = __fadd_rn(sum, c3);
  }
  for (; j < hi; j++) sum = __fadd_rn(sum, contrib[col[j]]);
  write_residual(u, sum, score_orig, perm, base, damping, resid_orig);
}

}  // namespace

cudaError_t VerifyResiduals(const DeviceGraph &g, const float *score_orig, float damping,
                            float *contrib, float *resid_orig, cudaStream_t s) {
  const int64_t n = g.n;
  if (n < 1) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  // the reference's base score: (1 - d) / N in float, N converted to float
  const float base = (1.0f - damping) / static_cast<float>(n);
  verify_contrib_kernel<<<static_cast<unsigned>((n + kVerifyThreads - 1) / kVerifyThreads),
                          kVerifyThreads, 0, s>>>(n, score_orig, g.perm, g.rowoff,
                                                  g.directed ? g.odeg : nullptr, contrib);
  // long rows: those of the degree bins of at least kLongRow entries (the
  // split only decides which kernel adds a row, never the result)
  int b = 0;
  while (b < kBinZero && g.bins.min_len[b] >= kLongRow) b++;
  const int64_t nlong = std::min<int64_t>(n, g.bin_row_start[b]);
  if (nlong > 0) {
    // up to 8 blocks of 8 warps per SM (the most that can be resident)
    const int64_t want = (nlong + kVerifyThreads / 32 - 1) / (kVerifyThreads / 32);
    const unsigned grid = static_cast<unsigned>(
        std::min<int64_t>(want, static_cast<int64_t>(sms) * (2048 / kVerifyThreads)));
    verify_long_rows_kernel<<<grid, kVerifyThreads, 0, s>>>(
        nlong, g.rowoff, g.col, contrib, score_orig, g.perm, base, damping, resid_orig);
  }
  if (n > nlong)
    verify_short_rows_kernel<<<static_cast<unsigned>((n - nlong + kVerifyThreads - 1) /
                                                     kVerifyThreads),
                               kVerifyThreads, 0, s>>>(nlong, n, g.rowoff, g.col, contrib,
                                                       score_orig, g.perm, base, damping,
                                                       resid_orig);
  return cudaGetLastError();
}

}  // namespace prgpu
