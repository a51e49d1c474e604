// prep.cu -- upload-time construction of the device graph mirror.
//
// Runs once per pr_gpu_upload, outside any timed solve:
//   1. validate the CSR on the device (offsets monotone from 0 to m, ids in
//      [0, n), weights finite and positive, out-rows sorted when weighted);
//   2. renumber vertices by descending in-degree (stable radix sort, so ties
//      keep the original order): perm[new] = old, inv[old] = new;
//   3. write the renumbered in-CSR (rows in new order, entries translated to
//      new ids, original entry order kept) and, for directed graphs, the
//      out-degrees and the renumbered out-CSR the adjoint gathers over;
//   4. weighted graphs: per-row out-weight sums S_v, the in-edge weights
//      aligned with the renumbered in-CSR (looked up by binary search in the
//      sorted out-rows), and the out-edge weights aligned with the
//      renumbered out-rows;
//   5. vertex bins: the first row of each length class, and the segment
//      table of the hub rows.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "internal.h"

namespace prgpu {

namespace {

enum : unsigned {
  kBadOffsetStart = 1u,
  kBadOffsetEnd = 2u,
  kBadOffsetOrder = 4u,
  kBadId = 8u,
  kBadWeight = 16u,
  kUnsortedRow = 32u,
};

__global__ void validate_offsets_kernel(int64_t n, int64_t m, const int32_t *off,
                                        unsigned *flag) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i > n) return;
  const int32_t o = off[i];
  if (i == 0 && o != 0) atomicOr(flag, kBadOffsetStart);
  if (i == n && o != m) atomicOr(flag, kBadOffsetEnd);
  if (i < n && o > off[i + 1]) atomicOr(flag, kBadOffsetOrder);
}

__global__ void validate_ids_kernel(int64_t m, int64_t n, const int32_t *nbr,
                                    unsigned *flag) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int32_t v = nbr[i];
  if (v < 0 || v >= n) atomicOr(flag, kBadId);
}

__global__ void validate_weights_kernel(int64_t m, const float *w, unsigned *flag) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const float x = w[i];
  if (!(x > 0.f) || !isfinite(x)) atomicOr(flag, kBadWeight);
}

// Out-rows must be strictly increasing for the weight lookup.
__global__ void validate_sorted_kernel(int64_t n, const int32_t *off, const int32_t *nbr,
                                       unsigned *flag) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= n) return;
  for (int32_t e = off[v] + 1; e < off[v + 1]; e++)
    if (nbr[e - 1] >= nbr[e]) {
      atomicOr(flag, kUnsortedRow);
      return;
    }
}

__global__ void degree_kernel(int64_t n, const int32_t *off, uint32_t *deg, int32_t *ids) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= n) return;
  deg[v] = static_cast<uint32_t>(off[v + 1] - off[v]);
  ids[v] = static_cast<int32_t>(v);
}

__global__ void invert_kernel(int64_t n, const int32_t *perm, int32_t *inv) {
  const int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u >= n) return;
  inv[perm[u]] = static_cast<int32_t>(u);
}

__global__ void set_last_kernel(int32_t *p, int64_t idx, int32_t value) { p[idx] = value; }

// One warp per renumbered row: copy the row of perm[u] from the source CSR,
// translating ids through inv (translate == nullptr copies them unchanged).
__global__ void renumber_rows_kernel(int64_t n, const int32_t *__restrict__ perm,
                                     const int32_t *__restrict__ src_off,
                                     const int32_t *__restrict__ src_nbr,
                                     const int32_t *__restrict__ dst_off,
                                     const int32_t *__restrict__ translate,
                                     int32_t *dst_nbr, const float *__restrict__ src_w,
                                     float *dst_w, int32_t *dst_pos) {
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int32_t v = perm[warp];
  const int32_t s = src_off[v], len = src_off[v + 1] - s;
  const int32_t d = dst_off[warp];
  for (int32_t j = lane; j < len; j += 32) {
    if (dst_nbr) {
      const int32_t x = src_nbr[s + j];
      dst_nbr[d + j] = translate ? translate[x] : x;
    }
    if (dst_w) dst_w[d + j] = src_w[s + j];
    if (dst_pos) dst_pos[d + j] = s + j;
  }
}

__global__ void out_degree_kernel(int64_t n, const int32_t *perm, const int32_t *out_off,
                                  int32_t *odeg) {
  const int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const int32_t v = perm[u];
  odeg[u] = out_off[v + 1] - out_off[v];
}

// S_v per renumbered vertex, summed in double in row order then rounded.
__global__ void row_weight_sum_kernel(int64_t n, const int32_t *perm, const int32_t *out_off,
                                      const float *ew, float *rsum) {
  const int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const int32_t v = perm[u];
  double acc = 0;
  for (int32_t e = out_off[v]; e < out_off[v + 1]; e++) acc += ew[e];
  rsum[u] = static_cast<float>(acc);
}

// In-edge weights aligned with the renumbered in-CSR: entry j of new row u is
// the in-edge x -> perm[u]; its weight sits at the position of perm[u] in
// x's (sorted) out-row.
__global__ void in_weight_kernel(int64_t n, const int32_t *__restrict__ perm,
                                 const int32_t *__restrict__ in_off,
                                 const int32_t *__restrict__ in_nbr,
                                 const int32_t *__restrict__ out_off,
                                 const int32_t *__restrict__ out_nbr,
                                 const float *__restrict__ ew,
                                 const int32_t *__restrict__ rowoff, float *win,
                                 int32_t *win_pos, unsigned *flag) {
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int32_t v = perm[warp];
  const int32_t s = in_off[v], len = in_off[v + 1] - s;
  const int32_t d = rowoff[warp];
  for (int32_t j = lane; j < len; j += 32) {
    const int32_t x = in_nbr[s + j];
    int32_t lo = out_off[x], hi = out_off[x + 1];
    while (lo < hi) {
      const int32_t mid = lo + ((hi - lo) >> 1);
      if (out_nbr[mid] < v) lo = mid + 1; else hi = mid;
    }
    if (lo < out_off[x + 1] && out_nbr[lo] == v) {
      win[d + j] = ew[lo];
      win_pos[d + j] = lo;
    } else {
      win[d + j] = 0.f;
      win_pos[d + j] = -1;
      atomicOr(flag, kBadOffsetOrder);  // in/out CSRs disagree
    }
  }
}

// Rows of the renumbered CSR are sorted by descending length, so the first
// row shorter than a threshold is a lower bound; one thread does all bins.
__global__ void bin_bounds_kernel(int64_t n, const uint32_t *deg_sorted, BinConfig cfg,
                                  int64_t *out_start) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  out_start[0] = 0;
  for (int b = 0; b + 1 < kNumBins; b++) {
    const uint32_t t = static_cast<uint32_t>(cfg.min_len[b]);
    int64_t lo = 0, hi = n;  // first index with deg < t
    while (lo < hi) {
      const int64_t mid = lo + ((hi - lo) >> 1);
      if (deg_sorted[mid] >= t) lo = mid + 1; else hi = mid;
    }
    out_start[b + 1] = lo;
  }
  out_start[kNumBins] = n;
}

inline unsigned Blocks(int64_t count, int threads) {
  return static_cast<unsigned>((count + threads - 1) / threads);
}

// win[j] = w[win_pos[j]] over the renumbered in-CSR entries.
__global__ void gather_weights_kernel(int64_t m, const int32_t *__restrict__ pos,
                                      const float *__restrict__ w, float *out) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int32_t p = pos[j];
  out[j] = p >= 0 ? w[p] : 0.f;
}

std::string FlagText(unsigned f) {
  std::string s;
  if (f & kBadOffsetStart) s += " offsets[0] != 0;";
  if (f & kBadOffsetEnd) s += " offsets[n] != m;";
  if (f & kBadOffsetOrder) s += " offsets not monotone or in/out CSRs disagree;";
  if (f & kBadId) s += " neighbour id outside [0, n);";
  if (f & kBadWeight) s += " edge weight not finite and positive;";
  if (f & kUnsortedRow) s += " weighted graphs need strictly increasing out-rows;";
  return s;
}

template <typename T>
cudaError_t Alloc(T **p, int64_t count) {
  *p = nullptr;
  if (count <= 0) count = 1;
  return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * static_cast<size_t>(count));
}

}  // namespace

void FreeDeviceGraph(DeviceGraph *g) {
  void *ptrs[] = {g->rowoff, g->col, g->win, g->win_pos, g->odeg, g->rsum, g->orowoff, g->ocol,
                  g->wout, g->orig_out_off, g->perm, g->inv, g->seg_row, g->seg_first, g->hub_ticket,
                  g->seg_partial};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  BinConfig keep = g->bins;
  *g = DeviceGraph();
  g->bins = keep;
}

#define PR_TRY(expr)                       \
  do {                                     \
    cudaError_t e_ = (expr);               \
    if (e_ != cudaSuccess) {               \
      *err = std::string(#expr) + ": " + cudaGetErrorString(e_); \
      cleanup();                           \
      return e_;                           \
    }                                      \
  } while (0)

cudaError_t BuildDeviceGraph(DeviceGraph *g, int64_t n, int64_t m,
                             const int32_t *d_out_off, const int32_t *d_out_nbr,
                             const int32_t *d_in_off, const int32_t *d_in_nbr,
                             const float *d_ew, bool directed, cudaStream_t s,
                             std::string *err) {
  FreeDeviceGraph(g);
  g->n = n;
  g->m = m;
  g->directed = directed;
  g->weighted = d_ew != nullptr;
  unsigned *d_flag = nullptr;
  uint32_t *deg = nullptr, *deg_sorted = nullptr;
  int32_t *ids = nullptr;
  void *tmp = nullptr;
  int64_t *d_bins = nullptr;
  auto cleanup = [&]() {
    if (d_flag) cudaFree(d_flag);
    if (deg) cudaFree(deg);
    if (deg_sorted) cudaFree(deg_sorted);
    if (ids) cudaFree(ids);
    if (tmp) cudaFree(tmp);
    if (d_bins) cudaFree(d_bins);
    d_flag = nullptr; deg = deg_sorted = nullptr; ids = nullptr; tmp = nullptr; d_bins = nullptr;
  };
  const int T = 256;
  PR_TRY(Alloc(&d_flag, 1));
  PR_TRY(cudaMemsetAsync(d_flag, 0, sizeof(unsigned), s));

  // 1. validation
  validate_offsets_kernel<<<Blocks(n + 1, T), T, 0, s>>>(n, m, d_in_off, d_flag);
  if (m) validate_ids_kernel<<<Blocks(m, T), T, 0, s>>>(m, n, d_in_nbr, d_flag);
  if (directed) {
    validate_offsets_kernel<<<Blocks(n + 1, T), T, 0, s>>>(n, m, d_out_off, d_flag);
    if (m) validate_ids_kernel<<<Blocks(m, T), T, 0, s>>>(m, n, d_out_nbr, d_flag);
  }
  if (g->weighted) {
    if (m) validate_weights_kernel<<<Blocks(m, T), T, 0, s>>>(m, d_ew, d_flag);
    validate_sorted_kernel<<<Blocks(n, T), T, 0, s>>>(n, d_out_off, d_out_nbr, d_flag);
  }
  PR_TRY(cudaGetLastError());
  unsigned flag = 0;
  PR_TRY(cudaMemcpyAsync(&flag, d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  PR_TRY(cudaStreamSynchronize(s));
  if (flag) {
    *err = "invalid CSR:" + FlagText(flag);
    cleanup();
    FreeDeviceGraph(g);
    return cudaErrorInvalidValue;
  }

  // 2. degree order
  PR_TRY(Alloc(&deg, n));
  PR_TRY(Alloc(&deg_sorted, n));
  PR_TRY(Alloc(&ids, n));
  PR_TRY(Alloc(&g->perm, n));
  PR_TRY(Alloc(&g->inv, n));
  degree_kernel<<<Blocks(n, T), T, 0, s>>>(n, d_in_off, deg, ids);
  size_t tmp_bytes = 0, scan_bytes = 0;
  PR_TRY(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, deg, deg_sorted, ids,
                                                   g->perm, static_cast<int>(n), 0, 32, s));
  PR_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, deg_sorted,
                                       reinterpret_cast<int32_t *>(ids), static_cast<int>(n), s));
  tmp_bytes = std::max(tmp_bytes, scan_bytes);
  PR_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, reinterpret_cast<int32_t *>(deg),
                                       reinterpret_cast<int32_t *>(ids), static_cast<int>(n), s));
  tmp_bytes = std::max(tmp_bytes, scan_bytes);
  PR_TRY(cudaMalloc(&tmp, tmp_bytes));
  PR_TRY(cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_bytes, deg, deg_sorted, ids,
                                                   g->perm, static_cast<int>(n), 0, 32, s));
  invert_kernel<<<Blocks(n, T), T, 0, s>>>(n, g->perm, g->inv);
  uint32_t maxdeg = 0;
  if (n) PR_TRY(cudaMemcpyAsync(&maxdeg, deg_sorted, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));

  // 3. renumbered in-CSR
  PR_TRY(Alloc(&g->rowoff, n + 1));
  PR_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, deg_sorted, g->rowoff,
                                       static_cast<int>(n), s));
  set_last_kernel<<<1, 1, 0, s>>>(g->rowoff, n, static_cast<int32_t>(m));
  const int64_t m_pad = ((m + 3) / 4) * 4 + 4;
  PR_TRY(Alloc(&g->col, m_pad));
  PR_TRY(cudaMemsetAsync(g->col, 0, sizeof(int32_t) * m_pad, s));
  renumber_rows_kernel<<<Blocks(n * 32, T), T, 0, s>>>(n, g->perm, d_in_off, d_in_nbr, g->rowoff,
                                                       g->inv, g->col, nullptr, nullptr, nullptr);
  PR_TRY(cudaGetLastError());

  if (directed) {
    PR_TRY(Alloc(&g->odeg, n));
    out_degree_kernel<<<Blocks(n, T), T, 0, s>>>(n, g->perm, d_out_off, g->odeg);
    PR_TRY(Alloc(&g->orowoff, n + 1));
    PR_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, g->odeg, g->orowoff,
                                         static_cast<int>(n), s));
    set_last_kernel<<<1, 1, 0, s>>>(g->orowoff, n, static_cast<int32_t>(m));
    PR_TRY(Alloc(&g->ocol, m_pad));
    PR_TRY(cudaMemsetAsync(g->ocol, 0, sizeof(int32_t) * m_pad, s));
    renumber_rows_kernel<<<Blocks(n * 32, T), T, 0, s>>>(n, g->perm, d_out_off, d_out_nbr,
                                                         g->orowoff, g->inv, g->ocol, nullptr,
                                                         nullptr, nullptr);
    PR_TRY(cudaGetLastError());
  }

  // 4. weights
  if (g->weighted) {
    PR_TRY(Alloc(&g->rsum, n));
    row_weight_sum_kernel<<<Blocks(n, T), T, 0, s>>>(n, g->perm, d_out_off, d_ew, g->rsum);
    PR_TRY(Alloc(&g->win, m_pad));
    PR_TRY(cudaMemsetAsync(g->win, 0, sizeof(float) * m_pad, s));
    PR_TRY(Alloc(&g->win_pos, m_pad));
    in_weight_kernel<<<Blocks(n * 32, T), T, 0, s>>>(n, g->perm, d_in_off, d_in_nbr, d_out_off,
                                                     d_out_nbr, d_ew, g->rowoff, g->win,
                                                     g->win_pos, d_flag);
    const int32_t *oro = directed ? g->orowoff : g->rowoff;
    PR_TRY(Alloc(&g->wout, m_pad));
    PR_TRY(cudaMemsetAsync(g->wout, 0, sizeof(float) * m_pad, s));
    renumber_rows_kernel<<<Blocks(n * 32, T), T, 0, s>>>(n, g->perm, d_out_off, d_out_nbr, oro,
                                                         g->inv, nullptr, d_ew, g->wout,
                                                         nullptr);
    PR_TRY(cudaGetLastError());
    PR_TRY(cudaMemcpyAsync(&flag, d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  }

  PR_TRY(Alloc(&g->orig_out_off, n + 1));
  PR_TRY(cudaMemcpyAsync(g->orig_out_off, d_out_off, sizeof(int32_t) * (n + 1),
                         cudaMemcpyDeviceToDevice, s));

  // 5. bins and hub segments
  PR_TRY(Alloc(&d_bins, kNumBins + 1));
  bin_bounds_kernel<<<1, 32, 0, s>>>(n, deg_sorted, g->bins, d_bins);
  PR_TRY(cudaMemcpyAsync(g->bin_row_start, d_bins, sizeof(int64_t) * (kNumBins + 1),
                         cudaMemcpyDeviceToHost, s));
  PR_TRY(cudaStreamSynchronize(s));
  if (flag) {
    *err = "invalid CSR:" + FlagText(flag);
    cleanup();
    FreeDeviceGraph(g);
    return cudaErrorInvalidValue;
  }
  g->max_degree = maxdeg;
  const int64_t H = g->bin_row_start[1];
  g->num_hub_rows = H;
  std::vector<uint32_t> hub_len(H);
  if (H)
    PR_TRY(cudaMemcpy(hub_len.data(), deg_sorted, sizeof(uint32_t) * H, cudaMemcpyDeviceToHost));
  std::vector<int32_t> seg_first(H + 1), seg_row;
  int64_t nseg = 0;
  for (int64_t r = 0; r < H; r++) {
    seg_first[r] = static_cast<int32_t>(nseg);
    const int64_t k = (static_cast<int64_t>(hub_len[r]) + kSegEntries - 1) / kSegEntries;
    for (int64_t j = 0; j < k; j++) seg_row.push_back(static_cast<int32_t>(r));
    nseg += k;
  }
  seg_first[H] = static_cast<int32_t>(nseg);
  g->num_segments = nseg;
  PR_TRY(Alloc(&g->seg_first, H + 1));
  PR_TRY(Alloc(&g->seg_row, nseg));
  PR_TRY(Alloc(&g->hub_ticket, H));
  PR_TRY(Alloc(&g->seg_partial, nseg));
  PR_TRY(cudaMemcpy(g->seg_first, seg_first.data(), sizeof(int32_t) * (H + 1),
                    cudaMemcpyHostToDevice));
  if (nseg)
    PR_TRY(cudaMemcpy(g->seg_row, seg_row.data(), sizeof(int32_t) * nseg, cudaMemcpyHostToDevice));
  PR_TRY(cudaMemsetAsync(g->hub_ticket, 0, sizeof(unsigned) * std::max<int64_t>(H, 1), s));
  PR_TRY(cudaStreamSynchronize(s));
  cleanup();
  return cudaSuccess;
}

cudaError_t UpdateDeviceWeights(DeviceGraph *g, const float *d_w, cudaStream_t s,
                                std::string *err) {
  if (!g->weighted || !g->win_pos) {
    *err = "the graph on the device has no edge weights";
    return cudaErrorInvalidValue;
  }
  const int64_t n = g->n, m = g->m;
  const int T = 256;
  unsigned *d_flag = nullptr;
  auto cleanup = [&]() {
    if (d_flag) cudaFree(d_flag);
    d_flag = nullptr;
  };
  PR_TRY(Alloc(&d_flag, 1));
  PR_TRY(cudaMemsetAsync(d_flag, 0, sizeof(unsigned), s));
  if (m) validate_weights_kernel<<<Blocks(m, T), T, 0, s>>>(m, d_w, d_flag);
  PR_TRY(cudaGetLastError());
  unsigned flag = 0;
  PR_TRY(cudaMemcpyAsync(&flag, d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  PR_TRY(cudaStreamSynchronize(s));
  if (flag) {
    *err = "invalid edge weights:" + FlagText(flag);
    cleanup();
    return cudaErrorInvalidValue;
  }
  // the same three arrays BuildDeviceGraph derives from the weights
  row_weight_sum_kernel<<<Blocks(n, T), T, 0, s>>>(n, g->perm, g->orig_out_off, d_w, g->rsum);
  if (m) gather_weights_kernel<<<Blocks(m, T), T, 0, s>>>(m, g->win_pos, d_w, g->win);
  const int32_t *oro = g->directed ? g->orowoff : g->rowoff;
  renumber_rows_kernel<<<Blocks(n * 32, T), T, 0, s>>>(n, g->perm, g->orig_out_off, nullptr, oro,
                                                       nullptr, nullptr, d_w, g->wout, nullptr);
  PR_TRY(cudaGetLastError());
  PR_TRY(cudaStreamSynchronize(s));
  cleanup();
  return cudaSuccess;
}

#undef PR_TRY

}  // namespace prgpu
