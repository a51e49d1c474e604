// generate.cu -- the reference's synthetic graphs built on the device
// (pr_gpu_generate / pr_gpu_download_csr in include/pr_gpu.h).
//
// Edge generation follows the reference's streams exactly
// (src/generator.h:105-155): edges come in blocks of 2^18, block b drawn from
// its own std::mt19937 seeded kRandSeed + b.  R-MAT edges take one 32-bit
// draw per level (quadrant thresholds 0.57/0.19/0.19 of 2^32); uniform edges
// take two draws reduced modulo 2^scale.  R-MAT ids are then relabelled
// through the reference's seeded permutation (std::shuffle, computed on the
// host and passed in).  The edge list is symmetrised and squished (rows
// sorted, duplicates and self-loops removed; src/builder.h:141-170,300-315)
// by one radix sort of (row, column) keys, so the CSR is the reference's CSR
// bit for bit; N is the largest id plus one (src/builder.h:322-323).
//
// One warp owns one 2^18-edge block and its generator.  MT19937 (Matsumoto
// and Nishimura, 1998): 624-word state; a twist regenerates all 624 words,
// word k from words k, k+1 and k+397 (mod 624), and each output is the
// tempered state word.  The warp runs a twist as three dependency-free
// ranges ([0,227) reads only old words; [227,454) reads new words of the
// first range; [454,623) new words of the second) plus word 623, 32 words at
// a time, then tempers into a ring of draws that its lanes consume, one edge
// per lane.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "internal.h"
#include "pr_gpu.h"

namespace prgpu {

namespace {

constexpr int64_t kGenBlockEdges = int64_t(1) << 18;
constexpr uint32_t kGenSeed = 27491095u;  // the reference's kRandSeed (src/util.h)
constexpr int kMtN = 624;
constexpr int kMtM = 397;
constexpr uint32_t kMtMatrixA = 0x9908b0dfu;
constexpr uint32_t kMtUpper = 0x80000000u;
constexpr uint32_t kMtLower = 0x7fffffffu;
constexpr int kRing = 2048;  // draws buffered per warp (>= 32 * 30 + 624)
constexpr int kGenWarps = 4;

__device__ __forceinline__ uint32_t mt_mix(uint32_t cur, uint32_t next, uint32_t far) {
  const uint32_t y = (cur & kMtUpper) | (next & kMtLower);
  return far ^ (y >> 1) ^ ((y & 1u) ? kMtMatrixA : 0u);
}

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

// Regenerates the warp's state x[0..624) in place.
__device__ void mt_twist(uint32_t *x, int lane) {
  // words [lo, hi), word k from x[k], x[k+1] and x[k + off]; within a chunk
  // every lane reads before any lane writes
  auto range = [&](int lo, int hi, int off) {
    for (int base = lo; base < hi; base += 32) {
      const int k = base + lane;
      uint32_t v = 0;
      if (k < hi) v = mt_mix(x[k], x[k + 1], x[k + off]);
      __syncwarp();
      if (k < hi) x[k] = v;
      __syncwarp();
    }
  };
  range(0, kMtN - kMtM, kMtM);
  range(kMtN - kMtM, 2 * (kMtN - kMtM), kMtM - kMtN);
  range(2 * (kMtN - kMtM), kMtN - 1, kMtM - kMtN);
  if (lane == 0) x[kMtN - 1] = mt_mix(x[kMtN - 1], x[0], x[kMtM - 1]);
  __syncwarp();
}

// Edges of the reference's generators.  D = draws per edge (scale for
// R-MAT, 2 for uniform).
template <bool RMAT>
__global__ void __launch_bounds__(kGenWarps * 32)
    gen_edges_kernel(int scale, int64_t m, uint32_t A, uint32_t AB, uint32_t ABC, int32_t *eu,
                     int32_t *ev) {
  __shared__ uint32_t s_state[kGenWarps][kMtN];
  __shared__ uint32_t s_ring[kGenWarps][kRing];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t b = static_cast<int64_t>(blockIdx.x) * kGenWarps + warp;
  const int64_t nblocks = (m + kGenBlockEdges - 1) / kGenBlockEdges;
  if (b >= nblocks) return;  // whole warp
  uint32_t *x = s_state[warp];
  uint32_t *ring = s_ring[warp];
  if (lane == 0) {
    uint32_t v = kGenSeed + static_cast<uint32_t>(b);
    x[0] = v;
    for (int i = 1; i < kMtN; i++) {
      v = 1812433253u * (v ^ (v >> 30)) + static_cast<uint32_t>(i);
      x[i] = v;
    }
  }
  __syncwarp();
  const int D = RMAT ? scale : 2;
  const int64_t lo = b * kGenBlockEdges;
  const int64_t hi = min(lo + kGenBlockEdges, m);
  int64_t produced = 0, consumed = 0;
  const uint32_t mask = (scale >= 32) ? 0xffffffffu : ((1u << scale) - 1u);
  for (int64_t e0 = lo; e0 < hi; e0 += 32) {
    const int cnt = static_cast<int>(hi - e0 < 32 ? hi - e0 : 32);
    while (produced - consumed < static_cast<int64_t>(cnt) * D) {
      mt_twist(x, lane);
      for (int i = lane; i < kMtN; i += 32)
        ring[(produced + i) & (kRing - 1)] = mt_temper(x[i]);
      __syncwarp();
      produced += kMtN;
    }
    if (lane < cnt) {
      const int64_t at = consumed + static_cast<int64_t>(lane) * D;
      uint32_t s = 0, d = 0;
      if (RMAT) {
        for (int t = 0; t < D; t++) {
          const uint32_t r = ring[(at + t) & (kRing - 1)];
          s <<= 1;
          d <<= 1;
          if (r < AB) {
            d += (r > A) ? 1u : 0u;
          } else {
            s += 1u;
            d += (r > ABC) ? 1u : 0u;
          }
        }
      } else {
        // the two draws of an edge; the reference stores the second as the
        // source (the order is immaterial once symmetrised)
        d = ring[at & (kRing - 1)] & mask;
        s = ring[(at + 1) & (kRing - 1)] & mask;
      }
      eu[e0 + lane] = static_cast<int32_t>(s);
      ev[e0 + lane] = static_cast<int32_t>(d);
    }
    __syncwarp();
    consumed += static_cast<int64_t>(cnt) * D;
  }
}

// Relabels (R-MAT) and expands every edge into both directions as sortable
// (row << 32 | column) keys; records the largest id.
__global__ void expand_keys_kernel(int64_t m, const int32_t *__restrict__ perm,
                                   const int32_t *__restrict__ eu, const int32_t *__restrict__ ev,
                                   uint64_t *__restrict__ keys, int *max_id) {
  int local = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < m; e += stride) {
    uint32_t a = static_cast<uint32_t>(eu[e]), b = static_cast<uint32_t>(ev[e]);
    if (perm) {
      a = static_cast<uint32_t>(perm[a]);
      b = static_cast<uint32_t>(perm[b]);
    }
    keys[2 * e] = (static_cast<uint64_t>(a) << 32) | b;
    keys[2 * e + 1] = (static_cast<uint64_t>(b) << 32) | a;
    local = max(local, static_cast<int>(max(a, b)));
  }
  for (int o = 16; o > 0; o >>= 1) local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
  if ((threadIdx.x & 31) == 0) atomicMax(max_id, local);
}

// Keeps the first key of every run that is not a self-loop.
__global__ void squish_flags_kernel(int64_t k, const uint64_t *__restrict__ keys,
                                    uint8_t *__restrict__ flags) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < k; i += stride) {
    const uint64_t key = keys[i];
    const bool first = (i == 0) || keys[i - 1] != key;
    const bool self = (key >> 32) == (key & 0xffffffffull);
    flags[i] = (first && !self) ? 1 : 0;
  }
}

// Neighbour ids of the kept keys and the length of every row.
__global__ void split_keys_kernel(int64_t k, const uint64_t *__restrict__ kept,
                                  int32_t *__restrict__ nbr, int32_t *__restrict__ rowlen) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < k; i += stride) {
    const uint64_t key = kept[i];
    nbr[i] = static_cast<int32_t>(key & 0xffffffffull);
    atomicAdd(rowlen + (key >> 32), 1);
  }
}

__global__ void widen_offsets_kernel(int64_t n1, const int32_t *__restrict__ off32,
                                     int64_t *__restrict__ off64) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n1; i += stride)
    off64[i] = off32[i];
}

unsigned GridFor(int64_t items) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((items + 255) / 256, sms * 8)));
}

#define GEN_TRY(expr)                                                  \
  do {                                                                 \
    cudaError_t e_ = (expr);                                           \
    if (e_ != cudaSuccess) {                                           \
      *err = std::string(#expr) + ": " + cudaGetErrorString(e_);       \
      return e_;                                                       \
    }                                                                  \
  } while (0)

// Device buffers freed on every exit path.
struct DevBufs {
  std::vector<void *> ptrs;
  template <typename T>
  cudaError_t Alloc(T **p, int64_t count) {
    *p = nullptr;
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<int64_t>(count, 1));
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
  void Release(void *p) {
    auto it = std::find(ptrs.begin(), ptrs.end(), p);
    if (it != ptrs.end()) {
      cudaFree(*it);
      ptrs.erase(it);
    }
  }
  void Keep(void *p) {
    auto it = std::find(ptrs.begin(), ptrs.end(), p);
    if (it != ptrs.end()) ptrs.erase(it);
  }
  ~DevBufs() {
    for (void *p : ptrs) cudaFree(p);
  }
};

}  // namespace

cudaError_t GenerateGraph(bool uniform, int scale, int degree, const int32_t *perm_host,
                          cudaStream_t s, int64_t *n_out, int64_t *m_out, int32_t **off_out,
                          int32_t **nbr_out, std::string *err) {
  const int64_t ngen = int64_t(1) << scale;
  const int64_t m = ngen * degree;  // generated edges
  DevBufs bufs;
  int32_t *eu = nullptr, *ev = nullptr, *perm = nullptr;
  GEN_TRY(bufs.Alloc(&eu, m));
  GEN_TRY(bufs.Alloc(&ev, m));
  const uint32_t top = 0xffffffffu;
  const uint32_t A = static_cast<uint32_t>(0.57 * top);
  const uint32_t B = static_cast<uint32_t>(0.19 * top);
  const uint32_t C = static_cast<uint32_t>(0.19 * top);
  const int64_t nblocks = (m + kGenBlockEdges - 1) / kGenBlockEdges;
  const unsigned gblocks = static_cast<unsigned>((nblocks + kGenWarps - 1) / kGenWarps);
  if (m > 0) {
    if (uniform)
      gen_edges_kernel<false><<<gblocks, kGenWarps * 32, 0, s>>>(scale, m, A, A + B, A + B + C, eu, ev);
    else
      gen_edges_kernel<true><<<gblocks, kGenWarps * 32, 0, s>>>(scale, m, A, A + B, A + B + C, eu, ev);
    GEN_TRY(cudaGetLastError());
  }
  if (!uniform) {
    GEN_TRY(bufs.Alloc(&perm, ngen));
    GEN_TRY(cudaMemcpyAsync(perm, perm_host, sizeof(int32_t) * ngen, cudaMemcpyHostToDevice, s));
  }
  // both directions as (row, column) keys, sorted on the bits in use
  const int64_t k = 2 * m;
  uint64_t *keys = nullptr, *alt = nullptr;
  int *dmax = nullptr;
  GEN_TRY(bufs.Alloc(&keys, k));
  GEN_TRY(bufs.Alloc(&alt, k));
  GEN_TRY(bufs.Alloc(&dmax, 1));
  GEN_TRY(cudaMemsetAsync(dmax, 0, sizeof(int), s));
  if (m > 0) {
    expand_keys_kernel<<<GridFor(m), 256, 0, s>>>(m, perm, eu, ev, keys, dmax);
    GEN_TRY(cudaGetLastError());
  }
  GEN_TRY(cudaStreamSynchronize(s));
  bufs.Release(eu);
  bufs.Release(ev);
  if (perm) bufs.Release(perm);
  int max_id = 0;
  GEN_TRY(cudaMemcpy(&max_id, dmax, sizeof(int), cudaMemcpyDeviceToHost));
  const int64_t n = static_cast<int64_t>(max_id) + 1;
  int64_t kept = 0;
  int32_t *nbr = nullptr, *off = nullptr;
  GEN_TRY(bufs.Alloc(&off, n + 1));
  GEN_TRY(cudaMemsetAsync(off, 0, sizeof(int32_t) * (n + 1), s));
  if (k > 0) {
    cub::DoubleBuffer<uint64_t> db(keys, alt);
    size_t tmp_bytes = 0;
    GEN_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, static_cast<int>(k), 0,
                                           32 + scale, s));
    void *tmp = nullptr;
    uint8_t *flags = nullptr;
    int *dkept = nullptr;
    size_t sel_bytes = 0;
    GEN_TRY(cub::DeviceSelect::Flagged(nullptr, sel_bytes, db.Current(), flags, db.Alternate(),
                                       dkept, static_cast<int>(k), s));
    GEN_TRY(bufs.Alloc(reinterpret_cast<unsigned char **>(&tmp),
                       static_cast<int64_t>(std::max(tmp_bytes, sel_bytes))));
    GEN_TRY(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, static_cast<int>(k), 0, 32 + scale,
                                           s));
    GEN_TRY(bufs.Alloc(&flags, k));
    GEN_TRY(bufs.Alloc(&dkept, 1));
    squish_flags_kernel<<<GridFor(k), 256, 0, s>>>(k, db.Current(), flags);
    GEN_TRY(cudaGetLastError());
    sel_bytes = std::max(tmp_bytes, sel_bytes);
    GEN_TRY(cub::DeviceSelect::Flagged(tmp, sel_bytes, db.Current(), flags, db.Alternate(), dkept,
                                       static_cast<int>(k), s));
    int kept32 = 0;
    GEN_TRY(cudaMemcpyAsync(&kept32, dkept, sizeof(int), cudaMemcpyDeviceToHost, s));
    GEN_TRY(cudaStreamSynchronize(s));
    kept = kept32;
    bufs.Release(flags);
    GEN_TRY(bufs.Alloc(&nbr, kept));
    if (kept > 0) {
      split_keys_kernel<<<GridFor(kept), 256, 0, s>>>(kept, db.Alternate(), nbr, off);
      GEN_TRY(cudaGetLastError());
    }
    // row lengths -> offsets (off[n] stays 0 before the scan, total after)
    size_t scan_bytes = 0;
    GEN_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, off, off, static_cast<int>(n + 1), s));
    if (scan_bytes > std::max(tmp_bytes, sel_bytes)) {
      bufs.Release(tmp);
      GEN_TRY(bufs.Alloc(reinterpret_cast<unsigned char **>(&tmp), static_cast<int64_t>(scan_bytes)));
    }
    GEN_TRY(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, off, off, static_cast<int>(n + 1), s));
    GEN_TRY(cudaStreamSynchronize(s));
  } else {
    GEN_TRY(bufs.Alloc(&nbr, 1));
  }
  bufs.Keep(off);
  bufs.Keep(nbr);
  *off_out = off;
  *nbr_out = nbr;
  *n_out = n;
  *m_out = kept;
  return cudaSuccess;
}

void WidenOffsets(int64_t n1, const int32_t *off32, int64_t *off64, cudaStream_t s) {
  widen_offsets_kernel<<<GridFor(n1), 256, 0, s>>>(n1, off32, off64);
}

namespace {
__global__ void narrow_offsets_kernel(int64_t count, const int64_t *__restrict__ wide,
                                      int32_t *__restrict__ narrow, int *bad) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += stride) {
    const int64_t v = wide[i];
    if (v < 0 || v > 0x7fffffffLL) {
      *bad = 1;
      narrow[i] = 0;
    } else {
      narrow[i] = static_cast<int32_t>(v);
    }
  }
}
}  // namespace

void NarrowOffsets(int64_t count, const int64_t *wide, int32_t *narrow, int *bad, cudaStream_t s) {
  narrow_offsets_kernel<<<GridFor(count), 256, 0, s>>>(count, wide, narrow, bad);
}

#undef GEN_TRY

}  // namespace prgpu
