// bfs.cu -- direction-optimizing breadth-first search on the device CSR
// mirror (pr_gpu_bfs in include/pr_gpu.h).
//
// The reference's DOBFS (src/bfs.cc:38-174), step for step:
//   * parent[v] starts at -out_degree(v) (-1 without out-edges), the source
//     is its own parent;
//   * top-down step: every frontier vertex claims its unvisited
//     out-neighbours by compare-and-swap on parent[], the claimed vertices
//     form the next frontier queue, and the step returns the scout count
//     (the summed out-degrees of the claimed vertices, read back from the
//     negative parents);
//   * bottom-up step: every unvisited vertex takes the first in-neighbour
//     found in the frontier bitmap as its parent, the found vertices form the
//     next bitmap, and the step returns their number;
//   * the same switching rule: top-down while scout_count <= edges_to_check /
//     alpha (edges_to_check starts at M and loses each top-down step's scout
//     count), bottom-up while the awake count grows or stays above N / beta,
//     then back to a queue (alpha = 15, beta = 18);
//   * unvisited vertices end with parent -1.
// The host drives the steps (one small read-back per step for the counts);
// ids are the mirror's degree-sorted ids and are mapped back at the end.
// Parents can differ from run to run (which frontier vertex wins a claim is
// a race, as in the reference); depths, reached sets and tree sizes cannot.
//
// Top-down work is spread over the frontier's edges, not its vertices
// (frontier degrees are scanned, each thread takes edges and finds its
// vertex by binary search), so a hub in the frontier does not serialise a
// warp.  Bottom-up work: each warp owns 32 consecutive vertices and writes
// their bitmap word with one ballot.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#include "internal.h"

namespace prgpu {

namespace {

struct BfsCounters {
  unsigned long long qtail;  // next-frontier queue length
  unsigned long long scout;  // top-down scout count
  unsigned long long awake;  // bottom-up awake count
};

__device__ __forceinline__ int32_t out_degree(const int32_t *ooff, int v) {
  return ooff[v + 1] - ooff[v];
}

// Warp-aggregated append of the flagged lanes' values to queue[] (tail).
__device__ __forceinline__ void warp_append(bool flag, int value, int32_t *queue,
                                            unsigned long long *tail) {
  const unsigned mask = __activemask();
  const unsigned ballot = __ballot_sync(mask, flag);
  if (!ballot) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(ballot) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(tail, static_cast<unsigned long long>(__popc(ballot)));
  base = __shfl_sync(mask, base, leader);
  if (flag) queue[base + __popc(ballot & ((1u << lane) - 1u))] = value;
}

__global__ void bfs_init_kernel(int32_t n, const int32_t *__restrict__ ooff, int src,
                                int32_t *parent, int32_t *queue) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += stride) {
    const int32_t d = out_degree(ooff, static_cast<int>(v));
    parent[v] = (v == src) ? src : (d != 0 ? -d : -1);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) queue[0] = src;
}

// Out-degree of every frontier vertex (input of the edge scan).
__global__ void bfs_frontier_degree_kernel(int64_t q, const int32_t *__restrict__ queue,
                                           const int32_t *__restrict__ ooff, int64_t *deg) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < q; i += stride)
    deg[i] = out_degree(ooff, queue[i]);
}

// Top-down step over the frontier's edges: edge e belongs to the frontier
// vertex i with eoff[i] <= e < eoff[i + 1] (eoff: exclusive scan of degrees).
__global__ void bfs_td_kernel(int64_t q, const int32_t *__restrict__ queue,
                              const int64_t *__restrict__ eoff, const int32_t *__restrict__ ooff,
                              const int32_t *__restrict__ onbr, int32_t *parent, int32_t *next,
                              BfsCounters *cnt) {
  const int64_t edges = eoff[q];  // the scan's total: no host round trip
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  unsigned long long scout = 0;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  // whole warps iterate together so the appends can use warp ballots
  const int64_t rounds = (edges + stride - 1) / stride;
  for (int64_t r = 0; r < rounds; r++) {
    const int64_t e = first + r * stride;
    bool claimed = false;
    int v = 0;
    if (e < edges) {
      int64_t lo = 0, hi = q - 1;  // last i with eoff[i] <= e
      while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (eoff[mid] <= e) lo = mid;
        else hi = mid - 1;
      }
      const int u = queue[lo];
      v = onbr[ooff[u] + (e - eoff[lo])];
      const int32_t cur = *reinterpret_cast<volatile int32_t *>(parent + v);
      if (cur < 0 && atomicCAS(parent + v, cur, u) == cur) {
        claimed = true;
        scout += static_cast<unsigned long long>(-cur);
      }
    }
    warp_append(claimed, v, next, &cnt->qtail);
  }
  for (int o = 16; o > 0; o >>= 1) scout += __shfl_xor_sync(0xffffffffu, scout, o);
  if ((threadIdx.x & 31) == 0 && scout) atomicAdd(&cnt->scout, scout);
}

__global__ void bfs_queue_to_bitmap_kernel(int64_t q, const int32_t *__restrict__ queue,
                                           unsigned *bm) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < q; i += stride) {
    const int v = queue[i];
    atomicOr(bm + (v >> 5), 1u << (v & 31));
  }
}

// Bottom-up step: each warp owns 32 consecutive vertices (one bitmap word).
__global__ void bfs_bu_kernel(int32_t n, const int32_t *__restrict__ ioff,
                              const int32_t *__restrict__ inbr, const unsigned *__restrict__ front,
                              unsigned *next, int32_t *parent, BfsCounters *cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t words = (static_cast<int64_t>(n) + 31) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  unsigned long long awake = 0;
  for (int64_t w = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < words;
       w += warps) {
    const int64_t v = (w << 5) + lane;
    bool found = false;
    if (v < n && parent[v] < 0) {
      for (int j = ioff[v]; j < ioff[v + 1]; j++) {
        const int u = inbr[j];
        if ((__ldg(front + (u >> 5)) >> (u & 31)) & 1u) {
          parent[v] = u;
          found = true;
          break;
        }
      }
    }
    const unsigned word = __ballot_sync(0xffffffffu, found);
    if (lane == 0) next[w] = word;
    awake += found ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) awake += __shfl_xor_sync(0xffffffffu, awake, o);
  if (lane == 0 && awake) atomicAdd(&cnt->awake, awake);
}

__global__ void bfs_bitmap_to_queue_kernel(int32_t n, const unsigned *__restrict__ bm,
                                           int32_t *queue, BfsCounters *cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t words = (static_cast<int64_t>(n) + 31) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t w = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < words;
       w += warps) {
    const unsigned word = bm[w];  // same value in every lane
    const int64_t v = (w << 5) + lane;
    warp_append(((word >> lane) & 1u) != 0u && v < n, static_cast<int>(v), queue, &cnt->qtail);
  }
}

// parent < -1 -> -1, in original ids: each original id gathers its row's
// parent (coalesced writes; a scatter through perm wrote partial sectors).
__global__ void bfs_finish_kernel(int32_t n, const int32_t *__restrict__ parent,
                                  const int32_t *__restrict__ perm,
                                  const int32_t *__restrict__ inv, int32_t *out_old) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += stride) {
    const int32_t p = parent[inv[v]];
    out_old[v] = p >= 0 ? perm[p] : -1;
  }
}

unsigned BfsGrid(int64_t items) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((items + 255) / 256, sms * 16)));
}

}  // namespace

void FreeBfsScratch(BfsScratch *b) {
  void *ptrs[] = {b->parent, b->queue[0], b->queue[1], b->bm[0], b->bm[1], b->deg, b->eoff,
                  b->cnt, b->tmp};
  // (all members are owned by the scratch)
  for (void *p : ptrs)
    if (p) cudaFree(p);
  *b = BfsScratch();
}

#define BFS_TRY(expr)                                                  \
  do {                                                                 \
    cudaError_t e_ = (expr);                                           \
    if (e_ != cudaSuccess) {                                           \
      *err = std::string("bfs: ") + #expr + ": " + cudaGetErrorString(e_); \
      return e_;                                                       \
    }                                                                  \
  } while (0)

cudaError_t BreadthFirstSearch(const DeviceGraph &g, BfsScratch &b, cudaStream_t s,
                               int source_old, int alpha, int beta, int32_t *out_old,
                               std::vector<BfsStep> *steps, std::string *err) {
  const int64_t n = g.n;
  const int64_t words = (n + 31) / 32;
  const int32_t *ooff = g.directed ? g.orowoff : g.rowoff;
  const int32_t *onbr = g.directed ? g.ocol : g.col;
  const int32_t *ioff = g.rowoff;
  const int32_t *inbr = g.col;
  if (!b.parent || b.cap_n < n) {
    FreeBfsScratch(&b);
    BFS_TRY(cudaMalloc(&b.parent, sizeof(int32_t) * std::max<int64_t>(n, 1)));
    BFS_TRY(cudaMalloc(&b.queue[0], sizeof(int32_t) * std::max<int64_t>(n, 1)));
    BFS_TRY(cudaMalloc(&b.queue[1], sizeof(int32_t) * std::max<int64_t>(n, 1)));
    BFS_TRY(cudaMalloc(&b.deg, sizeof(int64_t) * (n + 1)));
    BFS_TRY(cudaMalloc(&b.eoff, sizeof(int64_t) * (n + 1)));
    BFS_TRY(cudaMalloc(&b.bm[0], sizeof(unsigned) * std::max<int64_t>(words, 1)));
    BFS_TRY(cudaMalloc(&b.bm[1], sizeof(unsigned) * std::max<int64_t>(words, 1)));
    b.cap_n = n;
  }
  if (!b.cnt) BFS_TRY(cudaMalloc(&b.cnt, sizeof(BfsCounters)));
  BfsCounters *const cnt = static_cast<BfsCounters *>(b.cnt);
  size_t scan_bytes = 0;
  BFS_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, b.deg, b.eoff, static_cast<int>(n + 1),
                                        s));
  if (!b.tmp || b.cap_tmp < static_cast<int64_t>(scan_bytes)) {
    if (b.tmp) cudaFree(b.tmp);
    b.tmp = nullptr;
    b.cap_tmp = 0;
    BFS_TRY(cudaMalloc(&b.tmp, std::max<size_t>(scan_bytes, 1)));
    b.cap_tmp = static_cast<int64_t>(scan_bytes);
  }

  using clock = std::chrono::steady_clock;
  auto seconds = [](clock::time_point a, clock::time_point z) {
    return std::chrono::duration<double>(z - a).count();
  };
  auto record = [&](const char *kind, int64_t count, double sec) {
    if (steps) steps->push_back(BfsStep{kind, count, sec});
  };
  auto t0 = clock::now();
  int32_t src = 0;
  BFS_TRY(cudaMemcpyAsync(&src, g.inv + source_old, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BFS_TRY(cudaStreamSynchronize(s));
  const unsigned grid = BfsGrid(n);
  bfs_init_kernel<<<grid, 256, 0, s>>>(static_cast<int32_t>(n), ooff, src, b.parent, b.queue[0]);
  BFS_TRY(cudaGetLastError());
  int32_t src_off[2] = {0, 0};
  BFS_TRY(cudaMemcpyAsync(src_off, ooff + src, sizeof(src_off), cudaMemcpyDeviceToHost, s));
  BFS_TRY(cudaStreamSynchronize(s));
  record("i", -1, seconds(t0, clock::now()));

  BfsCounters hc{};
  auto read_counters = [&]() -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(&hc, b.cnt, sizeof(hc), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
  };
  int cur = 0;                // queue[cur] is the frontier
  int64_t qsize = 1;
  int64_t edges_to_check = g.m;
  int64_t scout_count = src_off[1] - src_off[0];
  // every step reaches at least one new vertex, so n + 2 steps bound the
  // search; the guard turns a defect into an error instead of a host loop
  int64_t guard = 0;
  while (qsize > 0) {
    if (++guard > n + 2) {
      *err = "bfs: step limit exceeded";
      return cudaErrorUnknown;
    }
    if (scout_count > edges_to_check / alpha) {
      auto ts = clock::now();
      BFS_TRY(cudaMemsetAsync(b.bm[0], 0, sizeof(unsigned) * words, s));
      bfs_queue_to_bitmap_kernel<<<BfsGrid(qsize), 256, 0, s>>>(qsize, b.queue[cur], b.bm[0]);
      BFS_TRY(cudaGetLastError());
      BFS_TRY(cudaStreamSynchronize(s));
      record("e", -1, seconds(ts, clock::now()));
      int front = 0;
      int64_t awake = qsize, old_awake = 0;
      do {
        ts = clock::now();
        old_awake = awake;
        BFS_TRY(cudaMemsetAsync(b.cnt, 0, sizeof(BfsCounters), s));
        bfs_bu_kernel<<<BfsGrid(words * 32), 256, 0, s>>>(static_cast<int32_t>(n), ioff, inbr,
                                                          b.bm[front], b.bm[front ^ 1], b.parent,
                                                          cnt);
        BFS_TRY(cudaGetLastError());
        BFS_TRY(read_counters());
        awake = static_cast<int64_t>(hc.awake);
        front ^= 1;
        record("bu", awake, seconds(ts, clock::now()));
        if (++guard > n + 2) {
          *err = "bfs: step limit exceeded";
          return cudaErrorUnknown;
        }
      } while (awake >= old_awake || awake > n / beta);
      ts = clock::now();
      BFS_TRY(cudaMemsetAsync(b.cnt, 0, sizeof(BfsCounters), s));
      bfs_bitmap_to_queue_kernel<<<BfsGrid(words * 32), 256, 0, s>>>(
          static_cast<int32_t>(n), b.bm[front], b.queue[cur], cnt);
      BFS_TRY(cudaGetLastError());
      BFS_TRY(read_counters());
      qsize = static_cast<int64_t>(hc.qtail);
      record("c", -1, seconds(ts, clock::now()));
      scout_count = 1;
    } else {
      auto ts = clock::now();
      edges_to_check -= scout_count;
      bfs_frontier_degree_kernel<<<BfsGrid(qsize), 256, 0, s>>>(qsize, b.queue[cur], ooff, b.deg);
      BFS_TRY(cudaGetLastError());
      BFS_TRY(cudaMemsetAsync(b.deg + qsize, 0, sizeof(int64_t), s));
      size_t bytes = static_cast<size_t>(b.cap_tmp);
      BFS_TRY(cub::DeviceScan::ExclusiveSum(b.tmp, bytes, b.deg, b.eoff, static_cast<int>(qsize + 1),
                                            s));
      BFS_TRY(cudaMemsetAsync(b.cnt, 0, sizeof(BfsCounters), s));
      // grid sized by the largest edge count the frontier can have
      bfs_td_kernel<<<BfsGrid(std::min<int64_t>(g.m, qsize * g.max_degree)), 256, 0, s>>>(
          qsize, b.queue[cur], b.eoff, ooff, onbr, b.parent, b.queue[cur ^ 1], cnt);
      BFS_TRY(cudaGetLastError());
      BFS_TRY(read_counters());
      scout_count = static_cast<int64_t>(hc.scout);
      qsize = static_cast<int64_t>(hc.qtail);
      cur ^= 1;
      record("td", qsize, seconds(ts, clock::now()));
    }
  }
  bfs_finish_kernel<<<grid, 256, 0, s>>>(static_cast<int32_t>(n), b.parent, g.perm, g.inv,
                                         out_old);
  BFS_TRY(cudaGetLastError());
  BFS_TRY(cudaStreamSynchronize(s));
  return cudaSuccess;
}

#undef BFS_TRY

}  // namespace prgpu
