// bfs.cu -- direction-optimizing breadth-first search on the device CSR
// mirror (pr_gpu_bfs in include/pr_gpu.h).
//
// The reference's DOBFS (src/bfs.cc:38-174), step for step:
//   * the source is its own parent;
//   * top-down step: every frontier vertex claims its unvisited
//     out-neighbours by compare-and-swap on parent[], the claimed vertices
//     form the next frontier queue, and the step returns the scout count
//     (the summed out-degrees of the claimed vertices, 1 for a vertex
//     without out-edges: the reference starts parent[v] at -out_degree(v),
//     or -1, and adds the negated parent it replaced; here unvisited parents
//     are all -1, set by one memset, and the degree is read at the claim);
//   * bottom-up step: every unvisited vertex takes the first in-neighbour
//     found in the frontier bitmap as its parent, the found vertices form the
//     next bitmap, and the step returns their number;
//   * the same switching rule: top-down while scout_count <= edges_to_check /
//     alpha (edges_to_check starts at M and loses each top-down step's scout
//     count), bottom-up while the awake count grows or stays above N / beta,
//     then back to a queue (alpha = 15, beta = 18);
//   * unvisited vertices end with parent -1.
// The host drives the steps (one small read-back per step for the counts);
// queues and bitmaps hold the mirror's degree-sorted ids; parent[] is indexed
// by mirror row but stores the parent's original id, so the write-back only
// gathers it into original order.
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

// The source (original id) becomes its own parent and the first frontier;
// its out-degree is the first scout count.  One thread.  parent[] is indexed
// by mirror row but holds original ids (only its sign is read during the
// search), so the write-back needs no second lookup.
__global__ void bfs_source_kernel(const int32_t *__restrict__ inv, int source_old,
                                  const int32_t *__restrict__ ooff, int32_t *parent,
                                  int32_t *queue, BfsCounters *cnt) {
  const int src = inv[source_old];
  parent[src] = source_old;
  queue[0] = src;
  cnt->qtail = 1;
  cnt->scout = static_cast<unsigned long long>(out_degree(ooff, src));
  cnt->awake = 0;
}

// Block-wide append: every thread holds up to K flagged values (bit k of
// `mask` set: vals[k] is appended).  One global atomic per block reserves
// the block's run of the queue; the block's values land contiguously.  Must
// be called by every thread of the block.
template <int NT, int K>
__device__ __forceinline__ void block_append(unsigned mask, const int (&vals)[K], int32_t *queue,
                                             unsigned long long *tail, unsigned *s_warp,
                                             unsigned long long *s_base) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned mine = __popc(mask);
  unsigned incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned tot = 0;
    for (int w = 0; w < NT / 32; w++) {
      const unsigned t = s_warp[w];
      s_warp[w] = tot;
      tot += t;
    }
    *s_base = tot ? atomicAdd(tail, static_cast<unsigned long long>(tot)) : 0ull;
  }
  __syncthreads();
  unsigned long long pos = *s_base + s_warp[wid] + (incl - mine);
#pragma unroll
  for (int k = 0; k < K; k++)
    if ((mask >> k) & 1u) queue[pos++] = vals[k];
  __syncthreads();  // s_warp / s_base are reused by the next call
}

// Out-degree of every frontier vertex (input of the edge scan).
__global__ void bfs_frontier_degree_kernel(int64_t q, const int32_t *__restrict__ queue,
                                           const int32_t *__restrict__ ooff, int64_t *deg) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < q; i += stride)
    deg[i] = out_degree(ooff, queue[i]);
}

// Top-down step over the frontier's edges: edge e belongs to the frontier
// vertex i with eoff[i] <= e < eoff[i + 1] (eoff: exclusive scan of the
// frontier's out-degrees, eoff[q] = edges).  Each block takes chunks of
// NT * PT consecutive edges; a thread's edges are NT apart, so its
// frontier index only moves forward and is re-searched only when it passes
// the current vertex.  SMALL (q <= NT): every block scans the frontier's
// degrees itself in shared memory, so a small step is one launch.
template <int NT, int PT, bool SMALL>
__global__ void __launch_bounds__(NT)
bfs_td_kernel(int64_t q, const int32_t *__restrict__ queue_g, const int64_t *__restrict__ eoff_g,
              const int32_t *__restrict__ ooff, const int32_t *__restrict__ onbr,
              const int32_t *__restrict__ perm, int32_t *parent, int32_t *next,
              BfsCounters *cnt) {
  __shared__ int64_t s_eoff[SMALL ? NT + 1 : 1];
  __shared__ int32_t s_q[SMALL ? NT : 1];
  __shared__ unsigned s_warp[NT / 32];
  __shared__ unsigned long long s_base;
  const int64_t *eoff = eoff_g;
  const int32_t *queue = queue_g;
  if (SMALL) {
    // exclusive scan of the frontier's out-degrees: warp scans, then the
    // warp totals (s_eoff[NT] ends as the edge count)
    __shared__ int64_t s_wsum[NT / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t u = 0;
    int64_t d = 0;
    if (threadIdx.x < q) {
      u = queue_g[threadIdx.x];
      d = out_degree(ooff, u);
    }
    int64_t incl = d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_wsum[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t run = 0;
      for (int w = 0; w < NT / 32; w++) {
        const int64_t t = s_wsum[w];
        s_wsum[w] = run;
        run += t;
      }
      s_eoff[NT] = run;
    }
    __syncthreads();
    s_eoff[threadIdx.x] = s_wsum[wid] + incl - d;
    s_q[threadIdx.x] = u;
    __syncthreads();
    eoff = s_eoff;
    queue = s_q;
  }
  const int64_t edges = eoff[q];  // the scan's total: no host round trip
  constexpr int64_t kChunk = static_cast<int64_t>(NT) * PT;
  unsigned long long scout = 0;
  int64_t lo = 0;  // frontier index of this thread's previous edge
  for (int64_t c0 = static_cast<int64_t>(blockIdx.x) * kChunk; c0 < edges;
       c0 += static_cast<int64_t>(gridDim.x) * kChunk) {
    int vals[PT];
    unsigned mask = 0;
#pragma unroll
    for (int k = 0; k < PT; k++) {
      const int64_t e = c0 + k * NT + threadIdx.x;
      vals[k] = 0;
      if (e < edges) {
        if (eoff[lo + 1] <= e) {  // past vertex lo: last i with eoff[i] <= e
          int64_t l = lo + 1, h = q - 1;
          while (l < h) {
            const int64_t mid = (l + h + 1) >> 1;
            if (eoff[mid] <= e) l = mid;
            else h = mid - 1;
          }
          lo = l;
        }
        const int u = queue[lo];
        const int v = onbr[ooff[u] + (e - eoff[lo])];
        // a weak load that L1 may serve (the popular targets are hubs read
        // by every block): a parent never returns to -1, so a value >= 0 is
        // final, and a stale -1 only costs a compare-and-swap that fails
        int32_t cur;
        asm volatile("ld.global.ca.s32 %0, [%1];" : "=r"(cur) : "l"(parent + v));
        if (cur < 0 && atomicCAS(parent + v, cur, __ldg(perm + u)) == cur) {
          vals[k] = v;
          mask |= 1u << k;
          scout += static_cast<unsigned long long>(max(out_degree(ooff, v), 1));
        }
      }
    }
    block_append<NT, PT>(mask, vals, next, &cnt->qtail, s_warp, &s_base);
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

__device__ __forceinline__ bool in_front(const unsigned *__restrict__ front, int u) {
  return (__ldg(front + (u >> 5)) >> (u & 31)) & 1u;
}

// Bottom-up step: each warp owns 32 consecutive vertices (one bitmap word).
// Only rows [0, rows) have in-neighbours (rows are sorted by in-degree), so
// only their words are visited; the words after them stay zero.
__global__ void bfs_bu_kernel(int32_t rows, const int32_t *__restrict__ ioff,
                              const int32_t *__restrict__ inbr, const unsigned *__restrict__ front,
                              const int32_t *__restrict__ perm, unsigned *next, int32_t *parent,
                              BfsCounters *cnt) {
  const int32_t n = rows;
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
        if (in_front(front, u)) {
          parent[v] = __ldg(perm + u);
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

// Set bits of the bitmap -> queue, over the words of vertices [0, n).  Each
// thread takes one word per block round and appends its vertices (up to 32)
// with one global atomic per block round.
constexpr int kB2qThreads = 256;

__global__ void __launch_bounds__(kB2qThreads)
bfs_bitmap_to_queue_kernel(int32_t n, const unsigned *__restrict__ bm, int32_t *queue,
                           BfsCounters *cnt) {
  __shared__ unsigned s_warp[kB2qThreads / 32];
  __shared__ unsigned long long s_base;
  const int64_t words = (static_cast<int64_t>(n) + 31) >> 5;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t w0 = static_cast<int64_t>(blockIdx.x) * kB2qThreads; w0 < words;
       w0 += static_cast<int64_t>(gridDim.x) * kB2qThreads) {
    const int64_t w = w0 + threadIdx.x;
    unsigned word = 0;
    if (w < words) {
      word = bm[w];
      const int64_t rest = static_cast<int64_t>(n) - (w << 5);
      if (rest < 32) word &= (1u << rest) - 1u;
    }
    const unsigned mine = __popc(word);
    unsigned incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned tot = 0;
      for (int k = 0; k < kB2qThreads / 32; k++) {
        const unsigned t = s_warp[k];
        s_warp[k] = tot;
        tot += t;
      }
      s_base = tot ? atomicAdd(&cnt->qtail, static_cast<unsigned long long>(tot)) : 0ull;
    }
    __syncthreads();
    unsigned long long pos = s_base + s_warp[wid] + (incl - mine);
    while (word) {
      const int b = __ffs(word) - 1;
      word &= word - 1u;
      queue[pos++] = static_cast<int32_t>((w << 5) + b);
    }
    __syncthreads();
  }
}

// Parents in original ids, -1 for unreached: each original id gathers its
// row's parent (coalesced writes; a scatter through perm wrote partial
// sectors).  Rows [in_rows, n) have no in-edges, so only the source among
// them is reached; their parents are not read.
__global__ void bfs_finish_kernel(int32_t n, int32_t in_rows, int source_old,
                                  const int32_t *__restrict__ parent,
                                  const int32_t *__restrict__ inv, int32_t *out_old) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t o = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; o < n; o += stride) {
    const int v = inv[o];
    int32_t r = -1;
    if (v < in_rows) {
      r = parent[v];
    } else if (o == source_old) {
      r = source_old;
    }
    out_old[o] = r;
  }
}

int NumSms() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

unsigned BfsGrid(int64_t items) {
  return static_cast<unsigned>(
      std::max<int64_t>(1, std::min<int64_t>((items + 255) / 256, NumSms() * 16)));
}

// top-down blocks: threads and edges per thread per chunk, with the
// frontier scanned by CUB, or scanned by each block itself (small frontiers)
constexpr int kTdThreads = 256, kTdPerThread = 8;
constexpr int kTdSmallThreads = 1024, kTdSmallPerThread = 4;

// Blocks for a top-down step of at most `edges` edges: one chunk each, at
// most two resident waves.
unsigned TdGrid(int64_t edges, int threads, int per_thread) {
  const int64_t chunk = static_cast<int64_t>(threads) * per_thread;
  const int64_t cap = static_cast<int64_t>(NumSms()) * (4096 / threads);
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((edges + chunk - 1) / chunk, cap)));
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
  // in-CSR rows with in-neighbours (rows are sorted by in-degree; the rest
  // can only be reached as the source)
  const int32_t in_rows = static_cast<int32_t>(g.bin_row_start[kBinZero]);
  const int64_t in_words = (static_cast<int64_t>(in_rows) + 31) / 32;
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
  BfsCounters hc{};
  auto read_counters = [&]() -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(&hc, b.cnt, sizeof(hc), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
  };
  auto t0 = clock::now();
  const unsigned grid = BfsGrid(n);
  BFS_TRY(cudaMemsetAsync(b.parent, 0xff, sizeof(int32_t) * n, s));  // every parent -1
  bfs_source_kernel<<<1, 1, 0, s>>>(g.inv, source_old, ooff, b.parent, b.queue[0], cnt);
  BFS_TRY(cudaGetLastError());
  BFS_TRY(read_counters());
  record("i", -1, seconds(t0, clock::now()));

  int cur = 0;                // queue[cur] is the frontier
  int64_t qsize = 1;
  int64_t edges_to_check = g.m;
  int64_t scout_count = static_cast<int64_t>(hc.scout);
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
      BFS_TRY(cudaMemsetAsync(b.bm[1], 0, sizeof(unsigned) * words, s));
      bfs_queue_to_bitmap_kernel<<<BfsGrid(qsize), 256, 0, s>>>(qsize, b.queue[cur], b.bm[0]);
      BFS_TRY(cudaGetLastError());
      if (steps) BFS_TRY(cudaStreamSynchronize(s));  // only to time the step
      record("e", -1, seconds(ts, clock::now()));
      int front = 0;
      int64_t awake = qsize, old_awake = 0;
      do {
        ts = clock::now();
        old_awake = awake;
        BFS_TRY(cudaMemsetAsync(b.cnt, 0, sizeof(BfsCounters), s));
        bfs_bu_kernel<<<BfsGrid(in_rows), 256, 0, s>>>(in_rows, ioff, inbr, b.bm[front], g.perm,
                                                       b.bm[front ^ 1], b.parent, cnt);
        BFS_TRY(cudaGetLastError());
        if (front == 0 && in_words < words)  // the frontier's bits past in_rows (a source
          BFS_TRY(cudaMemsetAsync(b.bm[0] + in_words, 0,  // without in-edges) are spent
                                  sizeof(unsigned) * (words - in_words), s));
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
      // the last bottom-up step wrote the words of rows [0, in_rows) only
      bfs_bitmap_to_queue_kernel<<<BfsGrid(in_rows), kB2qThreads, 0, s>>>(
          in_rows, b.bm[front], b.queue[cur], cnt);
      BFS_TRY(cudaGetLastError());
      BFS_TRY(read_counters());
      qsize = static_cast<int64_t>(hc.qtail);
      record("c", -1, seconds(ts, clock::now()));
      scout_count = 1;
    } else {
      auto ts = clock::now();
      edges_to_check -= scout_count;
      // grid sized by the largest edge count the frontier can have (the
      // kernels loop over whatever the real count is)
      const int64_t edge_bound = std::min<int64_t>(g.m, qsize * g.max_degree);
      if (qsize <= kTdSmallThreads) {
        BFS_TRY(cudaMemsetAsync(b.cnt, 0, sizeof(BfsCounters), s));
        bfs_td_kernel<kTdSmallThreads, kTdSmallPerThread, true>
            <<<TdGrid(edge_bound, kTdSmallThreads, kTdSmallPerThread), kTdSmallThreads, 0, s>>>(
                qsize, b.queue[cur], nullptr, ooff, onbr, g.perm, b.parent, b.queue[cur ^ 1],
                cnt);
      } else {
        bfs_frontier_degree_kernel<<<BfsGrid(qsize), 256, 0, s>>>(qsize, b.queue[cur], ooff,
                                                                  b.deg);
        BFS_TRY(cudaGetLastError());
        BFS_TRY(cudaMemsetAsync(b.deg + qsize, 0, sizeof(int64_t), s));
        size_t bytes = static_cast<size_t>(b.cap_tmp);
        BFS_TRY(cub::DeviceScan::ExclusiveSum(b.tmp, bytes, b.deg, b.eoff,
                                              static_cast<int>(qsize + 1), s));
        BFS_TRY(cudaMemsetAsync(b.cnt, 0, sizeof(BfsCounters), s));
        bfs_td_kernel<kTdThreads, kTdPerThread, false>
            <<<TdGrid(edge_bound, kTdThreads, kTdPerThread), kTdThreads, 0, s>>>(
            qsize, b.queue[cur], b.eoff, ooff, onbr, g.perm, b.parent, b.queue[cur ^ 1], cnt);
      }
      BFS_TRY(cudaGetLastError());
      BFS_TRY(read_counters());
      scout_count = static_cast<int64_t>(hc.scout);
      qsize = static_cast<int64_t>(hc.qtail);
      cur ^= 1;
      record("td", qsize, seconds(ts, clock::now()));
    }
  }
  bfs_finish_kernel<<<grid, 256, 0, s>>>(static_cast<int32_t>(n), in_rows, source_old, b.parent,
                                         g.inv, out_old);
  BFS_TRY(cudaGetLastError());
  BFS_TRY(cudaStreamSynchronize(s));
  return cudaSuccess;
}

#undef BFS_TRY

}  // namespace prgpu
