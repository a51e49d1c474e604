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
// The device drives the steps: a one-thread decide kernel applies the
// switching rule to the counts the last step left in a control block and
// picks the next step; the steps run as the cases of a SWITCH node inside a
// WHILE node of one CUDA graph, so a whole search is one graph launch with
// no host round trip.  (With GAPBS_PR_PLAIN_LAUNCH=1 the host launches the
// same kernels step by step, reading the decision back each time, for
// profilers that cannot replay kernels inside conditional graphs.)
// Queues and bitmaps hold the mirror's degree-sorted ids; parent[] is
// indexed by mirror row but stores the parent's original id, so the
// write-back only gathers it into original order.
// Parents can differ from run to run (which frontier vertex wins a claim is
// a race, as in the reference); depths, reached sets and tree sizes cannot.
//
// Top-down work is spread over the frontier's edges, not its vertices
// (frontier degrees are scanned, each thread takes edges and finds its
// vertex by a forward search in the scan), so a hub in the frontier does not
// serialise a warp.  Bottom-up work: each warp owns two words of 32
// consecutive vertices at a time, walks the two vertices of every lane
// together, and writes each bitmap word with one ballot.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "loop_graph.h"

namespace prgpu {

namespace {

// Step kinds; the first kNumCases are the SWITCH cases, in this order.
enum BfsKind : int32_t {
  kTdSmall = 0,   // "td", frontier scanned inside each block
  kTdBig = 1,     // "td", frontier scanned device-wide
  kToBitmap = 2,  // "e": queue -> bitmap (entering bottom-up)
  kBottomUp = 3,  // "bu"
  kToQueue = 4,   // "c": bitmap -> queue (leaving bottom-up)
  kNumCases = 5,
  kDone = 5,  // no case: the loop ends
  kInit = 6,  // "i": the source set-up
};

constexpr int kBfsMaxLog = 1024;  // logged steps (the count goes on beyond)

struct BfsCounters {
  unsigned long long qtail;  // next-frontier queue length
  unsigned long long scout;  // top-down scout count
  unsigned long long awake;  // bottom-up awake count
};

struct BfsLogRec {
  int32_t kind;
  int32_t unused;
  int64_t count;
  unsigned long long ns;
};

// Search state, in device memory.  The decide kernel owns every field but
// cnt, which the step kernels add to.
struct BfsCtl {
  int32_t src;    // the source's mirror row
  int32_t last;   // the step that ran last (kInit before the first)
  int32_t next;   // the step the last decide chose
  int32_t mode;   // 0: frontier in a queue (top-down), 1: in a bitmap
  int32_t cur;    // queue[cur] is the frontier
  int32_t front;  // bm[front] is the frontier bitmap
  int32_t error;  // the step guard tripped
  int32_t nlog;   // steps logged (all steps, also past kBfsMaxLog)
  int64_t qsize, edges_to_check, scout, awake, old_awake, guard;
  unsigned long long t_prev;
  BfsCounters cnt;
  BfsLogRec log[kBfsMaxLog];
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int32_t out_degree(const int32_t *ooff, int v) {
  return ooff[v + 1] - ooff[v];
}

// The source (original id) becomes its own parent and the first frontier;
// its out-degree is the first scout count; the control block starts over.
// One thread.  parent[] is indexed by mirror row but holds original ids
// (only its sign is read during the search), so the write-back needs no
// second lookup.
__global__ void bfs_source_kernel(const int32_t *__restrict__ inv, int source_old, int64_t m,
                                  const int32_t *__restrict__ ooff, int32_t *parent,
                                  int32_t *queue0, BfsCtl *ctl) {
  const int src = inv[source_old];
  parent[src] = source_old;
  queue0[0] = src;
  ctl->src = src;
  ctl->last = kInit;
  ctl->next = kInit;
  ctl->mode = 0;
  ctl->cur = 0;
  ctl->front = 0;
  ctl->error = 0;
  ctl->nlog = 0;
  ctl->qsize = 1;
  ctl->edges_to_check = m;
  ctl->scout = out_degree(ooff, src);
  ctl->awake = 0;
  ctl->old_awake = 0;
  ctl->guard = 0;
  ctl->cnt = BfsCounters{0, 0, 0};
  ctl->t_prev = global_ns();
}

// Folds the step that just ran into the state (src/bfs.cc:140-172), logs it,
// and picks the next one by the reference's rule.  One thread.  In a graph
// it also sets the SWITCH value and the WHILE condition; the step guard
// ends the loop after at most n + 2 steps whatever the counts say.
__global__ void bfs_decide_kernel(BfsCtl *ctl, int64_t n, int alpha, int beta, int in_graph,
                                  cudaGraphConditionalHandle loop_h,
                                  cudaGraphConditionalHandle kind_h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  BfsCtl &c = *ctl;
  const unsigned long long now = global_ns();
  int64_t count = -1;
  switch (c.last) {
    case kTdSmall:
    case kTdBig:
      c.scout = static_cast<int64_t>(c.cnt.scout);
      c.qsize = static_cast<int64_t>(c.cnt.qtail);
      c.cur ^= 1;
      count = c.qsize;
      break;
    case kToBitmap:
      c.awake = c.qsize;
      c.front = 0;
      break;
    case kBottomUp:
      c.awake = static_cast<int64_t>(c.cnt.awake);
      c.front ^= 1;
      count = c.awake;
      break;
    case kToQueue:
      c.qsize = static_cast<int64_t>(c.cnt.qtail);
      c.scout = 1;
      c.mode = 0;
      break;
    default:  // kInit
      break;
  }
  if (c.nlog < kBfsMaxLog) c.log[c.nlog] = BfsLogRec{c.last, 0, count, now - c.t_prev};
  c.nlog++;
  c.t_prev = now;
  int next;
  if (c.mode == 1) {
    if (c.last == kToBitmap || c.awake >= c.old_awake || c.awake > n / beta) {
      c.old_awake = c.awake;
      next = kBottomUp;
    } else {
      next = kToQueue;
    }
  } else if (c.qsize == 0) {
    next = kDone;
  } else if (c.scout > c.edges_to_check / alpha) {
    c.mode = 1;
    next = kToBitmap;
  } else {
    c.edges_to_check -= c.scout;
    next = c.qsize <= 1024 ? kTdSmall : kTdBig;
  }
  if (next != kDone && ++c.guard > n + 2) {
    c.error = 1;
    next = kDone;
  }
  c.cnt = BfsCounters{0, 0, 0};
  c.last = next;
  c.next = next;
  if (in_graph) {
    cudaGraphSetConditional(kind_h, static_cast<unsigned>(next));  // kDone: no case
    cudaGraphSetConditional(loop_h, next == kDone ? 0u : 1u);
  }
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

// ---- top-down ----------------------------------------------------------------

// Out-degree of every frontier vertex, and a zero after them (input of the
// edge scan).
__global__ void bfs_frontier_degree_kernel(const BfsCtl *ctl, const int32_t *__restrict__ q0,
                                           const int32_t *__restrict__ q1,
                                           const int32_t *__restrict__ ooff, int64_t *deg) {
  const int64_t q = ctl->qsize;
  const int32_t *queue = ctl->cur ? q1 : q0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= q; i += stride)
    deg[i] = i < q ? out_degree(ooff, queue[i]) : 0;
}

// Exclusive scan of deg[0, q] into eoff[0, q] for a q known only on the
// device: chunks of kScanChunk items scanned per block (chunk totals to
// sums[]), the chunk totals scanned by one block, the chunk offsets added.
constexpr int kScanThreads = 256, kScanPer = 8, kScanChunk = kScanThreads * kScanPer;
constexpr int kSumThreads = 1024;

__device__ __forceinline__ int64_t warp_incl_scan(int64_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__global__ void __launch_bounds__(kScanThreads)
bfs_scan_chunks_kernel(const BfsCtl *ctl, const int64_t *__restrict__ deg, int64_t *eoff,
                       int64_t *sums) {
  __shared__ int64_t s_w[kScanThreads / 32];
  const int64_t items = ctl->qsize + 1;
  const int64_t nch = (items + kScanChunk - 1) / kScanChunk;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {  // block-uniform
    const int64_t base = c * kScanChunk + static_cast<int64_t>(threadIdx.x) * kScanPer;
    int64_t v[kScanPer];
    int64_t run = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
      v[k] = base + k < items ? deg[base + k] : 0;
      run += v[k];
    }
    const int64_t incl = warp_incl_scan(run, lane);
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t t = 0;
      for (int w = 0; w < kScanThreads / 32; w++) {
        const int64_t x = s_w[w];
        s_w[w] = t;
        t += x;
      }
      sums[c] = t;
    }
    __syncthreads();
    int64_t pre = s_w[wid] + incl - run;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
      if (base + k < items) eoff[base + k] = pre;
      pre += v[k];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSumThreads) bfs_scan_sums_kernel(const BfsCtl *ctl,
                                                                    int64_t *sums) {
  __shared__ int64_t s_w[kSumThreads / 32];
  const int64_t nch = (ctl->qsize + 1 + kScanChunk - 1) / kScanChunk;
  const int64_t per = (nch + kSumThreads - 1) / kSumThreads;
  const int64_t lo = min(nch, per * threadIdx.x), hi = min(nch, lo + per);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t run = 0;
  for (int64_t i = lo; i < hi; i++) run += sums[i];
  const int64_t incl = warp_incl_scan(run, lane);
  if (lane == 31) s_w[wid] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t t = 0;
    for (int w = 0; w < kSumThreads / 32; w++) {
      const int64_t x = s_w[w];
      s_w[w] = t;
      t += x;
    }
  }
  __syncthreads();
  int64_t pre = s_w[wid] + incl - run;
  for (int64_t i = lo; i < hi; i++) {
    const int64_t x = sums[i];
    sums[i] = pre;
    pre += x;
  }
}

__global__ void bfs_scan_add_kernel(const BfsCtl *ctl, int64_t *eoff,
                                    const int64_t *__restrict__ sums) {
  const int64_t items = ctl->qsize + 1;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < items;
       i += stride)
    eoff[i] += sums[i / kScanChunk];
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
bfs_td_kernel(BfsCtl *ctl, const int32_t *__restrict__ q0, const int32_t *__restrict__ q1,
              int32_t *nq0, int32_t *nq1, const int64_t *__restrict__ eoff_g,
              const int32_t *__restrict__ ooff, const int32_t *__restrict__ onbr,
              const int32_t *__restrict__ perm, int32_t *parent) {
  __shared__ int64_t s_eoff[SMALL ? NT + 1 : 1];
  __shared__ int32_t s_q[SMALL ? NT : 1];
  __shared__ unsigned s_warp[NT / 32];
  __shared__ unsigned long long s_base;
  const int64_t q = ctl->qsize;
  const int cur = ctl->cur;
  const int32_t *queue_g = cur ? q1 : q0;
  int32_t *next = cur ? nq0 : nq1;
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
    const int64_t incl = warp_incl_scan(d, lane);
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
  const int64_t edges = eoff[q];  // the scan's total
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
        int32_t curp;
        asm volatile("ld.global.ca.s32 %0, [%1];" : "=r"(curp) : "l"(parent + v));
        if (curp < 0 && atomicCAS(parent + v, curp, __ldg(perm + u)) == curp) {
          vals[k] = v;
          mask |= 1u << k;
          scout += static_cast<unsigned long long>(max(out_degree(ooff, v), 1));
        }
      }
    }
    block_append<NT, PT>(mask, vals, next, &ctl->cnt.qtail, s_warp, &s_base);
  }
  for (int o = 16; o > 0; o >>= 1) scout += __shfl_xor_sync(0xffffffffu, scout, o);
  if ((threadIdx.x & 31) == 0 && scout) atomicAdd(&ctl->cnt.scout, scout);
}

// ---- bottom-up -----------------------------------------------------------------

__global__ void bfs_clear_bitmaps_kernel(unsigned *bm0, unsigned *bm1, int64_t words) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < words;
       i += stride) {
    bm0[i] = 0u;
    bm1[i] = 0u;
  }
}

__global__ void bfs_queue_to_bitmap_kernel(const BfsCtl *ctl, const int32_t *__restrict__ q0,
                                           const int32_t *__restrict__ q1, unsigned *bm) {
  const int64_t q = ctl->qsize;
  const int32_t *queue = ctl->cur ? q1 : q0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < q; i += stride) {
    const int v = queue[i];
    atomicOr(bm + (v >> 5), 1u << (v & 31));
  }
}

__device__ __forceinline__ bool in_front(const unsigned *__restrict__ front, int u) {
  return (__ldg(front + (u >> 5)) >> (u & 31)) & 1u;
}

// Bottom-up step: each warp owns two bitmap words (32 consecutive vertices
// each) at a time and every lane walks its two vertices' in-lists together,
// so two independent load chains (neighbour id, then its frontier bit) are
// in flight per lane; each vertex still takes the first in-neighbour in list
// order found in the frontier.  Only rows [0, rows) have in-neighbours (rows
// are sorted by in-degree), so only their words are visited; the words after
// them stay zero.
__global__ void bfs_bu_kernel(BfsCtl *ctl, int32_t rows, const int32_t *__restrict__ ioff,
                              const int32_t *__restrict__ inbr, const unsigned *bm0,
                              const unsigned *bm1, unsigned *nbm0, unsigned *nbm1,
                              const int32_t *__restrict__ perm, int32_t *parent) {
  const int f = ctl->front;
  const unsigned *front = f ? bm1 : bm0;
  unsigned *next = f ? nbm0 : nbm1;
  const int32_t n = rows;
  const int lane = threadIdx.x & 31;
  const int64_t words = (static_cast<int64_t>(n) + 31) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  unsigned long long awake = 0;
  for (int64_t w = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < words;
       w += 2 * warps) {
    const int64_t w2 = w + warps;  // the warp's second word (warp-uniform test)
    const int64_t v1 = (w << 5) + lane, v2 = (w2 << 5) + lane;
    int j1 = 0, e1 = 0, j2 = 0, e2 = 0;
    if (v1 < n && parent[v1] < 0) {
      j1 = ioff[v1];
      e1 = ioff[v1 + 1];
    }
    if (w2 < words && v2 < n && parent[v2] < 0) {
      j2 = ioff[v2];
      e2 = ioff[v2 + 1];
    }
    int p1 = -1, p2 = -1;  // the in-neighbour found (mirror row), if any
    while (j1 < e1 || j2 < e2) {
      const int u1 = j1 < e1 ? inbr[j1] : -1;
      const int u2 = j2 < e2 ? inbr[j2] : -1;
      const bool h1 = u1 >= 0 && in_front(front, u1);
      const bool h2 = u2 >= 0 && in_front(front, u2);
      if (h1) {
        p1 = u1;
        e1 = j1;  // chain 1 done
      } else {
        j1++;
      }
      if (h2) {
        p2 = u2;
        e2 = j2;
      } else {
        j2++;
      }
    }
    if (p1 >= 0) parent[v1] = __ldg(perm + p1);
    if (p2 >= 0) parent[v2] = __ldg(perm + p2);
    const unsigned word1 = __ballot_sync(0xffffffffu, p1 >= 0);
    if (lane == 0) next[w] = word1;
    if (w2 < words) {
      const unsigned word2 = __ballot_sync(0xffffffffu, p2 >= 0);
      if (lane == 0) next[w2] = word2;
    }
    awake += (p1 >= 0 ? 1 : 0) + (p2 >= 0 ? 1 : 0);
  }
  for (int o = 16; o > 0; o >>= 1) awake += __shfl_xor_sync(0xffffffffu, awake, o);
  if (lane == 0 && awake) atomicAdd(&ctl->cnt.awake, awake);
}

// After a bottom-up step that read bm0: the frontier's bits past the rows
// with in-edges (only a source without in-edges can have one) are spent;
// clear them so the next read of bm0 sees only the bottom-up steps' words.
__global__ void bfs_bu_tail_kernel(const BfsCtl *ctl, unsigned *bm0, int64_t in_words,
                                   int64_t words) {
  if (ctl->front != 0) return;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = in_words + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
       i < words; i += stride)
    bm0[i] = 0u;
}

// Set bits of the frontier bitmap -> queue[cur], over the words of vertices
// [0, n).  Each thread takes one word per block round and appends its
// vertices (up to 32) with one global atomic per block round.
constexpr int kB2qThreads = 256;

__global__ void __launch_bounds__(kB2qThreads)
bfs_bitmap_to_queue_kernel(BfsCtl *ctl, int32_t n, const unsigned *__restrict__ bm0,
                           const unsigned *__restrict__ bm1, int32_t *q0, int32_t *q1) {
  __shared__ unsigned s_warp[kB2qThreads / 32];
  __shared__ unsigned long long s_base;
  const unsigned *bm = ctl->front ? bm1 : bm0;
  int32_t *queue = ctl->cur ? q1 : q0;
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
      s_base = tot ? atomicAdd(&ctl->cnt.qtail, static_cast<unsigned long long>(tot)) : 0ull;
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

// ---- launch plan -----------------------------------------------------------------

int NumSms() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

unsigned GridFor(int64_t items, int threads, int per_sm) {
  return static_cast<unsigned>(std::max<int64_t>(
      1, std::min<int64_t>((items + threads - 1) / threads, int64_t(NumSms()) * per_sm)));
}

// top-down blocks: threads and edges per thread per chunk, with the
// frontier scanned device-wide, or scanned by each block itself
constexpr int kTdThreads = 256, kTdPerThread = 8;
constexpr int kTdSmallThreads = 1024, kTdSmallPerThread = 4;

// Every pointer, size and grid of a search's steps: fixed per graph and
// scratch, so the steps can be captured once into the loop graph.
struct BfsPlan {
  BfsCtl *ctl;
  int32_t *q0, *q1, *parent;
  unsigned *bm0, *bm1;
  int64_t *deg, *eoff, *sums;
  const int32_t *ooff, *onbr, *ioff, *inbr, *perm;
  int64_t n, words, in_words;
  int32_t in_rows;
  int32_t alpha, beta;
  unsigned g_small, g_big, g_n, g_rows, g_scan, g_words;
};

cudaError_t LaunchStep(const BfsPlan &p, int kind, cudaStream_t s) {
  switch (kind) {
    case kTdSmall:
      bfs_td_kernel<kTdSmallThreads, kTdSmallPerThread, true>
          <<<p.g_small, kTdSmallThreads, 0, s>>>(p.ctl, p.q0, p.q1, p.q0, p.q1, nullptr, p.ooff,
                                                 p.onbr, p.perm, p.parent);
      break;
    case kTdBig:
      bfs_frontier_degree_kernel<<<p.g_n, 256, 0, s>>>(p.ctl, p.q0, p.q1, p.ooff, p.deg);
      bfs_scan_chunks_kernel<<<p.g_scan, kScanThreads, 0, s>>>(p.ctl, p.deg, p.eoff, p.sums);
      bfs_scan_sums_kernel<<<1, kSumThreads, 0, s>>>(p.ctl, p.sums);
      bfs_scan_add_kernel<<<p.g_n, 256, 0, s>>>(p.ctl, p.eoff, p.sums);
      bfs_td_kernel<kTdThreads, kTdPerThread, false><<<p.g_big, kTdThreads, 0, s>>>(
          p.ctl, p.q0, p.q1, p.q0, p.q1, p.eoff, p.ooff, p.onbr, p.perm, p.parent);
      break;
    case kToBitmap:
      bfs_clear_bitmaps_kernel<<<p.g_words, 256, 0, s>>>(p.bm0, p.bm1, p.words);
      bfs_queue_to_bitmap_kernel<<<p.g_n, 256, 0, s>>>(p.ctl, p.q0, p.q1, p.bm0);
      break;
    case kBottomUp:
      bfs_bu_kernel<<<p.g_rows, 256, 0, s>>>(p.ctl, p.in_rows, p.ioff, p.inbr, p.bm0, p.bm1,
                                             p.bm0, p.bm1, p.perm, p.parent);
      bfs_bu_tail_kernel<<<p.g_words, 256, 0, s>>>(p.ctl, p.bm0, p.in_words, p.words);
      break;
    case kToQueue:
      bfs_bitmap_to_queue_kernel<<<p.g_rows, kB2qThreads, 0, s>>>(p.ctl, p.in_rows, p.bm0,
                                                                  p.bm1, p.q0, p.q1);
      break;
    default:
      break;
  }
  return cudaGetLastError();
}

// The search loop as one graph: WHILE { decide; SWITCH(kind) { steps } }.
cudaError_t BuildLoopGraph(const BfsPlan &p, cudaStream_t cap, cudaGraphExec_t *exec) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle loop_h = 0, kind_h = 0;
  cudaGraphNodeParams wp = {};
  cudaGraphNode_t while_node = nullptr, decide_node = nullptr, switch_node = nullptr;
  e = cudaGraphConditionalHandleCreate(&loop_h, g, 1, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = loop_h;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    e = cudaGraphAddNode(&while_node, g, nullptr, 0, &wp);
  }
  cudaGraph_t body = e == cudaSuccess ? wp.conditional.phGraph_out[0] : nullptr;
  if (e == cudaSuccess)
    e = cudaGraphConditionalHandleCreate(&kind_h, body, kDone, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    BfsCtl *ctl = p.ctl;
    int64_t n = p.n;
    int alpha = p.alpha, beta = p.beta, in_graph = 1;
    void *params[] = {&ctl, &n, &alpha, &beta, &in_graph, &loop_h, &kind_h};
    cudaKernelNodeParams kp = {};
    kp.func = reinterpret_cast<void *>(bfs_decide_kernel);
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = params;
    e = cudaGraphAddKernelNode(&decide_node, body, nullptr, 0, &kp);
  }
  cudaGraphNodeParams sp = {};
  if (e == cudaSuccess) {
    sp.type = cudaGraphNodeTypeConditional;
    sp.conditional.handle = kind_h;
    sp.conditional.type = cudaGraphCondTypeSwitch;
    sp.conditional.size = kNumCases;
    e = cudaGraphAddNode(&switch_node, body, &decide_node, 1, &sp);
  }
  for (int k = 0; e == cudaSuccess && k < kNumCases; k++) {
    e = cudaStreamBeginCaptureToGraph(cap, sp.conditional.phGraph_out[k], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) break;
    const cudaError_t le = LaunchStep(p, k, cap);
    cudaGraph_t out = nullptr;
    e = cudaStreamEndCapture(cap, &out);
    if (e == cudaSuccess) e = le;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  return e;
}

const char *StepName(int kind) {
  switch (kind) {
    case kInit: return "i";
    case kTdSmall:
    case kTdBig: return "td";
    case kToBitmap: return "e";
    case kBottomUp: return "bu";
    case kToQueue: return "c";
    default: return "?";
  }
}

}  // namespace

void FreeBfsScratch(BfsScratch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  void *ptrs[] = {b->parent, b->queue[0], b->queue[1], b->bm[0], b->bm[1], b->deg, b->eoff,
                  b->sums, b->ctl};
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
                               std::vector<BfsStep> *steps, int64_t *nsteps,
                               std::string *err) {
  const int64_t n = g.n;
  const int64_t words = (n + 31) / 32;
  const int64_t nch = (n + 1 + kScanChunk - 1) / kScanChunk;
  if (!b.parent || b.cap_n < n) {
    FreeBfsScratch(&b);
    BFS_TRY(cudaMalloc(&b.parent, sizeof(int32_t) * std::max<int64_t>(n, 1)));
    BFS_TRY(cudaMalloc(&b.queue[0], sizeof(int32_t) * std::max<int64_t>(n, 1)));
    BFS_TRY(cudaMalloc(&b.queue[1], sizeof(int32_t) * std::max<int64_t>(n, 1)));
    BFS_TRY(cudaMalloc(&b.deg, sizeof(int64_t) * (n + 1)));
    BFS_TRY(cudaMalloc(&b.eoff, sizeof(int64_t) * (n + 1)));
    BFS_TRY(cudaMalloc(&b.sums, sizeof(int64_t) * (nch + 1)));
    BFS_TRY(cudaMalloc(&b.bm[0], sizeof(unsigned) * std::max<int64_t>(words, 1)));
    BFS_TRY(cudaMalloc(&b.bm[1], sizeof(unsigned) * std::max<int64_t>(words, 1)));
    BFS_TRY(cudaMalloc(&b.ctl, sizeof(BfsCtl)));
    b.cap_n = n;
  }
  BfsPlan p;
  std::memset(&p, 0, sizeof(p));
  p.ctl = static_cast<BfsCtl *>(b.ctl);
  p.q0 = b.queue[0];
  p.q1 = b.queue[1];
  p.parent = b.parent;
  p.bm0 = b.bm[0];
  p.bm1 = b.bm[1];
  p.deg = b.deg;
  p.eoff = b.eoff;
  p.sums = b.sums;
  p.ooff = g.directed ? g.orowoff : g.rowoff;
  p.onbr = g.directed ? g.ocol : g.col;
  p.ioff = g.rowoff;
  p.inbr = g.col;
  p.perm = g.perm;
  p.n = n;
  p.words = words;
  // in-CSR rows with in-neighbours (rows are sorted by in-degree; the rest
  // can only be reached as the source)
  p.in_rows = static_cast<int32_t>(g.bin_row_start[kBinZero]);
  p.in_words = (static_cast<int64_t>(p.in_rows) + 31) / 32;
  p.alpha = alpha;
  p.beta = beta;
  // fixed grids, sized for the largest step of each kind (the kernels loop
  // over whatever the step's real size is)
  const int64_t small_edges = std::min<int64_t>(g.m, int64_t(kTdSmallThreads) * g.max_degree);
  p.g_small = GridFor((small_edges + kTdSmallPerThread - 1) / kTdSmallPerThread, kTdSmallThreads,
                      2048 / kTdSmallThreads * 2);
  p.g_big = GridFor((g.m + kTdPerThread - 1) / kTdPerThread, kTdThreads, 2048 / kTdThreads * 2);
  p.g_n = GridFor(n + 1, 256, 16);
  p.g_rows = GridFor(p.in_rows, 256, 16);
  p.g_scan = GridFor(nch * kScanThreads, kScanThreads, 8);
  p.g_words = GridFor(words, 256, 16);

  const unsigned grid = GridFor(n, 256, 16);
  BFS_TRY(cudaMemsetAsync(b.parent, 0xff, sizeof(int32_t) * n, s));  // every parent -1
  bfs_source_kernel<<<1, 1, 0, s>>>(g.inv, source_old, g.m, p.ooff, b.parent, b.queue[0], p.ctl);
  BFS_TRY(cudaGetLastError());
  if (PlainLaunchMode()) {
    for (;;) {  // the decide kernel's step guard ends this loop
      bfs_decide_kernel<<<1, 32, 0, s>>>(p.ctl, n, alpha, beta, 0, 0, 0);
      BFS_TRY(cudaGetLastError());
      int32_t next = kDone;
      BFS_TRY(cudaMemcpyAsync(&next, &p.ctl->next, sizeof(next), cudaMemcpyDeviceToHost, s));
      BFS_TRY(cudaStreamSynchronize(s));
      if (next == kDone) break;
      BFS_TRY(LaunchStep(p, next, s));
    }
  } else {
    const bool same = b.exec && b.plan.size() == sizeof(p) &&
                      std::memcmp(b.plan.data(), &p, sizeof(p)) == 0;
    if (!same) {
      if (b.exec) cudaGraphExecDestroy(b.exec);
      b.exec = nullptr;
      b.plan.clear();
      if (!b.cap_stream) BFS_TRY(cudaStreamCreateWithFlags(&b.cap_stream, cudaStreamNonBlocking));
      BFS_TRY(BuildLoopGraph(p, b.cap_stream, &b.exec));
      b.plan.assign(reinterpret_cast<const unsigned char *>(&p),
                    reinterpret_cast<const unsigned char *>(&p) + sizeof(p));
    }
    BFS_TRY(cudaGraphLaunch(b.exec, s));
  }
  bfs_finish_kernel<<<grid, 256, 0, s>>>(static_cast<int32_t>(n), p.in_rows, source_old, b.parent,
                                         g.inv, out_old);
  BFS_TRY(cudaGetLastError());
  // the control block up to its log, then the logged steps
  std::vector<unsigned char> head_bytes(sizeof(BfsCtl));
  BfsCtl *head = reinterpret_cast<BfsCtl *>(head_bytes.data());
  BFS_TRY(cudaMemcpyAsync(head, p.ctl, offsetof(BfsCtl, log), cudaMemcpyDeviceToHost, s));
  BFS_TRY(cudaStreamSynchronize(s));
  if (head->error) {
    *err = "bfs: step limit exceeded";
    return cudaErrorUnknown;
  }
  if (nsteps) *nsteps = head->nlog;
  if (steps) {
    const int k = std::min<int>(head->nlog, kBfsMaxLog);
    std::vector<BfsLogRec> log(k);
    if (k > 0) {
      BFS_TRY(cudaMemcpyAsync(log.data(), p.ctl->log, sizeof(BfsLogRec) * k,
                              cudaMemcpyDeviceToHost, s));
      BFS_TRY(cudaStreamSynchronize(s));
    }
    steps->clear();
    for (const BfsLogRec &r : log)
      steps->push_back(BfsStep{StepName(r.kind), r.count, static_cast<double>(r.ns) * 1e-9});
  }
  return cudaSuccess;
}

#undef BFS_TRY

}  // namespace prgpu
