// cc.cu -- connected components on the device CSR mirror
// (pr_gpu_connected_components in include/pr_gpu.h).
//
// The reference's Afforest (src/cc.cc:40-150) labels every vertex with the
// root of its component tree; its Link always hooks the larger root under
// the smaller one and Compress only shortens chains, so every label is at
// most the vertex's own id and the final root of a component is its
// smallest vertex id.  That labelling is canonical, and the device computes
// exactly it:
//   1. comp[v] = v;
//   2. two sampling rounds: every vertex links with its r-th out-neighbour
//      (r = 0, 1), each round followed by a compress (which keeps the next
//      round's link chases short);
//   3. the component of the highest-degree vertex (row 0 of the degree-sorted
//      mirror: a vertex of the largest intermediate component, which the
//      reference estimates by sampling) is skipped in the final phase; row 0
//      has the smallest id, so it is the root of its tree and that
//      component's label is 0;
//   4. every other vertex links with its remaining out-neighbours and, for a
//      directed graph, with all its in-neighbours; compress;
//   5. ids are mapped back: each root takes the smallest original id of its
//      component (atomicMin; the largest component's members reduced per
//      block first), every vertex that root's label; a vertex without edges
//      is its own component and keeps its own id.
// Link is the reference's lock-free hooking loop with compare-and-swap; it
// and the compress chase are bounded (an iteration limit sets an error flag
// instead of spinning), so a defect cannot hang the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <string>

#include "internal.h"

namespace prgpu {

namespace {

constexpr int kChaseLimit = 1 << 20;  // far above any tree depth reached

__device__ __forceinline__ int ld_comp(const int *comp, int x) {
  return *reinterpret_cast<const volatile int *>(comp + x);
}

// A weak load that may be served from this SM's L1 and so be stale.  Used
// where any ancestor of x serves as well as its current parent: comp values
// only ever move to other members of the same tree, and a root stays a root
// until a link hooks it.  Most chases end at the few roots of the largest
// components, whose lines would otherwise be requested from L2 by every warp.
__device__ __forceinline__ int ld_comp_cached(const int *comp, int x) {
  int r;
  asm volatile("ld.global.ca.s32 %0, [%1];" : "=r"(r) : "l"(comp + x));
  return r;
}

// src/cc.cc:40-55 with compare-and-swap on the device.  Reads that may come
// from L1 (stale) are safe here: a stale comp[x] is x itself or one of x's
// ancestors, a vertex that is not a root never becomes one again, and
// comp[high] == low at any time means high and low share a tree for good.
// A value that looks like a root is confirmed from L2 before the
// compare-and-swap, and a failed compare-and-swap returns the current
// parent.  Every pass of the loop moves high strictly up its tree, so the
// loop ends; the iteration limit only guards against a defect.  The roots
// of the large trees are read by almost every warp in the second sampling
// round, which is what keeps those reads in L1.
__device__ void cc_link(int u, int v, int *comp, int *err) {
  int p1 = ld_comp(comp, u);
  int p2 = ld_comp_cached(comp, v);
  // comp[u] == u read fresh: u is a root, so the first pass needs no re-read
  // of its line when u is the higher root (most links of the first round)
  bool u_root = p1 == u;
  for (int it = 0; p1 != p2; it++) {
    if (it >= kChaseLimit) {
      atomicExch(err, 1);
      return;
    }
    const int high = max(p1, p2), low = min(p1, p2);
    int p_high = (u_root && high == u) ? u : ld_comp_cached(comp, high);
    u_root = false;
    if (p_high == high) {
      p_high = ld_comp(comp, high);
      if (p_high == high) {
        const int old = atomicCAS(comp + high, high, low);
        if (old == high) return;
        p_high = old;
      }
    }
    if (p_high == low) return;
    p1 = ld_comp_cached(comp, p_high);  // at or above high's parent
    p2 = ld_comp_cached(comp, low);
  }
}

__global__ void cc_init_kernel(int32_t n, int *comp) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += stride)
    comp[v] = static_cast<int>(v);
}

// One sampling round (src/cc.cc:100-106): vertex u links with its r-th
// out-neighbour.  Each thread takes two vertices per pass and loads both
// neighbour ids (random reads of the neighbour array, one HBM sector each)
// before either link, so two such reads are in flight per thread.
__global__ void cc_sample_kernel(int32_t n, const int32_t *__restrict__ off,
                                 const int32_t *__restrict__ nbr, int r, int *comp, int *err) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < n;
       u += 2 * stride) {
    const int64_t u2 = u + stride;
    const int s1 = off[u], e1 = off[u + 1];
    int s2 = 0, e2 = 0;
    if (u2 < n) {
      s2 = off[u2];
      e2 = off[u2 + 1];
    }
    const int v1 = s1 + r < e1 ? nbr[s1 + r] : -1;
    const int v2 = s2 + r < e2 ? nbr[s2 + r] : -1;
    if (v1 >= 0) cc_link(static_cast<int>(u), v1, comp, err);
    if (v2 >= 0) cc_link(static_cast<int>(u2), v2, comp, err);
  }
}

// src/cc.cc:58-66.  No link runs during a compress, so roots are fixed and
// every non-root x has comp[x] != x at all times: c == comp[c] holds exactly
// when c is a root, whether comp[c] was read fresh or from L1.
__global__ void cc_compress_kernel(int32_t n, int *comp, int *err) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += stride) {
    int it = 0;
    int c = ld_comp(comp, static_cast<int>(v));
    int cc = ld_comp_cached(comp, c);
    while (c != cc) {
      if (++it >= kChaseLimit) {
        atomicExch(err, 1);
        break;
      }
      comp[v] = cc;
      c = cc;
      cc = ld_comp_cached(comp, c);
    }
  }
}

// Final phase: out-neighbours from index `skip` on and, for a directed graph,
// all in-neighbours; vertices of component `giant` are skipped
// (src/cc.cc:122-146).  Rows [row0, row1), one warp per vertex (the long
// rows at the front of the degree-sorted mirror).
__global__ void cc_finish_warp_kernel(int32_t row0, int32_t row1, const int32_t *__restrict__ ooff,
                                      const int32_t *__restrict__ onbr,
                                      const int32_t *__restrict__ ioff,
                                      const int32_t *__restrict__ inbr, int skip, int giant,
                                      int *comp, int *err) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t u = row0 + ((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
       u < row1; u += warps) {
    if (ld_comp(comp, static_cast<int>(u)) == giant) continue;
    for (int j = ooff[u] + skip + lane; j < ooff[u + 1]; j += 32)
      cc_link(static_cast<int>(u), onbr[j], comp, err);
    if (ioff)
      for (int j = ioff[u] + lane; j < ioff[u + 1]; j += 32)
        cc_link(static_cast<int>(u), inbr[j], comp, err);
  }
}

// The same for rows [row0, row1), one thread per vertex (the short rows).
__global__ void cc_finish_thread_kernel(int32_t row0, int32_t row1,
                                        const int32_t *__restrict__ ooff,
                                        const int32_t *__restrict__ onbr,
                                        const int32_t *__restrict__ ioff,
                                        const int32_t *__restrict__ inbr, int skip, int giant,
                                        int *comp, int *err) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t u = row0 + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < row1;
       u += stride) {
    if (ld_comp(comp, static_cast<int>(u)) == giant) continue;
    for (int j = ooff[u] + skip; j < ooff[u + 1]; j++) cc_link(static_cast<int>(u), onbr[j], comp, err);
    if (ioff)
      for (int j = ioff[u]; j < ioff[u + 1]; j++) cc_link(static_cast<int>(u), inbr[j], comp, err);
  }
}

// The last compress, fused with the ids mapped back: every vertex chases
// to its root (as cc_compress_kernel) and offers its original id to the
// root's minimum.  Members of the component of row 0 (the largest one; half
// the graph on Kronecker inputs) are reduced per thread and per block first,
// so its root takes one atomic per block instead of one per vertex.
__global__ void __launch_bounds__(256) cc_compress_min_kernel(int32_t n, int *comp,
                                                              const int32_t *__restrict__ perm,
                                                              int *root_min, int *err) {
  __shared__ int s_min[8];
  const int giant = 0;  // row 0 is the root of its component
  int local = INT_MAX;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += stride) {
    int it = 0;
    int c = ld_comp(comp, static_cast<int>(v));
    int cc = ld_comp_cached(comp, c);
    while (c != cc) {
      if (++it >= kChaseLimit) {
        atomicExch(err, 1);
        break;
      }
      comp[v] = cc;
      c = cc;
      cc = ld_comp_cached(comp, c);
    }
    if (c == giant) local = min(local, perm[v]);
    else atomicMin(root_min + c, perm[v]);
  }
  local = static_cast<int>(__reduce_min_sync(0xffffffffu, static_cast<unsigned>(local)));
  if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    int m = INT_MAX;
    for (int w = 0; w < (blockDim.x >> 5); w++) m = min(m, s_min[w]);
    if (m != INT_MAX) atomicMin(root_min + giant, m);
  }
}

// Label of every original id o (a gather, so the writes are coalesced):
// rows [active, n) have no edges and are their own components.
__global__ void cc_label_kernel(int32_t n, int32_t active, const int *comp,
                                const int32_t *__restrict__ inv, const int *root_min,
                                int32_t *out_old) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t o = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; o < n; o += stride) {
    const int v = inv[o];
    // comp and root_min are final here (read-only path)
    out_old[o] = v < active ? __ldg(root_min + __ldg(comp + v)) : static_cast<int32_t>(o);
  }
}

__global__ void fill_kernel(int32_t n, int value, int *a) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    a[i] = value;
}

unsigned CcGrid(int64_t items) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((items + 255) / 256, sms * 16)));
}

}  // namespace

void FreeCcScratch(CcScratch *c) {
  for (int *p : {c->comp, c->root_min, c->err})
    if (p) cudaFree(p);
  c->comp = c->root_min = c->err = nullptr;
  c->cap = 0;
}

cudaError_t ConnectedComponents(const DeviceGraph &g, CcScratch &cs, cudaStream_t s,
                                int32_t *out_old, std::string *err) {
  const int32_t n = static_cast<int32_t>(g.n);
  // out-CSR in new ids: the shared CSR of an undirected graph, the
  // renumbered out-CSR of a directed one
  const int32_t *ooff = g.directed ? g.orowoff : g.rowoff;
  const int32_t *onbr = g.directed ? g.ocol : g.col;
  cudaError_t e = cudaSuccess;
  if (!cs.comp || cs.cap < n) {
    FreeCcScratch(&cs);
    e = cudaMalloc(&cs.comp, sizeof(int) * std::max<int64_t>(n, 1));
    if (e == cudaSuccess) e = cudaMalloc(&cs.root_min, sizeof(int) * std::max<int64_t>(n, 1));
    if (e == cudaSuccess) e = cudaMalloc(&cs.err, sizeof(int));
    if (e != cudaSuccess) {
      FreeCcScratch(&cs);
      *err = std::string("connected components: ") + cudaGetErrorString(e);
      return e;
    }
    cs.cap = n;
  }
  int *comp = cs.comp, *root_min = cs.root_min, *derr = cs.err;
  e = cudaMemsetAsync(derr, 0, sizeof(int), s);
  const unsigned grid = CcGrid(n);
  const int kRounds = 2;  // neighbor_rounds of src/cc.cc:92
  // Rows without in-neighbours form the tail of the mirror; in an undirected
  // graph they have no edges at all, so no link ever touches them and they
  // stay their own components: the link and compress passes stop before them.
  const int32_t active = g.directed ? n : static_cast<int32_t>(g.bin_row_start[kBinZero]);
  // rows of at least 32 entries (the front of the mirror) take a warp each
  const int32_t long_rows = std::min<int32_t>(active, static_cast<int32_t>(g.bin_row_start[4]));
  if (e == cudaSuccess) {
    cc_init_kernel<<<CcGrid(active), 256, 0, s>>>(active, comp);
    for (int r = 0; r < kRounds; r++) {
      cc_sample_kernel<<<CcGrid(active), 256, 0, s>>>(active, ooff, onbr, r, comp, derr);
      cc_compress_kernel<<<CcGrid(active), 256, 0, s>>>(active, comp, derr);
    }
    e = cudaGetLastError();
  }
  const int giant = 0;  // the root, and label, of row 0's component
  if (e == cudaSuccess) {
    const int32_t *ioff = g.directed ? g.rowoff : nullptr;
    const int32_t *inbr = g.directed ? g.col : nullptr;
    if (long_rows > 0)
      cc_finish_warp_kernel<<<CcGrid(static_cast<int64_t>(long_rows) * 32), 256, 0, s>>>(
          0, long_rows, ooff, onbr, ioff, inbr, kRounds, giant, comp, derr);
    if (active > long_rows)
      cc_finish_thread_kernel<<<CcGrid(active - long_rows), 256, 0, s>>>(
          long_rows, active, ooff, onbr, ioff, inbr, kRounds, giant, comp, derr);
    // roots of the rows [0, active) are rows of [0, active)
    fill_kernel<<<CcGrid(active), 256, 0, s>>>(active, INT_MAX, root_min);
    cc_compress_min_kernel<<<CcGrid(active), 256, 0, s>>>(active, comp, g.perm, root_min, derr);
    cc_label_kernel<<<grid, 256, 0, s>>>(n, active, comp, g.inv, root_min, out_old);
    e = cudaGetLastError();
  }
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    *err = std::string("connected components: ") + cudaGetErrorString(e);
    return e;
  }
  if (herr) {
    *err = "connected components: link or compress exceeded its iteration limit";
    return cudaErrorUnknown;
  }
  return cudaSuccess;
}

}  // namespace prgpu
