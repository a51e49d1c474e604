// pr_gpu.cu -- the C ABI (include/pr_gpu.h): handle, upload, solve.
#include "pr_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"
#include "batched.h"
#include "blocked.h"

using prgpu::DeviceGraph;
using prgpu::Scratch;

struct pr_gpu {
  int device = 0;
  cudaStream_t stream = nullptr;      // stream in use
  cudaStream_t own_stream = nullptr;  // created by pr_gpu_create
  std::string err;
  DeviceGraph g;
  bool has_graph = false;
  Scratch sc;
  prgpu::BatchScratch bsc;
  prgpu::LoopGraph loop_single;   // cached sweep-loop graphs
  prgpu::LoopGraph loop_adjoint;
  prgpu::LoopGraph loop_blocked;
  // slice-blocked layout of the uploaded graph (built at upload unless the
  // layout is PR_GPU_SWEEP_GATHER) and the settings it was built with
  prgpu::SliceBlocks sb;
  int sweep_layout = PR_GPU_SWEEP_AUTO;
  int slice_verts = 0, bin_words = 0;
  bool sb_built = false;  // a build was attempted for the current graph and settings
  cudaEvent_t ev[4] = {};
  double last_sweep_ms = 0, last_total_ms = 0;
  int64_t last_launches = 0;
  int last_adjoint_sweeps = 0;
  bool last_blocked = false;
  // pr_gpu_sweep_kernel_times: per-kernel events of one timed solve and the
  // average device ms per sweep of each kernel of the sweep body
  bool time_kernels = false;
  std::vector<cudaEvent_t> kev;
  double kernel_ms[3] = {0, 0, 0};
  int kernel_n = 0;
  // pinned staging for host <-> device copies
  static constexpr size_t kChunk = 32u << 20;
  void *pinned[2] = {nullptr, nullptr};
  cudaEvent_t pin_ev[2] = {};
  // CSR of the last pr_gpu_generate (original ids), kept for download
  int32_t *gen_off = nullptr, *gen_nbr = nullptr;
  int64_t gen_n = 0, gen_m = 0;
  prgpu::CcScratch cc;    // connected-components work arrays
  prgpu::BfsScratch bfs;  // breadth-first-search work arrays
};

namespace {

int SetErr(pr_gpu_t *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  return code;
}

int CudaErr(pr_gpu_t *h, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return PR_GPU_OK;
  const int code = (e == cudaErrorMemoryAllocation) ? PR_GPU_ENOMEM : PR_GPU_ECUDA;
  return SetErr(h, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PR_CHECK(h, expr)                                   \
  do {                                                      \
    cudaError_t e_ = (expr);                                \
    if (e_ != cudaSuccess) return CudaErr((h), e_, #expr);  \
  } while (0)

// Parallel memcpy for the host-to-host staging copies: a process-wide pool of
// worker threads, started once (a staging chunk is copied in well under a
// millisecond, so starting threads per chunk would cost as much as the copy).
// One copy runs at a time; the caller copies the first share itself.  The
// pool is never destroyed: its idle workers end with the process.
class CopyPool {
 public:
  static CopyPool &Get() {
    static CopyPool *pool = new CopyPool();
    return *pool;
  }

  void Copy(void *dst, const void *src, size_t bytes) {
    std::lock_guard<std::mutex> one_at_a_time(call_mu_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      dst_ = static_cast<char *>(dst);
      src_ = static_cast<const char *>(src);
      bytes_ = bytes;
      pending_ = nt_ - 1;
      gen_++;
    }
    work_cv_.notify_all();
    Share(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return pending_ == 0; });
  }

 private:
  CopyPool() : nt_(Threads()) {
    for (int t = 1; t < nt_; t++) std::thread([this, t] { Worker(t); }).detach();
  }

  // half the hardware threads, at most 8 (GAPBS_PR_COPY_THREADS overrides;
  // on a 16-core host 16 or 24 threads staged a 4.3 GB CSR more slowly than
  // 8: the copy is bound by host memory bandwidth)
  static int Threads() {
    const char *v = std::getenv("GAPBS_PR_COPY_THREADS");
    if (v && *v) return static_cast<int>(std::max(1L, std::min(64L, std::strtol(v, nullptr, 10))));
    return static_cast<int>(std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2)));
  }

  void Share(int t) const {
    const size_t per = (bytes_ + nt_ - 1) / nt_;
    const size_t lo = std::min(bytes_, per * t), hi = std::min(bytes_, per * (t + 1));
    if (hi > lo) std::memcpy(dst_ + lo, src_ + lo, hi - lo);
  }

  void Worker(int t) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        work_cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
      }
      Share(t);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) done_cv_.notify_one();
    }
  }

  const int nt_;
  std::mutex call_mu_, mu_;
  std::condition_variable work_cv_, done_cv_;
  uint64_t gen_ = 0;
  int pending_ = 0;
  char *dst_ = nullptr;
  const char *src_ = nullptr;
  size_t bytes_ = 0;
};

void HostCopy(void *dst, const void *src, size_t bytes) {
  if (bytes < (size_t(8) << 20)) {
    std::memcpy(dst, src, bytes);
    return;
  }
  CopyPool::Get().Copy(dst, src, bytes);
}

void FreeGenerated(pr_gpu_t *h) {
  if (h->gen_off) cudaFree(h->gen_off);
  if (h->gen_nbr) cudaFree(h->gen_nbr);
  h->gen_off = h->gen_nbr = nullptr;
  h->gen_n = h->gen_m = 0;
}

int EnsurePinned(pr_gpu_t *h) {
  for (int i = 0; i < 2; i++) {
    if (!h->pinned[i]) {
      PR_CHECK(h, cudaMallocHost(&h->pinned[i], pr_gpu::kChunk));
      PR_CHECK(h, cudaEventCreateWithFlags(&h->pin_ev[i], cudaEventDisableTiming));
    }
  }
  return PR_GPU_OK;
}

// True when [p, p + bytes) starts and ends in page-locked host memory
// (cudaMallocHost, cudaHostRegister, torch pin_memory): such buffers are
// copied by DMA directly, without the staging chunks.
bool PageLocked(const void *p, size_t bytes) {
  cudaPointerAttributes a0, a1;
  if (cudaPointerGetAttributes(&a0, p) != cudaSuccess ||
      cudaPointerGetAttributes(&a1, static_cast<const char *>(p) + bytes - 1) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a0.type == cudaMemoryTypeHost && a1.type == cudaMemoryTypeHost;
}

// Host -> device: page-locked sources by one DMA; others through two pinned
// chunks (host copy of chunk k+1 overlaps the DMA of chunk k).
int CopyToDevice(pr_gpu_t *h, void *dst, const void *src, size_t bytes) {
  if (bytes == 0) return PR_GPU_OK;
  if (PageLocked(src, bytes)) {
    PR_CHECK(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream));
    PR_CHECK(h, cudaStreamSynchronize(h->stream));
    return PR_GPU_OK;
  }
  int rc = EnsurePinned(h);
  if (rc) return rc;
  size_t off = 0;
  int k = 0;
  while (off < bytes) {
    const size_t len = std::min(pr_gpu::kChunk, bytes - off);
    PR_CHECK(h, cudaEventSynchronize(h->pin_ev[k]));
    HostCopy(h->pinned[k], static_cast<const char *>(src) + off, len);
    PR_CHECK(h, cudaMemcpyAsync(static_cast<char *>(dst) + off, h->pinned[k], len,
                                cudaMemcpyHostToDevice, h->stream));
    PR_CHECK(h, cudaEventRecord(h->pin_ev[k], h->stream));
    off += len;
    k ^= 1;
  }
  PR_CHECK(h, cudaStreamSynchronize(h->stream));
  return PR_GPU_OK;
}

// Device -> host: page-locked destinations by one DMA; others through the
// pinned chunks.
int CopyToHost(pr_gpu_t *h, void *dst, const void *src, size_t bytes) {
  if (bytes == 0) return PR_GPU_OK;
  if (PageLocked(dst, bytes)) {
    PR_CHECK(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream));
    PR_CHECK(h, cudaStreamSynchronize(h->stream));
    return PR_GPU_OK;
  }
  int rc = EnsurePinned(h);
  if (rc) return rc;
  size_t off = 0, pend_off = 0, pend_len = 0;
  int k = 0, pend_k = -1;
  while (off < bytes) {
    const size_t len = std::min(pr_gpu::kChunk, bytes - off);
    PR_CHECK(h, cudaMemcpyAsync(h->pinned[k], static_cast<const char *>(src) + off, len,
                                cudaMemcpyDeviceToHost, h->stream));
    PR_CHECK(h, cudaEventRecord(h->pin_ev[k], h->stream));
    if (pend_k >= 0) {
      PR_CHECK(h, cudaEventSynchronize(h->pin_ev[pend_k]));
      HostCopy(static_cast<char *>(dst) + pend_off, h->pinned[pend_k], pend_len);
    }
    pend_k = k;
    pend_off = off;
    pend_len = len;
    off += len;
    k ^= 1;
  }
  PR_CHECK(h, cudaEventSynchronize(h->pin_ev[pend_k]));
  HostCopy(static_cast<char *>(dst) + pend_off, h->pinned[pend_k], pend_len);
  return PR_GPU_OK;
}

template <typename T>
cudaError_t Grow(T **p, int64_t *cap, int64_t need) {
  if (*p && *cap >= need) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<int64_t>(need, 1));
  if (e == cudaSuccess) *cap = need;
  return e;
}

void FreeScratch(Scratch *sc) {
  void *ptrs[] = {sc->score, sc->contrib[0], sc->contrib[1], sc->base, sc->outbuf, sc->tele,
                  sc->aux[0], sc->aux[1], sc->edge_buf, sc->norm,
                  sc->part1, sc->part2, sc->tick1, sc->trace, sc->ctl};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  *sc = Scratch();
}

// Scratch for an n-vertex, ncols-column solve of nblocks blocks and iters sweeps.
int EnsureScratch(pr_gpu_t *h, int64_t n, int ncols, int64_t nblocks, int iters) {
  Scratch &s = h->sc;
  const int64_t cells = n * ncols;
  if (!s.score || s.cap_n < cells) {
    for (float **p : {&s.score, &s.contrib[0], &s.contrib[1], &s.base, &s.outbuf, &s.tele,
                      &s.aux[0], &s.aux[1]}) {
      if (*p) cudaFree(*p);
      *p = nullptr;
    }
    s.cap_n = 0;
    for (float **p : {&s.score, &s.contrib[0], &s.contrib[1], &s.base, &s.outbuf, &s.tele,
                      &s.aux[0], &s.aux[1]})
      PR_CHECK(h, cudaMalloc(p, sizeof(float) * std::max<int64_t>(cells, 1)));
    s.cap_n = cells;
  }
  int64_t cap = s.cap_blocks;
  const int64_t ngroups = (nblocks + prgpu::kReduceGroup - 1) / prgpu::kReduceGroup;
  if (!s.part1 || cap < nblocks) {
    int64_t c1 = 0, c2 = 0, c3 = 0;
    if (s.part1) cudaFree(s.part1), s.part1 = nullptr;
    if (s.part2) cudaFree(s.part2), s.part2 = nullptr;
    if (s.tick1) cudaFree(s.tick1), s.tick1 = nullptr;
    PR_CHECK(h, Grow(&s.part1, &c1, nblocks));
    PR_CHECK(h, Grow(&s.part2, &c2, ngroups + 1));
    PR_CHECK(h, Grow(&s.tick1, &c3, ngroups + 1));
    s.cap_blocks = nblocks;
  }
  PR_CHECK(h, Grow(&s.trace, &s.cap_iters, std::max(iters, 1)));
  if (!s.ctl) PR_CHECK(h, cudaMalloc(&s.ctl, sizeof(prgpu::SweepCtl)));
  if (!s.norm) PR_CHECK(h, cudaMalloc(&s.norm, sizeof(double)));
  return PR_GPU_OK;
}

int CheckRunArgs(pr_gpu_t *h, int max_iters, int ncols) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return SetErr(h, PR_GPU_ENOGRAPH, "no graph uploaded");
  if (max_iters < 0) return SetErr(h, PR_GPU_EINVAL, "max_iters must be >= 0");
  if (ncols < 1) return SetErr(h, PR_GPU_EINVAL, "ncols must be >= 1");
  return PR_GPU_OK;
}

constexpr int64_t kAutoBlockedMinEdges = int64_t(48) << 20;

// Builds the slice-blocked layout of the current graph when the layout
// setting asks for it.  Under PR_GPU_SWEEP_AUTO a graph of fewer than 48 Mi
// edges, a graph outside the layout's limits, a device without room for
// it, or a graph whose in-edges hardly
// share (row, slice) pairs (more pairs than half the edges: one partial
// written and read per edge costs more than the gather it replaces, as on
// uniform random graphs) keeps the gather sweep.
int EnsureSliceBlocks(pr_gpu_t *h) {
  if (h->sb_built || h->sweep_layout == PR_GPU_SWEEP_GATHER || !h->has_graph) return PR_GPU_OK;
  h->sb_built = true;
  h->loop_blocked.Reset();
  std::string msg;
  // below about 48 M edges the gather sweep's contribs stay in L1 and L2
  // (measured: g20, 31 M edges, 0.117 against 0.125 ms per sweep; g21,
  // 64 M edges, 0.200 against 0.157)
  if (h->sweep_layout == PR_GPU_SWEEP_AUTO && h->g.m < kAutoBlockedMinEdges) return PR_GPU_OK;
  const int64_t max_pairs = h->sweep_layout == PR_GPU_SWEEP_AUTO
                                ? h->g.m / 2
                                : std::numeric_limits<int64_t>::max();
  cudaError_t e = prgpu::BuildSliceBlocks(h->g, h->slice_verts, h->bin_words, max_pairs, &h->sb,
                                          h->stream, &msg);
  if (e == cudaSuccess) return PR_GPU_OK;
  cudaGetLastError();
  if (h->sweep_layout == PR_GPU_SWEEP_AUTO && e == cudaErrorMemoryAllocation) return PR_GPU_OK;
  return SetErr(h, e == cudaErrorMemoryAllocation ? PR_GPU_ENOMEM : PR_GPU_ECUDA, msg);
}

// Drops everything derived from the uploaded graph before a new one arrives.
void DropGraph(pr_gpu_t *h) {
  h->has_graph = false;
  prgpu::FreeSliceBlocks(&h->sb);
  h->sb_built = false;
  h->loop_blocked.Reset();
  prgpu::FreeDeviceGraph(&h->g);
}

bool UseBlocked(const pr_gpu_t *h) {
  return h->sweep_layout != PR_GPU_SWEEP_GATHER && h->sb.ready && !h->g.weighted;
}

// Single-column solve on device buffers.  tele_old: teleport in original ids
// (device) or nullptr for the reference's uniform PageRank.  out_old: device
// buffer for scores in original ids.
int SolveSingle(pr_gpu_t *h, int max_iters, double epsilon, float damping,
                const float *tele_old, float *out_old, int32_t *sweeps_out, double *err_trace) {
  DeviceGraph &g = h->g;
  int rc = EnsureSliceBlocks(h);
  if (rc) return rc;
  if (h->sweep_layout == PR_GPU_SWEEP_BLOCKED && !UseBlocked(h))
    return SetErr(h, PR_GPU_EINVAL,
                  "the slice-blocked sweep does not fit this graph (weighted, no edges, or more "
                  "source slices than a bin holds)");
  const bool blocked = UseBlocked(h);
  int32_t task_start[prgpu::kNumBins + 1];
  prgpu::PullTasks(g, task_start);
  prgpu::PullArgs probe;
  std::memset(&probe, 0, sizeof(probe));
  probe.kind = tele_old ? prgpu::kKindPPR : prgpu::kKindPlain;
  probe.win = g.weighted ? g.win : nullptr;
  probe.odeg = (g.directed && !g.weighted) ? g.odeg : nullptr;
  const void *sweep_fn = prgpu::PullSweepKernel(probe);
  const int nblocks = blocked ? prgpu::BinRowGrid(h->sb, g.n) : prgpu::PullGrid(sweep_fn);
  rc = EnsureScratch(h, g.n, 1, nblocks, max_iters);
  if (rc) return rc;
  Scratch &sc = h->sc;
  cudaStream_t s = h->stream;
  int64_t launches = 0;
  PR_CHECK(h, cudaEventRecord(h->ev[0], s));
  const float *tele_new = nullptr;
  if (tele_old) {
    PR_CHECK(h, prgpu::LaunchScatterIn(g, tele_old, sc.contrib[1], 1, s));
    tele_new = sc.contrib[1];
    launches++;
  }
  const float n_f = static_cast<float>(g.n);
  const float init_score = 1.0f / n_f;                 // src/pr_spmv.cc:37
  const float base_score = (1.0f - damping) / n_f;     // src/pr_spmv.cc:38
  PR_CHECK(h, prgpu::LaunchResetCtl(sc, nblocks, max_iters, s));
  PR_CHECK(h, prgpu::LaunchPullInit(g, sc, tele_new, init_score, damping, s));
  launches++;
  prgpu::PullArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = static_cast<int32_t>(g.n);
  a.rowoff = g.rowoff;
  a.col = g.col;
  a.win = g.weighted ? g.win : nullptr;
  a.odeg = (g.directed && !g.weighted) ? g.odeg : nullptr;
  a.rsum = g.weighted ? g.rsum : nullptr;
  a.kind = tele_old ? prgpu::kKindPPR : prgpu::kKindPlain;
  a.base_vec = tele_old ? sc.base : nullptr;
  a.base_scalar = base_score;
  a.damping = damping;
  a.score = sc.score;
  for (int b = 0; b <= prgpu::kNumBins; b++) {
    a.task_start[b] = task_start[b];
    a.bin_row[b] = static_cast<int32_t>(g.bin_row_start[b]);
  }
  a.nseg = static_cast<int32_t>(g.num_segments);
  a.seg_row = g.seg_row;
  a.seg_first = g.seg_first;
  a.hub_ticket = g.hub_ticket;
  a.seg_partial = g.seg_partial;
  a.part1 = sc.part1;
  a.part2 = sc.part2;
  a.tick1 = sc.tick1;
  a.trace = sc.trace;
  a.ctl = sc.ctl;
  a.nblocks = nblocks;
  a.l1_rows = static_cast<int32_t>(std::min<int64_t>(g.n, prgpu::kL1HubBytes / 4));
  a.zero_final_sweep = g.directed ? 2 : 1;
  a.epsilon = epsilon;
  a.c0 = sc.contrib[0];
  a.c1 = sc.contrib[1];
  prgpu::BlockedArgs ba;
  prgpu::SweepKernel body[3];
  if (blocked) {
    const prgpu::SliceBlocks &sb = h->sb;
    std::memset(&ba, 0, sizeof(ba));
    ba.src = sb.src;
    ba.run = sb.run;
    ba.seg = sb.seg;
    ba.unit = sb.unit;
    ba.nunits_flat = sb.nunits_flat;
    ba.nunits = sb.nunits;
    ba.dest = sb.dest;
    ba.slice_verts = sb.slice_verts;
    ba.nsrc = sb.nsrc;
    ba.part = sb.part;
    ba.part_len = sb.part_len;
    ba.bin_words = sb.bin_words;
    ba.binbase = sb.binbase;
    ba.idx = sb.idx;
    ba.rowq = sb.rowq;
    ba.bin = sb.bin;
    ba.nbins = sb.nbins;
    ba.n = static_cast<int32_t>(g.n);
    ba.ndst = sb.ndst;
    ba.zero_blocks = nblocks - sb.nbins;
    ba.kind = a.kind;
    ba.rowoff = g.rowoff;
    ba.odeg = g.directed ? g.odeg : nullptr;
    ba.base_vec = a.base_vec;
    ba.base_scalar = a.base_scalar;
    ba.damping = damping;
    ba.score = sc.score;
    ba.contrib = sc.contrib[0];
    ba.part1 = sc.part1;
    ba.part2 = sc.part2;
    ba.tick1 = sc.tick1;
    ba.trace = sc.trace;
    ba.ctl = sc.ctl;
    ba.nblocks = nblocks;
    ba.epsilon = epsilon;
    const void *kf = prgpu::SlicePartialKernel(true), *kr = prgpu::SlicePartialKernel(false);
    const void *kb = prgpu::BinRowKernel(sb);
    for (const void *k : {kf, kr})
      PR_CHECK(h, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(prgpu::SliceSmemBytes(sb))));
    PR_CHECK(h, cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(prgpu::BinSmemBytes(sb))));
    for (int i = 0; i < 3; i++) {
      body[i].fn = i == 0 ? kf : (i == 1 ? kr : kb);
      body[i].grid = dim3(i < 2 ? sb.nctas : nblocks);
      body[i].block = dim3(i < 2 ? prgpu::kSliceThreads : prgpu::BinRowThreads(sb));
      body[i].smem = i < 2 ? prgpu::SliceSmemBytes(sb) : prgpu::BinSmemBytes(sb);
      body[i].args = &ba;
      body[i].args_size = sizeof(ba);
    }
  }
  PR_CHECK(h, cudaEventRecord(h->ev[1], s));
  prgpu::SweepKernel gather_body;
  gather_body.fn = sweep_fn;
  gather_body.grid = dim3(nblocks);
  gather_body.block = dim3(prgpu::kSweepThreads);
  gather_body.args = &a;
  gather_body.args_size = sizeof(a);
  const prgpu::SweepKernel *tk = blocked ? body : &gather_body;
  const int tnk = blocked ? 3 : 1;
  const bool timed = h->time_kernels && max_iters > 0 && (blocked || nblocks > 0);
  if (timed) {
    const size_t need = static_cast<size_t>(max_iters) * (tnk + 1);
    while (h->kev.size() < need) {
      cudaEvent_t e = nullptr;
      PR_CHECK(h, cudaEventCreate(&e));
      h->kev.push_back(e);
    }
    PR_CHECK(h, prgpu::LoopGraph::LaunchTimed(tk, tnk, &sc.ctl->loop, max_iters, s,
                                              h->kev.data()));
  } else if (blocked)
    PR_CHECK(h, h->loop_blocked.Launch(body, 3, &sc.ctl->loop, max_iters, s));
  else if (nblocks > 0)
    PR_CHECK(h, h->loop_single.Launch(sweep_fn, dim3(nblocks),
                                      dim3(prgpu::kSweepThreads), &a, sizeof(a), &sc.ctl->loop,
                                      max_iters, s));
  PR_CHECK(h, cudaEventRecord(h->ev[2], s));
  PR_CHECK(h, prgpu::LaunchGatherOut(g, sc.score, out_old, 1, s));
  launches++;
  PR_CHECK(h, cudaEventRecord(h->ev[3], s));
  prgpu::SweepCtl ctl;
  std::vector<double> trace(std::max(max_iters, 1));
  PR_CHECK(h, cudaMemcpyAsync(&ctl, sc.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, s));
  if (max_iters)
    PR_CHECK(h, cudaMemcpyAsync(trace.data(), sc.trace, sizeof(double) * max_iters,
                                cudaMemcpyDeviceToHost, s));
  PR_CHECK(h, cudaStreamSynchronize(s));
  float ms_sweep = 0, ms_total = 0;
  cudaEventElapsedTime(&ms_sweep, h->ev[1], h->ev[2]);
  cudaEventElapsedTime(&ms_total, h->ev[0], h->ev[3]);
  h->last_sweep_ms = ms_sweep;
  h->last_total_ms = ms_total;
  if (timed) {
    // the sweeps that ran: every one counted by the loop, none after it
    const int ran = std::min(ctl.loop.loops, max_iters);
    h->kernel_n = tnk;
    for (int k = 0; k < tnk; k++) {
      double sum = 0;
      for (int i = 0; i < ran; i++) {
        float t = 0;
        PR_CHECK(h, cudaEventElapsedTime(&t, h->kev[i * (tnk + 1) + k],
                                         h->kev[i * (tnk + 1) + k + 1]));
        sum += t;
      }
      h->kernel_ms[k] = ran ? sum / ran : 0.0;
    }
  }
  // per sweep: the sweep kernel(s) + the decide kernel
  h->last_launches = launches + (blocked ? 4 : 2) * static_cast<int64_t>(ctl.loop.loops);
  h->last_blocked = blocked;
  if (sweeps_out) *sweeps_out = max_iters ? ctl.sweeps : 0;
  if (err_trace)
    for (int i = 0; i < max_iters; i++) err_trace[i] = trace[i];
  return PR_GPU_OK;
}


// Adjoint solve on device buffers (original ids in, original ids out).
int SolveAdjoint(pr_gpu_t *h, int max_iters, double epsilon, float damping, const float *w_old,
                 const float *s_old, float *grad_t_old, float *grad_ew) {
  DeviceGraph &g = h->g;
  int32_t task_start[prgpu::kNumBins + 1];
  prgpu::PullTasks(g, task_start);
  const bool generic = g.directed;
  prgpu::PullArgs probe;
  std::memset(&probe, 0, sizeof(probe));
  probe.kind = prgpu::kKindAdjoint;
  probe.win = g.weighted ? g.wout : nullptr;
  const void *adj_fn = generic ? prgpu::PullGenericKernel(probe) : prgpu::PullSweepKernel(probe);
  const int nblocks = prgpu::PullGrid(adj_fn);
  int rc = EnsureScratch(h, g.n, 1, nblocks, max_iters);
  if (rc) return rc;
  Scratch &sc = h->sc;
  cudaStream_t s = h->stream;
  int64_t launches = 0;
  PR_CHECK(h, cudaEventRecord(h->ev[0], s));
  // w and s in new ids; lambda_0 = w
  PR_CHECK(h, prgpu::LaunchScatterIn(g, w_old, sc.base, 1, s));
  PR_CHECK(h, prgpu::LaunchScatterIn(g, s_old, sc.aux[0], 1, s));
  PR_CHECK(h, prgpu::LaunchL1Norm(w_old, g.n, sc.norm, s));
  launches += 3;
  PR_CHECK(h, cudaMemcpyAsync(sc.score, sc.base, sizeof(float) * g.n, cudaMemcpyDeviceToDevice, s));
  PR_CHECK(h, cudaMemcpyAsync(sc.contrib[0], sc.base, sizeof(float) * g.n, cudaMemcpyDeviceToDevice, s));
  double wnorm = 0;
  PR_CHECK(h, cudaMemcpyAsync(&wnorm, sc.norm, sizeof(double), cudaMemcpyDeviceToHost, s));
  PR_CHECK(h, cudaStreamSynchronize(s));
  PR_CHECK(h, prgpu::LaunchResetCtl(sc, nblocks, max_iters, s));
  const int32_t *orow = generic ? g.orowoff : g.rowoff;
  const int32_t *ocol = generic ? g.ocol : g.col;
  prgpu::PullArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = static_cast<int32_t>(g.n);
  a.kind = prgpu::kKindAdjoint;
  a.rowoff = orow;
  a.col = ocol;
  a.win = g.weighted ? g.wout : nullptr;
  a.odeg = nullptr;
  a.rsum = g.weighted ? g.rsum : nullptr;
  a.base_vec = sc.base;
  a.damping = damping;
  a.score = sc.score;
  if (!generic) {
    for (int b = 0; b <= prgpu::kNumBins; b++) {
      a.task_start[b] = task_start[b];
      a.bin_row[b] = static_cast<int32_t>(g.bin_row_start[b]);
    }
    a.nseg = static_cast<int32_t>(g.num_segments);
    a.seg_row = g.seg_row;
    a.seg_first = g.seg_first;
    a.hub_ticket = g.hub_ticket;
    a.seg_partial = g.seg_partial;
  }
  a.part1 = sc.part1;
  a.part2 = sc.part2;
  a.tick1 = sc.tick1;
  a.trace = sc.trace;
  a.ctl = sc.ctl;
  a.nblocks = nblocks;
  a.l1_rows = static_cast<int32_t>(std::min<int64_t>(g.n, prgpu::kL1HubBytes / 4));
  a.zero_final_sweep = 1;  // bins path: undirected only
  a.epsilon = epsilon * wnorm;
  a.c0 = sc.contrib[0];
  a.c1 = sc.contrib[1];
  PR_CHECK(h, cudaEventRecord(h->ev[1], s));
  if (nblocks > 0)
    PR_CHECK(h, h->loop_adjoint.Launch(adj_fn, dim3(nblocks), dim3(prgpu::kSweepThreads), &a, sizeof(a),
                                       &sc.ctl->loop, max_iters, s));
  PR_CHECK(h, cudaEventRecord(h->ev[2], s));
  PR_CHECK(h, prgpu::LaunchAdjointGrads(g, orow, ocol, g.weighted ? g.wout : nullptr, sc.score,
                                        sc.aux[0], damping, grad_ew, grad_t_old, s));
  launches += 2;
  PR_CHECK(h, cudaEventRecord(h->ev[3], s));
  prgpu::SweepCtl ctl;
  PR_CHECK(h, cudaMemcpyAsync(&ctl, sc.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, s));
  PR_CHECK(h, cudaStreamSynchronize(s));
  float ms_sweep = 0, ms_total = 0;
  cudaEventElapsedTime(&ms_sweep, h->ev[1], h->ev[2]);
  cudaEventElapsedTime(&ms_total, h->ev[0], h->ev[3]);
  h->last_sweep_ms = ms_sweep;
  h->last_total_ms = ms_total;
  h->last_launches = launches + 2 * static_cast<int64_t>(ctl.loop.loops);
  h->last_adjoint_sweeps = max_iters ? ctl.sweeps : 0;
  return PR_GPU_OK;
}
}  // namespace

extern "C" {

int pr_gpu_create(pr_gpu_t **out, int device) {
  if (!out) return PR_GPU_EINVAL;
  *out = nullptr;
  pr_gpu_t *h = new (std::nothrow) pr_gpu();
  if (!h) return PR_GPU_ENOMEM;
  h->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
  h->stream = h->own_stream;
  for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreate(&h->ev[i]);
  if (e != cudaSuccess) {
    delete h;
    return PR_GPU_ECUDA;
  }
  *out = h;
  return PR_GPU_OK;
}

void pr_gpu_destroy(pr_gpu_t *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  FreeGenerated(h);
  prgpu::FreeCcScratch(&h->cc);
  prgpu::FreeBfsScratch(&h->bfs);
  h->loop_single.Reset();
  h->loop_adjoint.Reset();
  DropGraph(h);
  FreeScratch(&h->sc);
  prgpu::FreeBatchScratch(&h->bsc);
  for (int i = 0; i < 2; i++) {
    if (h->pinned[i]) cudaFreeHost(h->pinned[i]);
    if (h->pin_ev[i]) cudaEventDestroy(h->pin_ev[i]);
  }
  for (auto &e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : h->kev)
    if (e) cudaEventDestroy(e);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

const char *pr_gpu_last_error(const pr_gpu_t *h) {
  return h ? h->err.c_str() : "invalid handle";
}

int pr_gpu_generate(pr_gpu_t *h, int uniform, int scale, int degree, const int32_t *perm,
                    int64_t *n_out, int64_t *m_out) {
  if (!h) return PR_GPU_EINVAL;
  if (scale < 1 || scale > 30 || degree < 0)
    return SetErr(h, PR_GPU_EINVAL, "need 1 <= scale <= 30 and degree >= 0");
  if ((int64_t(2) * degree) << scale > 0x7fffffffLL - 8)
    return SetErr(h, PR_GPU_ERANGE, "graph exceeds int32 offsets");
  if (!uniform && !perm) return SetErr(h, PR_GPU_EINVAL, "R-MAT needs the vertex permutation");
  PR_CHECK(h, cudaSetDevice(h->device));
  DropGraph(h);
  FreeGenerated(h);
  std::string msg;
  int64_t n = 0, m = 0;
  int32_t *off = nullptr, *nbr = nullptr;
  cudaError_t e = prgpu::GenerateGraph(uniform != 0, scale, degree, perm, h->stream, &n, &m, &off,
                                       &nbr, &msg);
  if (e != cudaSuccess)
    return SetErr(h, e == cudaErrorMemoryAllocation ? PR_GPU_ENOMEM : PR_GPU_ECUDA, msg);
  h->gen_off = off;
  h->gen_nbr = nbr;
  h->gen_n = n;
  h->gen_m = m;
  e = prgpu::BuildDeviceGraph(&h->g, n, m, off, nbr, off, nbr, nullptr, false, h->stream, &msg);
  if (e != cudaSuccess) {
    FreeGenerated(h);
    return SetErr(h, e == cudaErrorMemoryAllocation ? PR_GPU_ENOMEM : PR_GPU_ECUDA, msg);
  }
  h->has_graph = true;
  {
    const int brc = EnsureSliceBlocks(h);
    if (brc) return brc;
  }
  if (n_out) *n_out = n;
  if (m_out) *m_out = m;
  return PR_GPU_OK;
}

int pr_gpu_download_csr(pr_gpu_t *h, int64_t *out_off, int32_t *out_nbr) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->gen_off) return SetErr(h, PR_GPU_ENOGRAPH, "no generated graph to download");
  if (!out_off || (h->gen_m > 0 && !out_nbr)) return SetErr(h, PR_GPU_EINVAL, "null CSR array");
  PR_CHECK(h, cudaSetDevice(h->device));
  int64_t *off64 = nullptr;
  PR_CHECK(h, cudaMalloc(&off64, sizeof(int64_t) * (h->gen_n + 1)));
  prgpu::WidenOffsets(h->gen_n + 1, h->gen_off, off64, h->stream);
  cudaError_t e = cudaGetLastError();
  int rc = e == cudaSuccess ? PR_GPU_OK : CudaErr(h, e, "widen offsets");
  if (!rc) rc = CopyToHost(h, out_off, off64, sizeof(int64_t) * (h->gen_n + 1));
  if (!rc) rc = CopyToHost(h, out_nbr, h->gen_nbr, sizeof(int32_t) * h->gen_m);
  cudaFree(off64);
  if (!rc) FreeGenerated(h);
  return rc;
}

// Streams count elements of `elem` bytes from f to dst on the device through
// the two pinned chunks (the read of chunk k+1 overlaps the DMA of chunk k).
// narrow != nullptr: the elements are int64 offsets, DMA'd to `wide` (one
// chunk of device staging) and narrowed into narrow[] on the device, with
// *bad set for values outside [0, 2^31).
static int StreamFileToDevice(pr_gpu_t *h, FILE *f, int64_t count, size_t elem, void *dst,
                       int64_t *wide, int32_t *narrow, int *bad, const char *what) {
  int rc = EnsurePinned(h);
  if (rc) return rc;
  const size_t chunk = pr_gpu::kChunk / elem;
  int64_t done = 0;
  int k = 0;
  while (done < count) {
    const size_t len = static_cast<size_t>(std::min<int64_t>(chunk, count - done));
    PR_CHECK(h, cudaEventSynchronize(h->pin_ev[k]));
    if (std::fread(h->pinned[k], elem, len, f) != len)
      return SetErr(h, PR_GPU_EGRAPH, std::string("truncated serialized graph (") + what + ")");
    if (narrow) {
      // one device staging chunk: wait for the previous narrowing to finish
      PR_CHECK(h, cudaStreamSynchronize(h->stream));
      PR_CHECK(h, cudaMemcpyAsync(wide, h->pinned[k], len * elem, cudaMemcpyHostToDevice,
                                  h->stream));
      prgpu::NarrowOffsets(static_cast<int64_t>(len), wide, narrow + done, bad, h->stream);
      PR_CHECK(h, cudaGetLastError());
    } else {
      PR_CHECK(h, cudaMemcpyAsync(static_cast<char *>(dst) + done * elem, h->pinned[k], len * elem,
                                  cudaMemcpyHostToDevice, h->stream));
    }
    PR_CHECK(h, cudaEventRecord(h->pin_ev[k], h->stream));
    done += static_cast<int64_t>(len);
    k ^= 1;
  }
  return PR_GPU_OK;
}

int pr_gpu_upload_sg(pr_gpu_t *h, const char *path) {
  if (!h || !path) return PR_GPU_EINVAL;
  FILE *f = std::fopen(path, "rb");
  if (!f) return SetErr(h, PR_GPU_EINVAL, std::string("couldn't open file ") + path);
  unsigned char directed_byte = 0;
  int64_t entries = 0, n = 0;
  const bool header = std::fread(&directed_byte, 1, 1, f) == 1 &&
                      std::fread(&entries, sizeof(int64_t), 1, f) == 1 &&
                      std::fread(&n, sizeof(int64_t), 1, f) == 1;
  if (!header || n < 1 || entries < 0) {
    std::fclose(f);
    return SetErr(h, PR_GPU_EGRAPH, std::string("corrupt serialized graph ") + path);
  }
  if (n > 0x7fffffffLL - 1 || entries > 0x7fffffffLL - 8) {
    std::fclose(f);
    return SetErr(h, PR_GPU_ERANGE, "graph exceeds int32 ids / offsets");
  }
  const bool directed = directed_byte != 0;
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) {
    std::fclose(f);
    return CudaErr(h, e, "cudaSetDevice");
  }
  DropGraph(h);
  FreeGenerated(h);
  int32_t *d_oo = nullptr, *d_on = nullptr, *d_io = nullptr, *d_in = nullptr;
  int64_t *wide = nullptr;
  int *bad = nullptr;
  auto release = [&]() {
    cudaStreamSynchronize(h->stream);  // no copy into these buffers is in flight
    for (void *p : {static_cast<void *>(d_oo), static_cast<void *>(d_on),
                    static_cast<void *>(d_io), static_cast<void *>(d_in),
                    static_cast<void *>(wide), static_cast<void *>(bad)})
      if (p) cudaFree(p);
    std::fclose(f);
  };
  e = cudaMalloc(&d_oo, sizeof(int32_t) * (n + 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_on, sizeof(int32_t) * std::max<int64_t>(entries, 1));
  if (e == cudaSuccess && directed) e = cudaMalloc(&d_io, sizeof(int32_t) * (n + 1));
  if (e == cudaSuccess && directed)
    e = cudaMalloc(&d_in, sizeof(int32_t) * std::max<int64_t>(entries, 1));
  if (e == cudaSuccess) e = cudaMalloc(&wide, pr_gpu::kChunk);
  if (e == cudaSuccess) e = cudaMalloc(&bad, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), h->stream);
  if (e != cudaSuccess) {
    release();
    return CudaErr(h, e, "device allocation for upload");
  }
  int rc = StreamFileToDevice(h, f, n + 1, sizeof(int64_t), nullptr, wide, d_oo, bad, "offsets");
  if (!rc) rc = StreamFileToDevice(h, f, entries, sizeof(int32_t), d_on, nullptr, nullptr, nullptr,
                                   "neighbours");
  if (!rc && directed)
    rc = StreamFileToDevice(h, f, n + 1, sizeof(int64_t), nullptr, wide, d_io, bad, "offsets");
  if (!rc && directed)
    rc = StreamFileToDevice(h, f, entries, sizeof(int32_t), d_in, nullptr, nullptr, nullptr,
                            "neighbours");
  int hbad = 0;
  if (!rc) {
    e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = CudaErr(h, e, "reading the offsets check");
  }
  if (!rc && hbad) rc = SetErr(h, PR_GPU_EGRAPH, "invalid CSR: offsets outside int32");
  if (rc) {
    release();
    return rc;
  }
  std::string msg;
  e = prgpu::BuildDeviceGraph(&h->g, n, entries, d_oo, d_on, directed ? d_io : d_oo,
                              directed ? d_in : d_on, nullptr, directed, h->stream, &msg);
  release();
  if (e == cudaErrorInvalidValue && !msg.empty() && msg.rfind("invalid CSR", 0) == 0)
    return SetErr(h, PR_GPU_EGRAPH, msg);
  if (e != cudaSuccess) return SetErr(h, e == cudaErrorMemoryAllocation ? PR_GPU_ENOMEM : PR_GPU_ECUDA, msg);
  h->has_graph = true;
  return EnsureSliceBlocks(h);
}

int pr_gpu_connected_components_device(pr_gpu_t *h, int32_t *comp_out_dev) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return SetErr(h, PR_GPU_ENOGRAPH, "no graph uploaded");
  if (!comp_out_dev) return SetErr(h, PR_GPU_EINVAL, "comp_out is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  std::string msg;
  cudaError_t e = prgpu::ConnectedComponents(h->g, h->cc, h->stream, comp_out_dev, &msg);
  if (e != cudaSuccess) return SetErr(h, PR_GPU_ECUDA, msg);
  return PR_GPU_OK;
}

int pr_gpu_bfs_device(pr_gpu_t *h, int64_t source, int32_t *parent_out_dev,
                      pr_gpu_bfs_step_t *steps, int max_steps, int *nsteps) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return SetErr(h, PR_GPU_ENOGRAPH, "no graph uploaded");
  if (!parent_out_dev) return SetErr(h, PR_GPU_EINVAL, "parent_out is null");
  if (source < 0 || source >= h->g.n) return SetErr(h, PR_GPU_EINVAL, "source out of range");
  PR_CHECK(h, cudaSetDevice(h->device));
  std::string msg;
  std::vector<prgpu::BfsStep> log;
  int64_t total = 0;
  cudaError_t e = prgpu::BreadthFirstSearch(h->g, h->bfs, h->stream, static_cast<int>(source), 15,
                                            18, parent_out_dev, steps ? &log : nullptr, &total,
                                            &msg);
  if (e != cudaSuccess)
    return SetErr(h, e == cudaErrorMemoryAllocation ? PR_GPU_ENOMEM : PR_GPU_ECUDA, msg);
  int k = 0;
  for (const prgpu::BfsStep &st : log) {
    if (!steps || k >= max_steps) break;
    std::memset(steps[k].kind, 0, sizeof(steps[k].kind));
    std::strncpy(steps[k].kind, st.kind, sizeof(steps[k].kind) - 1);
    steps[k].count = st.count;
    steps[k].seconds = st.seconds;
    k++;
  }
  if (nsteps) *nsteps = static_cast<int>(total);
  return PR_GPU_OK;
}

int pr_gpu_bfs(pr_gpu_t *h, int64_t source, int32_t *parent_out, pr_gpu_bfs_step_t *steps,
               int max_steps, int *nsteps) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return SetErr(h, PR_GPU_ENOGRAPH, "no graph uploaded");
  if (!parent_out) return SetErr(h, PR_GPU_EINVAL, "parent_out is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  int32_t *d = nullptr;
  PR_CHECK(h, cudaMalloc(&d, sizeof(int32_t) * h->g.n));
  int rc = pr_gpu_bfs_device(h, source, d, steps, max_steps, nsteps);
  if (!rc) rc = CopyToHost(h, parent_out, d, sizeof(int32_t) * h->g.n);
  cudaFree(d);
  return rc;
}

int pr_gpu_connected_components(pr_gpu_t *h, int32_t *comp_out) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return SetErr(h, PR_GPU_ENOGRAPH, "no graph uploaded");
  if (!comp_out) return SetErr(h, PR_GPU_EINVAL, "comp_out is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  int32_t *d = nullptr;
  PR_CHECK(h, cudaMalloc(&d, sizeof(int32_t) * h->g.n));
  int rc = pr_gpu_connected_components_device(h, d);
  if (!rc) rc = CopyToHost(h, comp_out, d, sizeof(int32_t) * h->g.n);
  cudaFree(d);
  return rc;
}

int pr_gpu_upload(pr_gpu_t *h, int64_t n, int64_t m, const int32_t *out_off,
                  const int32_t *out_nbr, const int32_t *in_off, const int32_t *in_nbr,
                  const float *edge_w) {
  if (!h) return PR_GPU_EINVAL;
  if (n < 1 || m < 0) return SetErr(h, PR_GPU_EINVAL, "need n >= 1 and m >= 0");
  if (n > 0x7fffffffLL - 1 || m > 0x7fffffffLL - 8)
    return SetErr(h, PR_GPU_ERANGE, "graph exceeds int32 ids / offsets");
  if (!out_off || (m > 0 && !out_nbr)) return SetErr(h, PR_GPU_EINVAL, "null CSR array");
  const bool directed = in_off && (in_off != out_off || in_nbr != out_nbr);
  if (directed && m > 0 && !in_nbr) return SetErr(h, PR_GPU_EINVAL, "null in-CSR array");
  PR_CHECK(h, cudaSetDevice(h->device));
  DropGraph(h);
  FreeGenerated(h);
  int32_t *d_oo = nullptr, *d_on = nullptr, *d_io = nullptr, *d_in = nullptr;
  float *d_w = nullptr;
  auto release = [&]() {
    for (void *p : {static_cast<void *>(d_oo), static_cast<void *>(d_on),
                    static_cast<void *>(d_io), static_cast<void *>(d_in),
                    static_cast<void *>(d_w)})
      if (p) cudaFree(p);
  };
  cudaError_t e = cudaMalloc(&d_oo, sizeof(int32_t) * (n + 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_on, sizeof(int32_t) * std::max<int64_t>(m, 1));
  if (e == cudaSuccess && directed) e = cudaMalloc(&d_io, sizeof(int32_t) * (n + 1));
  if (e == cudaSuccess && directed) e = cudaMalloc(&d_in, sizeof(int32_t) * std::max<int64_t>(m, 1));
  if (e == cudaSuccess && edge_w) e = cudaMalloc(&d_w, sizeof(float) * std::max<int64_t>(m, 1));
  if (e != cudaSuccess) {
    release();
    return CudaErr(h, e, "device allocation for upload");
  }
  int rc = CopyToDevice(h, d_oo, out_off, sizeof(int32_t) * (n + 1));
  if (!rc) rc = CopyToDevice(h, d_on, out_nbr, sizeof(int32_t) * m);
  if (!rc && directed) rc = CopyToDevice(h, d_io, in_off, sizeof(int32_t) * (n + 1));
  if (!rc && directed) rc = CopyToDevice(h, d_in, in_nbr, sizeof(int32_t) * m);
  if (!rc && edge_w) rc = CopyToDevice(h, d_w, edge_w, sizeof(float) * m);
  if (rc) {
    release();
    return rc;
  }
  std::string msg;
  e = prgpu::BuildDeviceGraph(&h->g, n, m, d_oo, d_on, directed ? d_io : d_oo,
                              directed ? d_in : d_on, d_w, directed, h->stream, &msg);
  release();
  if (e == cudaErrorInvalidValue && !msg.empty() && msg.rfind("invalid CSR", 0) == 0)
    return SetErr(h, PR_GPU_EGRAPH, msg);
  if (e != cudaSuccess) return SetErr(h, e == cudaErrorMemoryAllocation ? PR_GPU_ENOMEM : PR_GPU_ECUDA, msg);
  h->has_graph = true;
  return EnsureSliceBlocks(h);
}

int pr_gpu_set_edge_weights_device(pr_gpu_t *h, const float *w_dev) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return SetErr(h, PR_GPU_ENOGRAPH, "no graph uploaded");
  if (!h->g.weighted)
    return SetErr(h, PR_GPU_EINVAL, "the uploaded graph has no edge weights");
  if (!w_dev && h->g.m) return SetErr(h, PR_GPU_EINVAL, "w_dev is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  std::string msg;
  cudaError_t e = prgpu::UpdateDeviceWeights(&h->g, w_dev, h->stream, &msg);
  if (e == cudaErrorInvalidValue && msg.rfind("invalid edge weights", 0) == 0)
    return SetErr(h, PR_GPU_EGRAPH, msg);
  if (e != cudaSuccess)
    return SetErr(h, e == cudaErrorMemoryAllocation ? PR_GPU_ENOMEM : PR_GPU_ECUDA,
                  msg.empty() ? std::string(cudaGetErrorString(e)) : msg);
  return PR_GPU_OK;
}

int pr_gpu_run_device(pr_gpu_t *h, int max_iters, double epsilon, float damping, int ncols,
                      const float *teleport_dev, float *scores_out_dev, int32_t *sweeps_out,
                      double *err_trace) {
  int rc = CheckRunArgs(h, max_iters, ncols);
  if (rc) return rc;
  if (!scores_out_dev) return SetErr(h, PR_GPU_EINVAL, "scores_out is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  if (ncols == 1)
    return SolveSingle(h, max_iters, epsilon, damping, teleport_dev, scores_out_dev, sweeps_out,
                       err_trace);
  double ms_sweep = 0, ms_total = 0;
  int64_t launches = 0;
  std::string msg;
  cudaError_t e = prgpu::SolveBatched(h->g, h->bsc, h->stream, max_iters, epsilon, damping,
                                      ncols, teleport_dev, scores_out_dev, sweeps_out, err_trace,
                                      &ms_sweep, &ms_total, &launches, &msg);
  if (e != cudaSuccess)
    return SetErr(h, e == cudaErrorMemoryAllocation ? PR_GPU_ENOMEM : PR_GPU_ECUDA, msg);
  h->last_sweep_ms = ms_sweep;
  h->last_total_ms = ms_total;
  h->last_launches = launches;
  return PR_GPU_OK;
}

int pr_gpu_run(pr_gpu_t *h, int max_iters, double epsilon, float damping, int ncols,
               const float *teleport, float *scores_out, int32_t *sweeps_out,
               double *err_trace) {
  int rc = CheckRunArgs(h, max_iters, ncols);
  if (rc) return rc;
  if (!scores_out) return SetErr(h, PR_GPU_EINVAL, "scores_out is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  const int64_t cells = h->g.n * ncols;
  // outbuf / tele live in the single-column scratch; make room for ncols.
  rc = EnsureScratch(h, h->g.n, ncols, 1, std::max(max_iters, 1));
  if (rc) return rc;
  const float *tele_dev = nullptr;
  if (teleport) {
    rc = CopyToDevice(h, h->sc.tele, teleport, sizeof(float) * cells);
    if (rc) return rc;
    tele_dev = h->sc.tele;
  }
  rc = pr_gpu_run_device(h, max_iters, epsilon, damping, ncols, tele_dev, h->sc.outbuf,
                         sweeps_out, err_trace);
  if (rc) return rc;
  return CopyToHost(h, scores_out, h->sc.outbuf, sizeof(float) * cells);
}


int pr_gpu_adjoint_device(pr_gpu_t *h, int max_iters, double epsilon, float damping,
                          const float *loss_w_dev, const float *scores_dev,
                          float *grad_teleport_dev, float *grad_edge_w_dev, int32_t *sweeps_out) {
  int rc = CheckRunArgs(h, max_iters, 1);
  if (rc) return rc;
  if (!loss_w_dev || !scores_dev) return SetErr(h, PR_GPU_EINVAL, "loss_w / scores is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  rc = SolveAdjoint(h, max_iters, epsilon, damping, loss_w_dev, scores_dev, grad_teleport_dev,
                    grad_edge_w_dev);
  if (rc) return rc;
  if (sweeps_out) *sweeps_out = h->last_adjoint_sweeps;
  return PR_GPU_OK;
}

int pr_gpu_adjoint(pr_gpu_t *h, int max_iters, double epsilon, float damping,
                   const float *loss_w, const float *scores, float *grad_teleport,
                   float *grad_edge_w, int32_t *sweeps_out) {
  int rc = CheckRunArgs(h, max_iters, 1);
  if (rc) return rc;
  if (!loss_w || !scores) return SetErr(h, PR_GPU_EINVAL, "loss_w / scores is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  const int64_t n = h->g.n, m = h->g.m;
  rc = EnsureScratch(h, n, 1, 1, std::max(max_iters, 1));
  if (rc) return rc;
  Scratch &sc = h->sc;
  if (grad_edge_w) PR_CHECK(h, Grow(&sc.edge_buf, &sc.cap_edges, std::max<int64_t>(m, 1)));
  rc = CopyToDevice(h, sc.tele, loss_w, sizeof(float) * n);
  if (!rc) rc = CopyToDevice(h, sc.aux[1], scores, sizeof(float) * n);
  if (rc) return rc;
  rc = pr_gpu_adjoint_device(h, max_iters, epsilon, damping, sc.tele, sc.aux[1],
                             grad_teleport ? sc.outbuf : nullptr,
                             grad_edge_w ? sc.edge_buf : nullptr, sweeps_out);
  if (rc) return rc;
  if (grad_teleport) rc = CopyToHost(h, grad_teleport, sc.outbuf, sizeof(float) * n);
  if (!rc && grad_edge_w) rc = CopyToHost(h, grad_edge_w, sc.edge_buf, sizeof(float) * m);
  return rc;
}

int pr_gpu_verify(pr_gpu_t *h, const float *scores, float damping, double *error_out) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return SetErr(h, PR_GPU_ENOGRAPH, "no graph uploaded");
  if (!scores || !error_out) return SetErr(h, PR_GPU_EINVAL, "scores or error_out is null");
  PR_CHECK(h, cudaSetDevice(h->device));
  const int64_t n = h->g.n;
  int rc = EnsureScratch(h, n, 1, 1, 1);
  if (!rc) rc = CopyToDevice(h, h->sc.tele, scores, sizeof(float) * n);
  if (rc) return rc;
  PR_CHECK(h, prgpu::VerifyResiduals(h->g, h->sc.tele, damping, h->sc.contrib[0], h->sc.outbuf,
                                     h->stream));
  std::unique_ptr<float[]> resid(new (std::nothrow) float[n]);
  if (!resid) return SetErr(h, PR_GPU_ENOMEM, "host buffer for the residuals");
  rc = CopyToHost(h, resid.get(), h->sc.outbuf, sizeof(float) * n);
  if (rc) return rc;
  // the reference's L1 sum: each float residual added in double, in vertex
  // order (src/pr_spmv.cc:88-91)
  double error = 0;
  for (int64_t v = 0; v < n; v++) error += static_cast<double>(resid[v]);
  *error_out = error;
  return PR_GPU_OK;
}

int pr_gpu_set_batch_tile(pr_gpu_t *h, int width) {
  if (!h) return PR_GPU_EINVAL;
  if (width != 0 && width != 8 && width != 16 && width != 32 && width != 64)
    return SetErr(h, PR_GPU_EINVAL, "batch tile width must be 0, 8, 16, 32 or 64");
  h->bsc.tile = width;
  return PR_GPU_OK;
}

int pr_gpu_get_batch_tile(const pr_gpu_t *h, int *width) {
  if (!h || !width) return PR_GPU_EINVAL;
  *width = h->bsc.tile ? h->bsc.tile : h->bsc.tuned_tile;
  return PR_GPU_OK;
}

int pr_gpu_set_batch_schedule(pr_gpu_t *h, int short_len, int l1_kb) {
  if (!h) return PR_GPU_EINVAL;
  bool ok_len = short_len == 0;
  for (int v : prgpu::kShortLens) ok_len = ok_len || v == short_len;
  if (!ok_len) return SetErr(h, PR_GPU_EINVAL, "short_len must be 0, 8, 16, 32, 64 or 128");
  if (l1_kb != 0 && (l1_kb < 16 || l1_kb > 224))
    return SetErr(h, PR_GPU_EINVAL, "l1_kb must be 0 or in [16, 224]");
  h->bsc.sched.short_len = short_len;
  h->bsc.sched.l1_kb = l1_kb;
  return PR_GPU_OK;
}

int pr_gpu_get_batch_schedule(const pr_gpu_t *h, int *width, int *short_len, int *l1_kb) {
  if (!h) return PR_GPU_EINVAL;
  const int w = h->bsc.tile ? h->bsc.tile : h->bsc.tuned_tile;
  if (width) *width = w;
  const prgpu::BatchSchedule r =
      w ? prgpu::ResolveSchedule(h->bsc, w) : prgpu::BatchSchedule();
  if (short_len) *short_len = w ? r.short_len : h->bsc.sched.short_len;
  if (l1_kb) *l1_kb = w ? r.l1_kb : h->bsc.sched.l1_kb;
  return PR_GPU_OK;
}

int pr_gpu_set_sweep_layout(pr_gpu_t *h, int layout, int slice_verts, int bin_words) {
  if (!h) return PR_GPU_EINVAL;
  if (layout < PR_GPU_SWEEP_AUTO || layout > PR_GPU_SWEEP_BLOCKED)
    return SetErr(h, PR_GPU_EINVAL, "sweep layout must be AUTO, GATHER or BLOCKED");
  if (slice_verts != 0 &&
      (slice_verts < 64 || slice_verts > prgpu::kMaxSliceVerts || slice_verts % 64 != 0))
    return SetErr(h, PR_GPU_EINVAL, "slice_verts must be 0 or a multiple of 64 in [64, 56320]");
  if (bin_words != 0 && (bin_words < 1024 || bin_words > prgpu::kMaxBinWords))
    return SetErr(h, PR_GPU_EINVAL, "bin_words must be 0 or in [1024, 28160]");
  PR_CHECK(h, cudaSetDevice(h->device));
  const bool rebuild = slice_verts != h->slice_verts || bin_words != h->bin_words ||
                       (layout != PR_GPU_SWEEP_GATHER && !h->sb.ready);
  h->sweep_layout = layout;
  h->slice_verts = slice_verts;
  h->bin_words = bin_words;
  if (rebuild) {
    PR_CHECK(h, cudaStreamSynchronize(h->stream));
    prgpu::FreeSliceBlocks(&h->sb);
    h->loop_blocked.Reset();
    h->sb_built = false;
  }
  return PR_GPU_OK;
}

int pr_gpu_sweep_layout_info(pr_gpu_t *h, int *blocked, int *slices, int *bins, int64_t *pairs,
                             int64_t *ids, int64_t *bytes, int *last_blocked) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return SetErr(h, PR_GPU_ENOGRAPH, "no graph uploaded");
  PR_CHECK(h, cudaSetDevice(h->device));
  int rc = EnsureSliceBlocks(h);
  if (rc) return rc;
  const bool on = UseBlocked(h);
  if (blocked) *blocked = on ? 1 : 0;
  if (slices) *slices = on ? h->sb.nslices : 0;
  if (bins) *bins = on ? h->sb.nbins : 0;
  if (pairs) *pairs = on ? h->sb.npairs : 0;
  if (ids) *ids = on ? h->sb.elems : 0;
  if (bytes) *bytes = on ? static_cast<int64_t>(h->sb.bytes) : 0;
  if (last_blocked) *last_blocked = h->last_blocked ? 1 : 0;
  return PR_GPU_OK;
}

int pr_gpu_sweep_kernel_times(pr_gpu_t *h, int max_iters, double epsilon, double *ms,
                              int max_kernels, int *nkernels, int32_t *sweeps_out) {
  int rc = CheckRunArgs(h, max_iters, 1);
  if (rc) return rc;
  if (!ms || max_kernels < 3) return SetErr(h, PR_GPU_EINVAL, "ms is null or max_kernels < 3");
  PR_CHECK(h, cudaSetDevice(h->device));
  rc = EnsureScratch(h, h->g.n, 1, 1, std::max(max_iters, 1));
  if (rc) return rc;
  h->time_kernels = true;
  h->kernel_n = 0;
  rc = SolveSingle(h, max_iters, epsilon, 0.85f, nullptr, h->sc.outbuf, sweeps_out, nullptr);
  h->time_kernels = false;
  if (rc) return rc;
  for (int k = 0; k < h->kernel_n; k++) ms[k] = h->kernel_ms[k];
  if (nkernels) *nkernels = h->kernel_n;
  return PR_GPU_OK;
}

int pr_gpu_set_stream(pr_gpu_t *h, void *stream) {
  if (!h) return PR_GPU_EINVAL;
  PR_CHECK(h, cudaSetDevice(h->device));
  PR_CHECK(h, cudaStreamSynchronize(h->stream));
  h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
  return PR_GPU_OK;
}

int pr_gpu_last_timing(const pr_gpu_t *h, double *sweep_ms, double *total_ms,
                       int64_t *kernel_launches) {
  if (!h) return PR_GPU_EINVAL;
  if (sweep_ms) *sweep_ms = h->last_sweep_ms;
  if (total_ms) *total_ms = h->last_total_ms;
  if (kernel_launches) *kernel_launches = h->last_launches;
  return PR_GPU_OK;
}

int pr_gpu_graph_info(const pr_gpu_t *h, int64_t *n, int64_t *m, int64_t *max_degree,
                      int64_t *bin_rows, int nbins) {
  if (!h) return PR_GPU_EINVAL;
  if (!h->has_graph) return PR_GPU_ENOGRAPH;
  if (n) *n = h->g.n;
  if (m) *m = h->g.m;
  if (max_degree) *max_degree = h->g.max_degree;
  if (bin_rows)
    for (int b = 0; b < nbins && b < prgpu::kNumBins; b++)
      bin_rows[b] = h->g.bin_row_start[b + 1] - h->g.bin_row_start[b];
  return PR_GPU_OK;
}

}  // extern "C"
