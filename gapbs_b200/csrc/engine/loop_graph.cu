// loop_graph.cu -- see loop_graph.h.
#include "loop_graph.h"

#include <cstdlib>
#include <cstring>

namespace prgpu {

namespace {

// In plain-launch mode Launch issues max_iters sweep launches (those after
// the loop stopped return at once), each followed by a one-thread kernel
// that advances the sweep index like the decide kernel: it counts every
// sweep that ran, including the one that set `done`, none after it, and
// stops the loop once the sweep index reaches max_iters.  Results and sweep
// counts are identical.
__global__ void loop_advance_kernel(LoopCtl *ctl, int max_iters) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || ctl->halted) return;
  const int loops = ctl->loops + 1;
  ctl->loops = loops;
  if (ctl->done || loops >= max_iters) {
    // the decide kernel's stop rule; later sweep launches see done and return
    ctl->halted = 1;
    ctl->done = 1;
  }
}

__global__ void loop_decide_kernel(LoopCtl *ctl, int max_iters,
                                   cudaGraphConditionalHandle cond) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int loops = ctl->loops + 1;
  ctl->loops = loops;
  const int go = (ctl->done == 0 && loops < max_iters) ? 1 : 0;
  cudaGraphSetConditional(cond, static_cast<unsigned>(go));
}

}  // namespace

// Profilers that replay kernels one by one cannot replay kernel nodes inside
// a graph with conditional nodes.
bool PlainLaunchMode() {
  static const bool plain = [] {
    const char *v = std::getenv("GAPBS_PR_PLAIN_LAUNCH");
    return v && v[0] == '1';
  }();
  return plain;
}

void LoopGraph::Reset() {
  if (exec_) cudaGraphExecDestroy(exec_);
  exec_ = nullptr;
  body_.clear();
  ctl_ = nullptr;
  max_iters_ = 0;
}

cudaError_t LoopGraph::Build(const SweepKernel *ks, int nk, LoopCtl *ctl, int max_iters) {
  Reset();
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle cond;
  // The condition starts at 1 on every launch: the body runs at least once.
  e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNode_t loop_node = nullptr;
  cudaGraphNodeParams cp = {};
  if (e == cudaSuccess) {
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&loop_node, g, nullptr, 0, &cp);
  }
  std::vector<Cached> body;
  if (e == cudaSuccess) {
    cudaGraph_t bg = cp.conditional.phGraph_out[0];
    cudaGraphNode_t prev = nullptr;
    for (int i = 0; i < nk && e == cudaSuccess; i++) {
      Cached c{ks[i].fn, ks[i].grid, ks[i].block, ks[i].smem,
               std::vector<unsigned char>(static_cast<const unsigned char *>(ks[i].args),
                                          static_cast<const unsigned char *>(ks[i].args) +
                                              ks[i].args_size)};
      void *params[] = {c.args.data()};
      cudaKernelNodeParams kp = {};
      kp.func = const_cast<void *>(c.fn);
      kp.gridDim = c.grid;
      kp.blockDim = c.block;
      kp.sharedMemBytes = static_cast<unsigned>(c.smem);
      kp.kernelParams = params;
      cudaGraphNode_t node = nullptr;
      e = cudaGraphAddKernelNode(&node, bg, prev ? &prev : nullptr, prev ? 1 : 0, &kp);
      prev = node;
      body.push_back(std::move(c));
    }
    if (e == cudaSuccess) {
      LoopCtl *c = ctl;
      int mi = max_iters;
      cudaGraphConditionalHandle h = cond;
      void *decide_params[] = {&c, &mi, &h};
      cudaKernelNodeParams dp = {};
      dp.func = reinterpret_cast<void *>(loop_decide_kernel);
      dp.gridDim = dim3(1);
      dp.blockDim = dim3(32);
      dp.kernelParams = decide_params;
      cudaGraphNode_t decide_node = nullptr;
      e = cudaGraphAddKernelNode(&decide_node, bg, prev ? &prev : nullptr, prev ? 1 : 0, &dp);
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec_, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    exec_ = nullptr;
    return e;
  }
  body_ = std::move(body);
  ctl_ = ctl;
  max_iters_ = max_iters;
  return cudaSuccess;
}

bool LoopGraph::Same(const SweepKernel *ks, int nk, LoopCtl *ctl, int max_iters) const {
  if (!exec_ || ctl != ctl_ || max_iters != max_iters_ || static_cast<int>(body_.size()) != nk)
    return false;
  for (int i = 0; i < nk; i++) {
    const Cached &c = body_[i];
    if (c.fn != ks[i].fn || c.grid.x != ks[i].grid.x || c.block.x != ks[i].block.x ||
        c.smem != ks[i].smem || c.args.size() != ks[i].args_size ||
        std::memcmp(c.args.data(), ks[i].args, ks[i].args_size) != 0)
      return false;
  }
  return true;
}

cudaError_t LoopGraph::Launch(const SweepKernel *ks, int nk, LoopCtl *ctl, int max_iters,
                              cudaStream_t s) {
  if (max_iters < 1) return cudaSuccess;
  if (PlainLaunchMode()) {
    std::vector<std::vector<unsigned char>> blobs;
    for (int k = 0; k < nk; k++)
      blobs.emplace_back(static_cast<const unsigned char *>(ks[k].args),
                         static_cast<const unsigned char *>(ks[k].args) + ks[k].args_size);
    for (int i = 0; i < max_iters; i++) {
      for (int k = 0; k < nk; k++) {
        void *params[] = {blobs[k].data()};
        cudaError_t e = cudaLaunchKernel(ks[k].fn, ks[k].grid, ks[k].block, params,
                                         ks[k].smem, s);
        if (e != cudaSuccess) return e;
      }
      loop_advance_kernel<<<1, 32, 0, s>>>(ctl, max_iters);
    }
    return cudaGetLastError();
  }
  if (!Same(ks, nk, ctl, max_iters)) {
    cudaError_t e = Build(ks, nk, ctl, max_iters);
    if (e != cudaSuccess) return e;
  }
  return cudaGraphLaunch(exec_, s);
}

cudaError_t LoopGraph::LaunchTimed(const SweepKernel *ks, int nk, LoopCtl *ctl, int max_iters,
                                   cudaStream_t s, const cudaEvent_t *ev) {
  std::vector<std::vector<unsigned char>> blobs;
  for (int k = 0; k < nk; k++)
    blobs.emplace_back(static_cast<const unsigned char *>(ks[k].args),
                       static_cast<const unsigned char *>(ks[k].args) + ks[k].args_size);
  for (int i = 0; i < max_iters; i++) {
    for (int k = 0; k < nk; k++) {
      cudaError_t e = cudaEventRecord(ev[i * (nk + 1) + k], s);
      if (e != cudaSuccess) return e;
      void *params[] = {blobs[k].data()};
      e = cudaLaunchKernel(ks[k].fn, ks[k].grid, ks[k].block, params, ks[k].smem, s);
      if (e != cudaSuccess) return e;
    }
    cudaError_t e = cudaEventRecord(ev[i * (nk + 1) + nk], s);
    if (e != cudaSuccess) return e;
    loop_advance_kernel<<<1, 32, 0, s>>>(ctl, max_iters);
  }
  return cudaGetLastError();
}

cudaError_t LoopGraph::Launch(const void *fn, dim3 grid, dim3 block, const void *args,
                              size_t args_size, LoopCtl *ctl, int max_iters, cudaStream_t s) {
  SweepKernel k;
  k.fn = fn;
  k.grid = grid;
  k.block = block;
  k.args = args;
  k.args_size = args_size;
  return Launch(&k, 1, ctl, max_iters, s);
}

}  // namespace prgpu
