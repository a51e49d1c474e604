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
  fn_ = nullptr;
  args_.clear();
  ctl_ = nullptr;
  max_iters_ = 0;
}

cudaError_t LoopGraph::Build(const void *fn, dim3 grid, dim3 block, const void *args,
                             size_t args_size, LoopCtl *ctl, int max_iters) {
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
  if (e == cudaSuccess) {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    std::vector<unsigned char> arg_copy(static_cast<const unsigned char *>(args),
                                        static_cast<const unsigned char *>(args) + args_size);
    void *sweep_params[] = {arg_copy.data()};
    cudaKernelNodeParams kp = {};
    kp.func = const_cast<void *>(fn);
    kp.gridDim = grid;
    kp.blockDim = block;
    kp.sharedMemBytes = 0;
    kp.kernelParams = sweep_params;
    cudaGraphNode_t sweep_node = nullptr, decide_node = nullptr;
    e = cudaGraphAddKernelNode(&sweep_node, body, nullptr, 0, &kp);
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
      e = cudaGraphAddKernelNode(&decide_node, body, &sweep_node, 1, &dp);
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec_, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    exec_ = nullptr;
    return e;
  }
  fn_ = fn;
  grid_ = grid;
  block_ = block;
  args_.assign(static_cast<const unsigned char *>(args),
               static_cast<const unsigned char *>(args) + args_size);
  ctl_ = ctl;
  max_iters_ = max_iters;
  return cudaSuccess;
}

cudaError_t LoopGraph::Launch(const void *fn, dim3 grid, dim3 block, const void *args,
                              size_t args_size, LoopCtl *ctl, int max_iters, cudaStream_t s) {
  if (max_iters < 1) return cudaSuccess;
  if (PlainLaunchMode()) {
    std::vector<unsigned char> blob(static_cast<const unsigned char *>(args),
                                    static_cast<const unsigned char *>(args) + args_size);
    void *params[] = {blob.data()};
    for (int i = 0; i < max_iters; i++) {
      cudaError_t e = cudaLaunchKernel(fn, grid, block, params, 0, s);
      if (e != cudaSuccess) return e;
      loop_advance_kernel<<<1, 32, 0, s>>>(ctl, max_iters);
    }
    return cudaGetLastError();
  }
  const bool same = exec_ && fn == fn_ && grid.x == grid_.x && block.x == block_.x &&
                    ctl == ctl_ && max_iters == max_iters_ && args_.size() == args_size &&
                    std::memcmp(args_.data(), args, args_size) == 0;
  if (!same) {
    cudaError_t e = Build(fn, grid, block, args, args_size, ctl, max_iters);
    if (e != cudaSuccess) return e;
  }
  return cudaGraphLaunch(exec_, s);
}

}  // namespace prgpu
