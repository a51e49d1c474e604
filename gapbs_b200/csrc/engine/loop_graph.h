// loop_graph.h -- a solve's sweep loop as one CUDA graph with a device-side
// WHILE condition.
//
// Body = { sweep kernel(s), decide kernel }.  The sweep kernels read the
// sweep index from LoopCtl::loops and the last one records convergence in
// LoopCtl::done; the one-thread decide kernel then increments loops and sets
// the loop condition to (!done && loops < max_iters).  The loop therefore ends after at most
// max_iters bodies whatever the sweep kernel computes, and no launch is spent
// after convergence.
#ifndef GAPBS_B200_ENGINE_LOOP_GRAPH_H_
#define GAPBS_B200_ENGINE_LOOP_GRAPH_H_

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace prgpu {

// Shared prefix of every solve's device control block.
struct LoopCtl {
  int done;    // set by the sweep kernel when the solve converged
  int loops;   // sweeps issued so far; owned by the decide kernel
  int halted;  // plain-launch mode: the sweep that set `done` has been counted
};

// GAPBS_PR_PLAIN_LAUNCH=1: device-driven loops are issued as ordinary
// launches instead (for profilers that cannot replay kernel nodes inside
// graphs with conditional nodes); results are identical.
bool PlainLaunchMode();

// One kernel of a sweep body: fn<<<grid, block, smem>>>(args), where args
// points to the kernel's single by-value parameter of args_size bytes.
struct SweepKernel {
  const void *fn = nullptr;
  dim3 grid, block;
  size_t smem = 0;
  const void *args = nullptr;
  size_t args_size = 0;
};

class LoopGraph {
 public:
  LoopGraph() = default;
  LoopGraph(const LoopGraph &) = delete;
  LoopGraph &operator=(const LoopGraph &) = delete;
  ~LoopGraph() { Reset(); }

  // Launches up to max_iters (>= 1) sweeps of `fn<<<grid, block>>>(args)` on
  // stream s.  The instantiated graph is cached and reused while the kernel,
  // launch shape, argument bytes, control block and max_iters are unchanged.
  cudaError_t Launch(const void *fn, dim3 grid, dim3 block, const void *args,
                     size_t args_size, LoopCtl *ctl, int max_iters, cudaStream_t s);
  // The same for a body of several kernels run in order (then the decide
  // kernel); the sweep index they read is the same within one body.
  cudaError_t Launch(const SweepKernel *ks, int nk, LoopCtl *ctl, int max_iters,
                     cudaStream_t s);
  void Reset();
  // Measurement: the same sweeps as Launch(ks, nk, ...) issued as ordinary
  // launches, with ev[i (nk + 1) + k] recorded before kernel k of sweep i
  // and ev[i (nk + 1) + nk] after its last kernel (max_iters (nk + 1)
  // events).  Sweeps after the loop stopped return at once.
  static cudaError_t LaunchTimed(const SweepKernel *ks, int nk, LoopCtl *ctl, int max_iters,
                                 cudaStream_t s, const cudaEvent_t *ev);

 private:
  cudaError_t Build(const SweepKernel *ks, int nk, LoopCtl *ctl, int max_iters);
  bool Same(const SweepKernel *ks, int nk, LoopCtl *ctl, int max_iters) const;

  struct Cached {
    const void *fn;
    dim3 grid, block;
    size_t smem;
    std::vector<unsigned char> args;
  };
  cudaGraphExec_t exec_ = nullptr;
  std::vector<Cached> body_;
  LoopCtl *ctl_ = nullptr;
  int max_iters_ = 0;
};

}  // namespace prgpu

#endif  // GAPBS_B200_ENGINE_LOOP_GRAPH_H_
