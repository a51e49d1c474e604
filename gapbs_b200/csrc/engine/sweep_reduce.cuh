// sweep_reduce.cuh -- the end of every sweep kernel: the L1 change of the
// sweep reduced over the grid in FP64 and the convergence decision.
//
// Deterministic two-stage tree: every block writes its partial, the last
// block of each group of kReduceGroup blocks (per-group ticket) sums that
// group in block order, and the last group (a second ticket) sums the group
// sums, records the sweep's L1 change in trace[it] and sets ctl->loop.done
// when it is below epsilon (src/pr_spmv.cc:55-58).  Tickets never wait: a
// block that is not last simply returns.
#ifndef GAPBS_B200_ENGINE_SWEEP_REDUCE_CUH_
#define GAPBS_B200_ENGINE_SWEEP_REDUCE_CUH_

#include "common.cuh"
#include "internal.h"

namespace prgpu {

struct SweepReduce {
  double *part1;   // per block
  double *part2;   // per group
  unsigned *tick1; // per group
  double *trace;   // per sweep
  SweepCtl *ctl;
  int32_t nblocks;
  double epsilon;
};

// Called by every thread of every block of the sweep, after block_err (valid
// in thread 0) has been formed.
template <int THREADS>
__device__ __forceinline__ void sweep_grid_finish(const SweepReduce &r, int it,
                                                  double block_err, double *sred) {
  __shared__ int s_last;
  const int b = blockIdx.x;
  const int g = b / kReduceGroup;
  const int gsize = min(kReduceGroup, r.nblocks - g * kReduceGroup);
  const int ngroups = (r.nblocks + kReduceGroup - 1) / kReduceGroup;
  if (threadIdx.x == 0) {
    r.part1[b] = block_err;
    __threadfence();
    const unsigned t = atomicAdd(&r.tick1[g], 1u);
    s_last = (t == static_cast<unsigned>(gsize - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v = 0;
  for (int i = threadIdx.x; i < gsize; i += THREADS) v += __ldcg(r.part1 + g * kReduceGroup + i);
  double tot = block_sum_d<THREADS>(v, sred);
  if (threadIdx.x == 0) {
    r.part2[g] = tot;
    r.tick1[g] = 0;
    __threadfence();
    const unsigned t2 = atomicAdd(&r.ctl->tick2, 1u);
    s_last = (t2 == static_cast<unsigned>(ngroups - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  v = 0;
  for (int i = threadIdx.x; i < ngroups; i += THREADS) v += __ldcg(r.part2 + i);
  tot = block_sum_d<THREADS>(v, sred);
  if (threadIdx.x == 0) {
    r.trace[it] = tot;
    r.ctl->sweeps = it + 1;
    r.ctl->tick2 = 0;
    if (tot < r.epsilon) r.ctl->loop.done = 1;
    __threadfence();
  }
}

}  // namespace prgpu

#endif  // GAPBS_B200_ENGINE_SWEEP_REDUCE_CUH_
