// batched.h -- batched personalized PageRank (many teleport vectors at once).
#ifndef GAPBS_B200_ENGINE_BATCHED_H_
#define GAPBS_B200_ENGINE_BATCHED_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "internal.h"

namespace prgpu {

// Widest column tile one batched sweep processes (two columns per lane).
constexpr int kMaxTile = 64;

struct BatchCtl {
  LoopCtl loop;               // done flag + sweep index (see loop_graph.h)
  unsigned tick2;             // stage-2 ticket of the grid reduction
  int pad;
  unsigned long long active;  // bit c set while column c of the tile iterates
};

struct BatchScratch {
  float *S = nullptr, *C[2] = {nullptr, nullptr}, *base = nullptr;
  double *part1 = nullptr, *part2 = nullptr, *trace = nullptr;
  unsigned *tick1 = nullptr;
  int32_t *sweeps = nullptr;
  float *seg_partial = nullptr;
  BatchCtl *ctl = nullptr;
  int64_t cap_cells = 0, cap_part = 0, cap_trace = 0, cap_seg = 0;
  int tile = 0;  // column tile width (0 = automatic)
  LoopGraph loop;
};

void FreeBatchScratch(BatchScratch *b);

// Solves ncols personalized PageRank columns (teleport N x ncols, original
// ids, device) into out (N x ncols, original ids, device), in tiles of up
// to kMaxTile columns.  sweeps_out / err_trace are host arrays (nullable)
// laid out as in pr_gpu_run.
cudaError_t SolveBatched(const DeviceGraph &g, BatchScratch &bs, cudaStream_t s,
                         int max_iters, double epsilon, float damping, int ncols,
                         const float *tele_old, float *out_old, int32_t *sweeps_out,
                         double *err_trace, double *ms_sweep, double *ms_total,
                         int64_t *launches, std::string *err);

}  // namespace prgpu

#endif  // GAPBS_B200_ENGINE_BATCHED_H_
