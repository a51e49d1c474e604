// batched.h -- batched personalized PageRank (many teleport vectors at once).
#ifndef GAPBS_B200_ENGINE_BATCHED_H_
#define GAPBS_B200_ENGINE_BATCHED_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "internal.h"

namespace prgpu {

// Column tile widths a batched sweep supports (floats per score-block row).
// Widths are padded up to one of these; padding columns never iterate.
constexpr int kMaxTile = 64;
constexpr int kTileWidths[4] = {8, 16, 32, 64};

// Work schedule of a batched sweep (chosen by the autotuner with the tile
// width, or set by the caller): rows with fewer than short_len in-entries go
// one row per lane group of width/4 lanes (the rest one warp per row), and
// the contribs of the highest-degree rows, l1_kb KB per SM, are gathered
// through L1 (all others bypass it).  0 = the default for the width:
// short_len = 1024 / width (two rounds of a warp's gathers), l1_kb = 96.
struct BatchSchedule {
  int short_len = 0;
  int l1_kb = 0;
};
// short_len values a schedule may take: the lengths that start a degree bin.
constexpr int kShortLens[5] = {8, 16, 32, 64, 128};

struct BatchCtl {
  LoopCtl loop;               // done flag + sweep index (see loop_graph.h)
  unsigned tick2;             // stage-2 ticket of the grid reduction
  int compact;                // loop stopped so the survivors can be repacked
  unsigned long long active;  // bit c set while column c of the tile iterates
};

struct BatchScratch {
  // S is an arena of N x 2*kMaxTile floats: every phase of a tile gets its
  // own N x width score block in it (widths at least halve from phase to
  // phase, so they fit), and a column that retires keeps its final scores
  // in the block of the phase it retired in until the tile's one write-back.
  // base alternates between two blocks: a repack copies the surviving
  // columns of one into the other.  The two contrib buffers serve every
  // phase.  base rows are written and read only where tflag[u] is set (the
  // row has a nonzero teleport entry in the tile); elsewhere base is zero by
  // definition.
  float *S = nullptr, *C[2] = {nullptr, nullptr}, *base = nullptr;
  float *base2 = nullptr;
  uint8_t *tflag = nullptr;
  int64_t cap_flag = 0;
  // pinned host mirror of the phase results (ctl, sweeps, trace)
  unsigned char *host = nullptr;
  int64_t cap_host = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double *part1 = nullptr, *part2 = nullptr, *trace = nullptr;
  unsigned *tick1 = nullptr;
  int32_t *sweeps = nullptr;
  float *seg_partial = nullptr;
  BatchCtl *ctl = nullptr;
  int64_t cap_cells = 0, cap_cells2 = 0, cap_part = 0, cap_groups = 0, cap_trace = 0, cap_seg = 0;
  // Column tile width: 0 = chosen by the autotuner (once per uploaded graph
  // and column count), else one of kTileWidths.
  int tile = 0;
  BatchSchedule sched;      // caller's schedule (0 fields: the autotuner's)
  int tuned_tile = 0;       // autotuner's choice for tuned_ncols
  BatchSchedule tuned_sched;
  int tuned_ncols = 0;
  const void *tuned_graph = nullptr;
  LoopGraph loop[4];        // one cached sweep-loop graph per tile width
};

void FreeBatchScratch(BatchScratch *b);

// The schedule a tile of width Bp runs with: the caller's fields where set,
// else the autotuner's (when tuned for this width), else the defaults.
BatchSchedule ResolveSchedule(const BatchScratch &bs, int Bp);

// Solves ncols personalized PageRank columns (teleport N x ncols, original
// ids, device; nullptr = every column uniform 1/N) into out (N x ncols,
// original ids, device), one column tile at a time.  sweeps_out / err_trace
// are host arrays (nullable) laid out as in pr_gpu_run.
cudaError_t SolveBatched(const DeviceGraph &g, BatchScratch &bs, cudaStream_t s,
                         int max_iters, double epsilon, float damping, int ncols,
                         const float *tele_old, float *out_old, int32_t *sweeps_out,
                         double *err_trace, double *ms_sweep, double *ms_total,
                         int64_t *launches, std::string *err);

}  // namespace prgpu

#endif  // GAPBS_B200_ENGINE_BATCHED_H_
