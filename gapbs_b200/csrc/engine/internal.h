// internal.h -- device data layout and launch plumbing shared by the engine's
// translation units.  Not part of the public ABI (include/pr_gpu.h is).
//
// Device mirror of a graph (all arrays in HBM, built once per upload):
//   Vertices are renumbered by descending in-degree (ties by original id):
//   perm[new] = old, inv[old] = new.  Row u of the renumbered in-CSR holds
//   the in-neighbours of perm[u], translated to new ids, in their original
//   order.  Rows of equal length class are therefore contiguous, which makes
//   every vertex bin a plain row range, and the most-gathered contrib entries
//   (the hubs) a dense prefix of the contrib array that stays in L2.
#ifndef GAPBS_B200_ENGINE_INTERNAL_H_
#define GAPBS_B200_ENGINE_INTERNAL_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "loop_graph.h"

namespace prgpu {

// Vertex bins, in row order (rows sorted by descending length):
//   0 HUB   rows of >= hub_min entries, split into segments of kSegEntries;
//           one block per segment, the last segment's block finishes the row
//   1..6    G = 32, 16, 8, 4, 2, 1 lanes per row (one row per lane group)
//   7 ZERO  rows without in-neighbours
constexpr int kNumBins = 8;
constexpr int kBinHub = 0;
constexpr int kBinZero = 7;
constexpr int kSweepThreads = 256;
constexpr int kSegEntries = 8192;
constexpr int kZeroRowsPerThread = 4;
// Lane-group size of bins 1..6.
constexpr int kBinGroup[kNumBins] = {kSweepThreads, 32, 16, 8, 4, 2, 1, 1};
// Grid reduction: stage-1 groups of this many blocks.
constexpr int kReduceGroup = 512;

// Default minimum row length of each bin (bin b takes rows with
// length >= min_len[b] not taken by an earlier bin).
struct BinConfig {
  int min_len[kNumBins] = {4096, 128, 64, 32, 16, 8, 1, 0};
};

struct DeviceGraph {
  int64_t n = 0, m = 0;
  bool directed = false;
  bool weighted = false;
  int64_t max_degree = 0;
  // renumbered in-CSR
  int32_t *rowoff = nullptr;   // n+1
  int32_t *col = nullptr;      // m rounded up to a multiple of 4
  float *win = nullptr;        // weighted: w(v->u) aligned with col
  int32_t *win_pos = nullptr;  // weighted: where each win entry's weight sits in
                               // the caller's out-CSR (for weight updates)
  // out-direction data in new ids
  int32_t *odeg = nullptr;     // directed: out-degree per new id
  float *rsum = nullptr;       // weighted: S_v = sum of out-weights per new id
  int32_t *orowoff = nullptr;  // directed: renumbered out-CSR (adjoint)
  int32_t *ocol = nullptr;
  float *wout = nullptr;       // weighted: w(v->u) aligned with the out rows
  int32_t *orig_out_off = nullptr;  // the caller's out-offsets (original ids):
                                    // entry j of renumbered out-row v sits at
                                    // orig_out_off[perm[v]] + j in the caller's CSR
  int32_t *perm = nullptr;     // new -> old
  int32_t *inv = nullptr;      // old -> new
  // bins
  BinConfig bins;
  int64_t bin_row_start[kNumBins + 1] = {};
  int64_t num_hub_rows = 0;
  int64_t num_segments = 0;
  int32_t *seg_row = nullptr;     // segment -> hub row
  int32_t *seg_first = nullptr;   // hub row -> first segment (num_hub_rows+1)
  unsigned *hub_ticket = nullptr; // per hub row
  float *seg_partial = nullptr;   // per segment
};

// Per-solve convergence control, in device memory.
struct SweepCtl {
  LoopCtl loop;     // done flag + sweep index (see loop_graph.h)
  int sweeps;       // sweeps completed
  unsigned tick2;   // stage-2 ticket of the grid reduction
  int unit_next[2]; // slice-blocked sweeps: phase-1 units taken (flat, other)
};

struct Scratch {
  float *score = nullptr;      // n x ncols (new ids)
  float *contrib[2] = {nullptr, nullptr};
  float *base = nullptr;       // per-vertex (1-d) t (PPR), new ids
  float *outbuf = nullptr;     // n x ncols scores in original ids
  float *tele = nullptr;       // teleport staging (original ids)
  float *aux[2] = {nullptr, nullptr};  // adjoint: forward scores (new ids), staging
  float *edge_buf = nullptr;   // adjoint: m edge gradients (device staging)
  double *norm = nullptr;      // adjoint: ||w||_1
  int64_t cap_edges = 0;
  double *part1 = nullptr;     // per block
  double *part2 = nullptr;     // per stage-1 group
  unsigned *tick1 = nullptr;   // per stage-1 group
  double *trace = nullptr;     // max_iters
  SweepCtl *ctl = nullptr;
  int64_t cap_n = 0, cap_blocks = 0, cap_iters = 0, cap_cols = 0;
};

// What one pull sweep computes per row u (sum = gathered neighbour values):
//   kKindPlain    new = base + d * sum, base a scalar (the reference's PR)
//   kKindPPR      new = base[u] + d * sum          (personalized PR)
//   kKindAdjoint  new = base[u] + d * sum / S_u, and the gathered value of u
//                 is new itself (adjoint iteration over out-rows)
constexpr int kKindPlain = 0;
constexpr int kKindPPR = 1;
constexpr int kKindAdjoint = 2;

// Kernel-side view of one plain / single-column sweep.
struct PullArgs {
  int32_t n;
  int32_t kind;
  const int32_t *__restrict__ rowoff;
  const int32_t *__restrict__ col;
  const float *__restrict__ win;
  const int32_t *__restrict__ odeg;
  const float *__restrict__ rsum;
  const float *__restrict__ base_vec;  // nullptr => base_scalar
  float base_scalar;
  float damping;
  float *score;
  // contrib ping-pong: sweep k gathers c[k & 1] and writes c[(k + 1) & 1]
  float *c0;
  float *c1;
  // hub segments (block-cooperative) and warp tasks of bins 1..7
  int32_t nseg;
  int32_t task_start[kNumBins + 1];  // first task of bin b; [kNumBins] = total
  int32_t bin_row[kNumBins + 1];     // first row of bin b; [kNumBins] = n
  const int32_t *__restrict__ seg_row;
  const int32_t *__restrict__ seg_first;
  unsigned *hub_ticket;
  float *seg_partial;
  // grid reduction
  double *part1;
  double *part2;
  unsigned *tick1;
  double *trace;
  SweepCtl *ctl;
  int32_t nblocks;
  // Vertices [0, l1_rows) -- the highest-degree ones after renumbering -- are
  // gathered through L1; the rest bypass L1 so they cannot evict them.
  int32_t l1_rows;
  // From this sweep on, rows without in-neighbours are final and skipped.
  int32_t zero_final_sweep;
  double epsilon;
};

// L1 budget per SM for hub contribs of a single-column sweep.
constexpr int kL1HubBytes = 128 * 1024;

// Launchers (kernels.cu / prep.cu).
cudaError_t BuildDeviceGraph(DeviceGraph *g, int64_t n, int64_t m,
                             const int32_t *d_out_off, const int32_t *d_out_nbr,
                             const int32_t *d_in_off, const int32_t *d_in_nbr,
                             const float *d_ew, bool directed,
                             cudaStream_t s, std::string *err);
void FreeDeviceGraph(DeviceGraph *g);
// New edge weights for a weighted graph already on the device: d_w holds one
// weight per entry of the caller's out-CSR (as uploaded).  Checked first
// (finite and positive, else cudaErrorInvalidValue and the old weights stay),
// then rsum, win and wout are rebuilt on the device.
cudaError_t UpdateDeviceWeights(DeviceGraph *g, const float *d_w, cudaStream_t s,
                                std::string *err);

// The reference's PRVerifier residuals (verify.cu): score_orig holds n
// scores in original ids; contrib (n floats, scratch) receives score /
// out_degree in new ids and resid_orig[v] = |base + d * incoming[v] -
// score[v]| in original ids, incoming summed in row order.  Edge weights are
// not used.
cudaError_t VerifyResiduals(const DeviceGraph &g, const float *score_orig, float damping,
                            float *contrib, float *resid_orig, cudaStream_t s);

// The reference's -g / -u graph built on the device (generate.cu): CSR of
// the symmetrised, squished graph in original ids, int32 offsets (n+1) and
// neighbours (m), owned by the caller.  perm_host: the R-MAT relabelling.
cudaError_t GenerateGraph(bool uniform, int scale, int degree, const int32_t *perm_host,
                          cudaStream_t s, int64_t *n_out, int64_t *m_out, int32_t **off_out,
                          int32_t **nbr_out, std::string *err);
void WidenOffsets(int64_t n1, const int32_t *off32, int64_t *off64, cudaStream_t s);

// Connected components of the uploaded graph (cc.cu): out_old[v] = the
// smallest original vertex id of v's component (device buffer, n entries).
struct CcScratch {
  int *comp = nullptr, *root_min = nullptr, *err = nullptr;
  int64_t cap = 0;
};
void FreeCcScratch(CcScratch *c);

// Breadth-first search (bfs.cu).  Work arrays kept between calls.
struct BfsScratch {
  int32_t *parent = nullptr, *queue[2] = {nullptr, nullptr};
  unsigned *bm[2] = {nullptr, nullptr};
  int64_t *deg = nullptr, *eoff = nullptr, *sums = nullptr;
  void *ctl = nullptr;  // the search's control block (bfs.cu)
  int64_t cap_n = 0;
  // the search loop graph and the launch plan it was captured with
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap_stream = nullptr;
  std::vector<unsigned char> plan;
};
struct BfsStep {
  const char *kind;  // "i", "td", "e", "bu", "c" as the reference logs them
  int64_t count;     // frontier size after td, awake count after bu, else -1
  double seconds;
};
void FreeBfsScratch(BfsScratch *b);
// parent_old[v] (device, n entries, original ids): v's BFS parent from
// source_old, the source itself for the source, -1 when unreached.  steps
// (nullable): the first steps with device-measured durations; *nsteps
// (nullable): the number of steps, init included.
cudaError_t BreadthFirstSearch(const DeviceGraph &g, BfsScratch &b, cudaStream_t s,
                               int source_old, int alpha, int beta, int32_t *parent_old,
                               std::vector<BfsStep> *steps, int64_t *nsteps, std::string *err);
cudaError_t ConnectedComponents(const DeviceGraph &g, CcScratch &cs, cudaStream_t s,
                                int32_t *out_old, std::string *err);
// int64 CSR offsets -> int32, setting *bad for values outside [0, 2^31).
void NarrowOffsets(int64_t count, const int64_t *wide, int32_t *narrow, int *bad, cudaStream_t s);

// Warp tasks per bin (fills task_start, returns the total) and the
// persistent grid size of a sweep kernel (SMs x resident blocks per SM).
int PullTasks(const DeviceGraph &g, int32_t task_start[kNumBins + 1]);
int PullGrid(const void *kernel);

cudaError_t LaunchPullInit(const DeviceGraph &g, Scratch &sc, const float *tele_new,
                           float init_scalar, float damping, cudaStream_t s);
// Kernel to run for one sweep of `a` (a function pointer for LoopGraph).
const void *PullSweepKernel(const PullArgs &a);
// Warp-per-row sweep over an arbitrary (unsorted) CSR given in a.rowoff /
// a.col, a.nblocks blocks, grid-stride; used for adjoint sweeps over the
// out-rows of directed graphs.
const void *PullGenericKernel(const PullArgs &a);
// Per-edge weight gradient and teleport gradient of the adjoint (pull.cu).
cudaError_t LaunchAdjointGrads(const DeviceGraph &g, const int32_t *orow, const int32_t *ocol,
                               const float *wout, const float *lam_new, const float *s_new,
                               float damping, float *grad_ew, float *grad_t_old,
                               cudaStream_t s);
cudaError_t LaunchL1Norm(const float *x, int64_t n, double *out, cudaStream_t s);
cudaError_t LaunchGatherOut(const DeviceGraph &g, const float *src_new, float *dst_old,
                            int ncols, cudaStream_t s);
cudaError_t LaunchScatterIn(const DeviceGraph &g, const float *src_old, float *dst_new,
                            int ncols, cudaStream_t s);
cudaError_t LaunchResetCtl(Scratch &sc, int nblocks, int iters, cudaStream_t s);

}  // namespace prgpu

#endif  // GAPBS_B200_ENGINE_INTERNAL_H_
