/*
 * pr_gpu.h -- C ABI of the B200 PageRank engine (libgapbs_pr.so, sm_100a).
 *
 * This is the drop-in boundary for the GAP Benchmark Suite's pull-direction
 * Jacobi PageRank.  A reference-side caller replaces the body of
 *
 *   pvector<ScoreT> PageRankPull(const Graph &g, int max_iters,
 *                                double epsilon, bool logging_enabled)
 *                                              (src/pr_spmv.cc:35-61)
 *
 * with pr_gpu_upload (once per graph) + pr_gpu_run, and gets the same float
 * scores (within FP32 summation-order tolerance), the same sweep count and
 * the same per-sweep L1 error trace (src/pr_spmv.cc:55-58).
 *
 * Conventions
 *   - Every int function returns PR_GPU_OK (0) or a negative PR_GPU_E* code;
 *     pr_gpu_last_error(h) describes the last failure on that handle.  No
 *     C++ exception crosses this boundary.
 *   - All pointers are plain host pointers unless the function name ends in
 *     _device, in which case they are device pointers on the handle's GPU.
 *   - Graph ids are int32 (NodeID, src/benchmark.h:31); offsets are int32, so
 *     an uploaded graph holds at most 2^31-1 CSR entries per direction.
 *   - Score blocks with ncols columns are vertex-major: element (v, c) lives
 *     at [v * ncols + c] (an N x ncols row-major block).
 *   - One handle is used by one host thread at a time.  It owns every device
 *     allocation; callers own every host buffer they pass.
 */
#ifndef GAPBS_PR_GPU_H_
#define GAPBS_PR_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PR_GPU_OK 0
#define PR_GPU_EINVAL (-1)    /* bad argument */
#define PR_GPU_ECUDA (-2)     /* CUDA runtime error */
#define PR_GPU_ENOMEM (-3)    /* device or pinned allocation failed */
#define PR_GPU_ENOGRAPH (-4)  /* no graph uploaded on this handle */
#define PR_GPU_EGRAPH (-5)    /* CSR failed validation (offsets / ids) */
#define PR_GPU_ERANGE (-6)    /* graph exceeds int32 offsets */

typedef struct pr_gpu pr_gpu_t;

/* Creates a handle bound to CUDA device `device` with its own stream.  The
 * handle owns the device mirror of one CSRGraph (src/graph.h:98-273, which
 * the reference keeps in host memory only) and every device allocation. */
int pr_gpu_create(pr_gpu_t **h, int device);

/* Uploads a CSR graph and builds the device mirror (degree-ordered rows and
 * the vertex bins the sweep uses).  Replaces the CSRGraph the reference's
 * PageRankPull reads through out_degree / in_neigh (src/graph.h:205-221).
 *
 *   n                 number of vertices
 *   m                 entries per direction (num_edges_directed)
 *   out_off/out_nbr   out-CSR (n+1 offsets, m neighbour ids)
 *   in_off/in_nbr     in-CSR; NULL (or equal to out_*) for an undirected
 *                     graph, whose single CSR serves both directions
 *                     (src/graph.h:138-143)
 *   edge_w            optional FP32 weight per out-CSR entry (weight of v->u
 *                     at v's out-list position); NULL means unit weights.
 *                     Transition probabilities are w(v->u) / sum_u' w(v->u').
 *
 * The CSR is validated on the device (monotone offsets starting at 0 and
 * ending at m, every id in [0, n)); failures return PR_GPU_EGRAPH.  A new
 * upload replaces the previous graph. */
int pr_gpu_upload(pr_gpu_t *h, int64_t n, int64_t m,
                  const int32_t *out_off, const int32_t *out_nbr,
                  const int32_t *in_off, const int32_t *in_nbr,
                  const float *edge_w);

/* New edge weights for the weighted graph on the device, from DEVICE memory
 * on the handle's device: w_dev holds one FP32 weight per entry of the
 * out-CSR as it was uploaded (the edge_w layout of pr_gpu_upload).  The
 * weights are checked on the device first (finite and positive, else
 * PR_GPU_EGRAPH and the previous weights stay); then the per-vertex weight
 * sums and the engine's two weight arrays are rebuilt by device gathers, in
 * the handle's stream.  No host copy, no re-upload, no renumbering: a
 * caller whose weights change every step (a training loop) pays three
 * device kernels.  A graph uploaded without weights returns PR_GPU_EINVAL.
 * No counterpart in the reference (its graphs are fixed). */
int pr_gpu_set_edge_weights_device(pr_gpu_t *h, const float *w_dev);

/* Uploads a serialized graph file (.sg, the layout of src/writer.h:39-69 that
 * the reference's reader loads in src/reader.h:254-307) straight from the
 * file to the device: the file is read in chunks into pinned buffers and
 * copied by DMA while the next chunk is read; int64 offsets are narrowed to
 * int32 on the device.  No host copy of the CSR is built.  Same validation
 * and result as pr_gpu_upload of the same graph; a truncated or corrupt file
 * returns PR_GPU_EGRAPH. */
int pr_gpu_upload_sg(pr_gpu_t *h, const char *path);

/* Builds the reference's synthetic graph on the device and uploads it as
 * pr_gpu_upload would: pr_spmv -g scale -k degree (R-MAT, quadrant
 * probabilities 0.57/0.19/0.19) or, with uniform != 0, -u scale -k degree;
 * 2^scale * degree edges from the reference's per-block mt19937 streams
 * (src/generator.h:105-155), symmetrised and squished as its builder does
 * (src/builder.h:141-170,300-323).  The CSR is identical to the reference's.
 * R-MAT ids are relabelled through the reference's seeded permutation, which
 * the caller computes on the host (gapbs_rmat_permutation in gapbs_graph.h,
 * 2^scale entries); uniform graphs pass NULL.  Replaces the Generator /
 * BuilderBase::MakeGraph path of src/builder.h:343-364 for -g / -u.
 *   n_out  vertices (largest id + 1)    m_out  CSR entries (both directions)
 * The original-id CSR stays on the device until pr_gpu_download_csr, the
 * next upload or generate, or pr_gpu_destroy. */
int pr_gpu_generate(pr_gpu_t *h, int uniform, int scale, int degree,
                    const int32_t *perm, int64_t *n_out, int64_t *m_out);

/* Copies the CSR of the last pr_gpu_generate to host buffers (n_out + 1
 * offsets, m_out neighbours), then frees the device copy: the host CSR the
 * reference's BuilderBase::MakeGraph returns (src/builder.h:343-364), for
 * host code such as PRVerifier. */
int pr_gpu_download_csr(pr_gpu_t *h, int64_t *out_off, int32_t *out_nbr);

/* One step of a breadth-first search as the reference logs it with -l
 * (src/bfs.cc:118-160): kind "i" (init), "td" (top-down; count = next
 * frontier size), "e" (queue to bitmap), "bu" (bottom-up; count = vertices
 * found), "c" (bitmap to queue); count -1 where the reference prints none.
 * seconds: the step's duration measured on the device (the steps run as
 * one CUDA graph, so no host clock sees them one by one). */
typedef struct pr_gpu_bfs_step {
  char kind[4];
  int64_t count;
  double seconds;
} pr_gpu_bfs_step_t;

/* Direction-optimizing breadth-first search from `source` (original id) over
 * the uploaded graph, the reference's DOBFS (src/bfs.cc:38-174: the same
 * top-down / bottom-up steps and switching rule, alpha 15, beta 18).
 * parent_out[v] (n entries, original ids) = v's parent in a BFS tree, the
 * source for the source, -1 when unreachable; depths along the tree are BFS
 * depths, so the reference's BFSVerifier (src/bfs.cc:201-245) accepts
 * it.  Which of several same-depth candidates becomes a parent is a race,
 * as in the reference.  steps (nullable): the first max_steps steps;
 * *nsteps: their total.  Host buffer / device buffer forms. */
int pr_gpu_bfs(pr_gpu_t *h, int64_t source, int32_t *parent_out,
               pr_gpu_bfs_step_t *steps, int max_steps, int *nsteps);
int pr_gpu_bfs_device(pr_gpu_t *h, int64_t source, int32_t *parent_out_dev,
                      pr_gpu_bfs_step_t *steps, int max_steps, int *nsteps);

/* Connected components of the uploaded graph, the reference's Afforest
 * (src/cc.cc:40-150: two neighbour-sampling rounds, the largest
 * intermediate component skipped in the final link phase, a directed graph
 * linked through its in-neighbours too).  comp_out[v] (n entries, original
 * ids) = the smallest vertex id of v's component, which is the label the
 * reference's Link/Compress produce.  Host buffer / device buffer forms. */
int pr_gpu_connected_components(pr_gpu_t *h, int32_t *comp_out);
int pr_gpu_connected_components_device(pr_gpu_t *h, int32_t *comp_out_dev);

/* Runs Jacobi PageRank sweeps until the L1 change of a sweep is < epsilon or
 * max_iters sweeps have run (src/pr_spmv.cc:41-58).
 *
 *   ncols == 1, teleport == NULL : the reference's PageRankPull exactly
 *       (init 1/N, base (1-d)/N in float, contrib = score / out_degree).
 *   teleport != NULL : personalized PageRank, s = (1-d) t + d P^T s started
 *       from s_0 = t, one column per teleport vector (n x ncols block);
 *       columns retire independently when their own L1 change < epsilon.
 *   scores_out   n x ncols floats (caller-owned host buffer)
 *   sweeps_out   ncols ints: sweeps executed per column (nullable)
 *   err_trace    max_iters x ncols doubles, [iter * ncols + c], the FP64 L1
 *                change of each sweep; 0 after a column retired (nullable)
 * damping is the reference's kDamp (0.85f, src/pr_spmv.cc:33). */
int pr_gpu_run(pr_gpu_t *h, int max_iters, double epsilon, float damping,
               int ncols, const float *teleport, float *scores_out,
               int32_t *sweeps_out, double *err_trace);

/* Same as pr_gpu_run (PageRankPull, src/pr_spmv.cc:35-61) with teleport /
 * scores_out as DEVICE pointers on the handle's GPU (no host copies; the
 * call still returns after the solve). */
int pr_gpu_run_device(pr_gpu_t *h, int max_iters, double epsilon,
                      float damping, int ncols, const float *teleport_dev,
                      float *scores_out_dev, int32_t *sweeps_out,
                      double *err_trace);

/* Reverse-mode derivative of L = sum_v loss_w[v] * s[v] at the fixed point
 * s of the last single-column pr_gpu_run (scores passed back in `scores`).
 * Solves lambda = w + d P lambda (a gather over OUT-neighbours) until its L1
 * change < epsilon * ||w||_1 or max_iters sweeps, then
 *   grad_teleport[u]  = (1-d) lambda[u]
 *   grad_edge_w[e]    = d s[v] / S_v (lambda[u] - (P lambda)[v]),  e = (v->u)
 * with grad_edge_w aligned with the uploaded out-CSR (nullable).
 * The reference has no adjoint; this is the engine's own extension.
 * Host-pointer form. */
int pr_gpu_adjoint(pr_gpu_t *h, int max_iters, double epsilon, float damping,
                   const float *loss_w, const float *scores,
                   float *grad_teleport, float *grad_edge_w,
                   int32_t *sweeps_out);

/* Device-pointer form of pr_gpu_adjoint (no counterpart in the reference). */
int pr_gpu_adjoint_device(pr_gpu_t *h, int max_iters, double epsilon,
                          float damping, const float *loss_w_dev,
                          const float *scores_dev, float *grad_teleport_dev,
                          float *grad_edge_w_dev, int32_t *sweeps_out);

/* The reference's PRVerifier (src/pr_spmv.cc:78-94) on the device: one
 * push-direction sweep from `scores` (n floats in original ids, host buffer),
 *   error = sum_n |base + d * incoming[n] - scores[n]|,
 *   incoming[n] = sum over in-neighbours u of scores[u] / out_degree(u),
 * base = (1 - d) / N, every per-vertex operation in float as the reference
 * computes it and the sum over vertices in double in vertex order.  When each
 * row of the uploaded in-CSR lists its sources in ascending order (the
 * reference's builder sorts and deduplicates every row), incoming[n] is added
 * in the reference's push order and *error_out equals the reference's error
 * bit for bit; other row orders change only its rounding.  Edge weights, if
 * uploaded, are not used: this is the unweighted check.  The caller compares
 * *error_out with its tolerance (the reference passes when error < target).
 * damping is the reference's kDamp (0.85f). */
int pr_gpu_verify(pr_gpu_t *h, const float *scores, float damping, double *error_out);

/* Engine controls below have no counterpart in the reference.
 *
 * Column tile width of batched (ncols > 1) solves: 8, 16, 32 or 64 score
 * columns per block row, or 0 (the default) to let the engine's autotuner
 * time each width on the first batched solve of a graph and column count
 * and keep the fastest.  pr_gpu_get_batch_tile reports the width in use
 * (0 before any batched solve under the autotuner). */
int pr_gpu_set_batch_tile(pr_gpu_t *h, int width);
int pr_gpu_get_batch_tile(const pr_gpu_t *h, int *width);

/* Work schedule of batched solves, chosen by the same autotuner after the
 * width (at the chosen width it times half and twice the default short-row
 * length, then L1 budgets of 64 and 160 KB, keeping what is faster):
 *   short_len  rows with fewer in-entries go one row per group of width/4
 *              lanes, longer ones one warp per row: 8, 16, 32, 64 or 128
 *              (default 1024 / width);
 *   l1_kb      KB per SM of the highest-degree rows' contribs gathered
 *              through L1, the rest bypassing it: 16..224 (default 96).
 * 0 leaves a field to the autotuner.  pr_gpu_get_batch_schedule reports
 * the schedule the current width runs with (the tuned one after the first
 * batched solve). */
int pr_gpu_set_batch_schedule(pr_gpu_t *h, int short_len, int l1_kb);
int pr_gpu_get_batch_schedule(const pr_gpu_t *h, int *width, int *short_len, int *l1_kb);

/* Sweep layout of single-column solves (plain and personalized PageRank) on
 * unweighted graphs:
 *   PR_GPU_SWEEP_AUTO     slice-blocked when the graph has at least 48 Mi
 *                         (48 x 2^20) edges (below that the gather sweep's
 *                         contribs stay in the caches), fits that layout's
 *                         limits, the device has room for it and its
 *                         in-edges form at most M/2 (row, slice) pairs
 *                         (skewed graphs such as Kronecker ones; on uniform
 *                         random graphs nearly every edge is a pair of its
 *                         own and gather is faster), else gather
 *   PR_GPU_SWEEP_GATHER   one sweep kernel that gathers contrib[v] for every
 *                         in-edge (no extra device memory)
 *   PR_GPU_SWEEP_BLOCKED  slice-blocked; a run on a graph it does not fit
 *                         returns PR_GPU_EINVAL
 * The slice-blocked sweep is three kernels per sweep: per slice of
 * slice_verts consecutive source vertices (held in shared memory) a partial
 * sum for every destination row the slice reaches (one launch for the
 * (row, slice) pairs of 1, 2, 4 or 8 edges, one for the others), then per
 * bin of rows (bin_words shared-memory words of partials and row sums) the
 * row update.  It holds about 2.6 bytes per edge and 14 bytes per (row,
 * slice) pair of extra device memory, built from the device CSR at upload.
 * slice_verts (multiple of 64, 64..56320) and bin_words (1024..28160): 0
 * keeps the defaults (49152; 6144, or 12288 on graphs whose pairs and rows
 * fill at least 64 such bins per SM).  Changing them rebuilds the layout at the next
 * run.  Weighted graphs, the adjoint and batched solves use gather sweeps.
 * No counterpart in the reference. */
#define PR_GPU_SWEEP_AUTO 0
#define PR_GPU_SWEEP_GATHER 1
#define PR_GPU_SWEEP_BLOCKED 2
int pr_gpu_set_sweep_layout(pr_gpu_t *h, int layout, int slice_verts, int bin_words);

/* The layout of the uploaded graph: *blocked = 1 when single-column solves
 * use the slice-blocked sweep; its slice count, bin count, (row, slice)
 * pairs, stored source ids (the edges plus padding) and device bytes (all
 * nullable; 0 when not built).  *last_blocked: whether the last
 * single-column run used it. */
int pr_gpu_sweep_layout_info(pr_gpu_t *h, int *blocked, int *slices, int *bins,
                             int64_t *pairs, int64_t *ids, int64_t *bytes,
                             int *last_blocked);

/* Measurement aid: runs one plain PageRank solve of the uploaded graph
 * (uniform teleport, damping 0.85; scores left in an internal buffer) with
 * every sweep kernel launched on its own between CUDA events on the
 * handle's stream, and writes the average device time per sweep of each
 * kernel of the sweep body, in launch order, to ms[0 .. *nkernels):
 * slice-blocked: flat-pair partials, other partials, row update; gather:
 * the sweep kernel.  max_kernels: room in ms (at least 3).  *sweeps_out:
 * the sweeps the solve ran.  The timings include no loop or launch
 * overhead of the regular CUDA-graph loop.  No counterpart in the
 * reference. */
int pr_gpu_sweep_kernel_times(pr_gpu_t *h, int max_iters, double epsilon, double *ms,
                              int max_kernels, int *nkernels, int32_t *sweeps_out);

/* Makes the handle issue its work on `stream` (a cudaStream_t of the
 * handle's device, e.g. the caller's framework stream) instead of its own;
 * NULL restores the handle's own stream.  The handle does not take
 * ownership.  Calls still synchronize that stream before returning. */
int pr_gpu_set_stream(pr_gpu_t *h, void *stream);

/* Device time (CUDA events on the handle's stream) of the sweep kernels of
 * the last run and the number of engine kernel launches it made. */
int pr_gpu_last_timing(const pr_gpu_t *h, double *sweep_ms, double *total_ms,
                       int64_t *kernel_launches);

/* Graph facts after upload: vertices and entries (CSRGraph::num_nodes,
 * num_edges_directed, src/graph.h:193-203), rows per vertex bin (nbins
 * entries, bin order as documented in the engine), max in-degree. */
int pr_gpu_graph_info(const pr_gpu_t *h, int64_t *n, int64_t *m,
                      int64_t *max_degree, int64_t *bin_rows, int nbins);

/* Diagnostic: the random-gather ceiling of this GPU.  Times independent
 * 4-byte loads at hashed addresses inside a device array of array_bytes
 * (rounded down to a power of two; far larger than L1), and returns the loads
 * completed per second.  A pull sweep issues one such load per edge, so with
 * an array that fits in L2 this is the rate that bounds the sweep kernels
 * when their gathers miss L1 (each costs a 32-byte sector request between
 * the SM and L2).  Allocates and frees its own buffers.  No counterpart in
 * the reference. */
int pr_gpu_measure_gather_rate(int device, int64_t array_bytes, double *gathers_per_s);

/* The same for whole rows: gathers random rows of row_bytes (16..512, a power
 * of two) from an array of about array_bytes with 16-byte loads, row_bytes/16
 * lanes per row, and returns the bytes gathered per second.  A batched PPR
 * sweep gathers one row of its contrib tile (4 bytes per column) per edge,
 * so this is its gather roofline.  No counterpart in the reference. */
int pr_gpu_measure_row_gather_rate(int device, int64_t array_bytes, int row_bytes,
                                   double *bytes_per_s);

/* Upper limits of pr_gpu_run_noalloc (sizes of its fixed scratch area). */
#define PR_GPU_NOALLOC_MAX_VERTICES (1 << 20)
#define PR_GPU_NOALLOC_MAX_ITERS 1024

/* PageRankPull on a graph that is already in device memory, for callers that
 * cannot allocate GPU memory: this call makes no cudaMalloc / cudaFree and no
 * other allocating call.  Typical such callers are applications whose GPU
 * memory is handed out by their own pool allocator and reserved up front, and
 * services that must not take the device-wide synchronisation cudaMalloc /
 * cudaFree can cause while requests are in flight.  It has no counterpart in
 * the reference (which has no GPU path at all).
 *
 * The caller owns every buffer: in_off_dev (n+1) / in_nbr_dev (m) are the
 * in-CSR (int32, device), out_deg_dev the out-degree per vertex (device;
 * NULL for an undirected graph, whose in-row length is its out-degree), and
 * scores_out_dev (n floats, device) receives the scores.  sweeps_out and
 * err_trace (max_iters doubles) are host pointers and may be NULL.  stream
 * is a cudaStream_t (NULL = the legacy default stream); the call returns
 * after the solve.  The result is the reference's PageRankPull (init 1/N,
 * base (1-d)/N, contrib = score / out-degree, stop when the L1 change of a
 * sweep < epsilon or after max_iters sweeps) up to FP32 summation order.
 *
 * Its working memory is one fixed scratch area compiled into the library
 * (about 8.4 MB), so n may be at most PR_GPU_NOALLOC_MAX_VERTICES and
 * max_iters at most PR_GPU_NOALLOC_MAX_ITERS; larger requests return
 * PR_GPU_ERANGE with a message.  The CUDA runtime loads that area onto a GPU
 * at the first call on that GPU (the call looks up its device address with
 * cudaGetSymbolAddress, which loads the library's module there): that first
 * call reserves the area and the module's code, and the GPU holds them until
 * the process exits.  So make the first call on each device -- max_iters = 0
 * on any small graph you hold on the device will do -- before your pool
 * allocator reserves the GPU's memory and before any stream capture begins;
 * later calls allocate nothing.  The address is kept per device index and
 * belongs to the device's primary context (the one the CUDA runtime API
 * uses).  All calls share the area: calls whose GPU work overlaps in time
 * (several host threads, or several streams, on one device) race on it and
 * must be serialised by the caller.  Returns PR_GPU_OK or a PR_GPU_E* code; err_msg
 * (err_len bytes, nullable) receives a message on failure. */
int pr_gpu_run_noalloc(int device, int64_t n, int64_t m,
                       const int32_t *in_off_dev, const int32_t *in_nbr_dev,
                       const int32_t *out_deg_dev, int max_iters,
                       double epsilon, float damping, float *scores_out_dev,
                       int32_t *sweeps_out, double *err_trace, void *stream,
                       char *err_msg, size_t err_len);

/* Frees the handle and all its device memory (the mirror's counterpart of
 * ~CSRGraph, src/graph.h:165-167).  NULL is ignored. */
void pr_gpu_destroy(pr_gpu_t *h);

/* Message for the last failure on h (h may be NULL for create failures). */
const char *pr_gpu_last_error(const pr_gpu_t *h);

#ifdef __cplusplus
}
#endif

#endif /* GAPBS_PR_GPU_H_ */
