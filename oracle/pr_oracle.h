/*
 * pr_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the GAP Benchmark Suite's pull-direction Jacobi PageRank
 * (src/pr_spmv.cc, PageRankPull :35-61, PRVerifier :78-94) plus the
 * personalized-PageRank and adjoint extensions that the GPU engine adds.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker.  The product path never links
 * or calls it.
 *
 * Graphs are passed as CSR arrays with 64-bit offsets (the reference's
 * SGOffset, src/graph.h:94) and 32-bit neighbour ids (NodeID, src/benchmark.h:31).
 * For an undirected graph the caller passes the same arrays as "in" and "out"
 * (src/graph.h:138-143 aliases them the same way).
 *
 * Parity is pinned: oracle_pr_pull_f32 reproduces the reference's float
 * scores bit for bit on the reference's own graphs (golden fixtures under
 * tests/golden/ were produced by the reference compiled from source; see
 * oracle/Makefile and tests/golden/make_golden.py).
 */
#ifndef GAPBS_PR_ORACLE_H_
#define GAPBS_PR_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* FP32 mirror of PageRankPull (src/pr_spmv.cc:35-61): identical float
 * operations in identical order (contrib = score / out_degree, sequential
 * float sum over in-neighbours in list order, base + d * sum, |new-old| in
 * float added to a double error).  Returns the number of sweeps executed.
 * err_trace (nullable) receives one double per sweep. */
int oracle_pr_pull_f32(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                       const int64_t *out_off, int max_iters, double epsilon,
                       float damping, float *scores, double *err_trace);

/* Same algorithm with every quantity in double.  Returns sweeps. */
/* L1 distance of the FP32 mirror's scores from FP64 Jacobi after each of
 * nsweeps sweeps from the same start (the reference's rounding per sweep). */
void oracle_pr_rounding_f32(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                            const int64_t *out_off, int nsweeps, float damping, double *l1);
int oracle_pr_pull_f64(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                       const int64_t *out_off, int max_iters, double epsilon,
                       double damping, double *scores, double *err_trace);

/* PRVerifier (src/pr_spmv.cc:78-94): one serial push-direction sweep with
 * float incoming sums, L1 of base + d*incoming - score accumulated in double.
 * Returns the total error (the reference passes when it is < tolerance). */
double oracle_pr_verify_f32(int64_t n, const int64_t *out_off,
                            const int32_t *out_nbr, float damping,
                            const float *scores);

/* Double-precision residual sum_u |base + d * sum_{v in in(u)} s[v]/outdeg(v)
 * - s[u]| using a pull formulation (parallel, order-independent up to
 * double rounding).  Used as the size-independent property on large graphs. */
double oracle_pr_residual_f64(int64_t n, const int64_t *in_off,
                              const int32_t *in_nbr, const int64_t *out_off,
                              float damping, const float *scores);

/* Double-precision personalized-PageRank residual
 *   sum_u |(1-d) t[u] + d * sum_{v in in(u)} s[v]/outdeg(v) - s[u]|
 * of one FP32 score column s for teleport column t (unit weights).  After a
 * Jacobi sweep whose L1 change was c, the residual is at most d * c. */
double oracle_ppr_residual_f64(int64_t n, const int64_t *in_off,
                               const int32_t *in_nbr, const int64_t *out_off,
                               float damping, const float *t, const float *s);

/* Personalized PageRank, one column, FP64.
 *   s = (1-d) t + d P^T s,  P[v,u] = w(v->u) / S_v,  S_v = sum_u w(v->u)
 * in_w (nullable => unit weights) holds w(v->u) aligned with in_nbr (the
 * weight of the in-edge at the same position); rowsum holds S_v per vertex
 * (nullable => out-degree).  Start s_0 = t.  Stops when the L1 change of a
 * sweep is < epsilon or after max_iters sweeps.  Returns sweeps. */
int oracle_ppr_f64(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                   const double *in_w, const double *rowsum,
                   const int64_t *out_off, double damping, const double *t,
                   int max_iters, double epsilon, double *s, double *err_trace);

/* Same iteration started from s_init instead of t (warm start); used to
 * converge perturbed problems for finite differences. */
int oracle_ppr_f64_from(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                        const double *in_w, const double *rowsum,
                        const int64_t *out_off, double damping, const double *t,
                        const double *s_init, int max_iters, double epsilon,
                        double *s, double *err_trace);

/* Adjoint of L = w^T s at the PPR fixed point.  Solves
 *   lambda = w + d P lambda          (gather over OUT-neighbours)
 * from lambda_0 = w until the L1 change < epsilon * ||w||_1 or max_iters.
 * out_w (nullable => unit weights) is w(v->u) aligned with out_nbr.
 * Then
 *   grad_t[u]        = (1-d) lambda[u]
 *   grad_ew[e=(v,u)] = d s[v] / S_v * (lambda[u] - sum_u' P[v,u'] lambda[u'])
 * with grad_ew aligned with out_nbr.  Returns adjoint sweeps. */
int oracle_ppr_adjoint_f64(int64_t n, const int64_t *out_off,
                           const int32_t *out_nbr, const double *out_w,
                           double damping, const double *loss_w,
                           const double *s, int max_iters, double epsilon,
                           double *lambda, double *grad_t, double *grad_ew);

/* Connected components, the reference's Afforest (src/cc.cc:40-150) run
 * serially: two sampling rounds linking each vertex with its r-th
 * out-neighbour, compress, then every vertex outside the largest sampled
 * component links with its remaining out-neighbours (and, when directed,
 * all in-neighbours), compress.  comp[v] = the smallest vertex id of v's
 * component, as the reference's Link/Compress leave it. */
void oracle_cc_afforest(int64_t n, const int64_t *out_off, const int32_t *out_nbr,
                        const int64_t *in_off, const int32_t *in_nbr, int directed,
                        int32_t *comp);

/* Breadth-first depths from source (-1 when unreachable), the serial search
 * of the reference's BFSVerifier (src/bfs.cc:203-215). */
void oracle_bfs_depths(int64_t n, const int64_t *out_off, const int32_t *out_nbr,
                       int32_t source, int32_t *depth);

/* The reference's BFSVerifier (src/bfs.cc:201-245): 1 when parent[] is a
 * BFS tree from source (the source its own parent at depth 0, every other
 * reached vertex's parent an in-neighbour one level up, unreached vertices
 * -1), else 0. */
int oracle_bfs_verify(int64_t n, const int64_t *out_off, const int32_t *out_nbr,
                      const int64_t *in_off, const int32_t *in_nbr, int32_t source,
                      const int32_t *parent);

#ifdef __cplusplus
}
#endif

#endif  /* GAPBS_PR_ORACLE_H_ */
