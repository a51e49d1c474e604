/*
 * pr_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement of the reference's pull-direction Jacobi PageRank and of
 * the PPR / adjoint mathematics the GPU engine implements.  Every function
 * cites the reference lines it follows.  Compiled with -ffp-contract=off and
 * without -march so that the FP32 mirror performs exactly the float
 * operations the reference performs (no fused multiply-add).
 */
#include "pr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline int64_t deg_of(const int64_t *off, int64_t v) {
  return off[v + 1] - off[v];
}

/* src/pr_spmv.cc:35-61 */
int oracle_pr_pull_f32(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                       const int64_t *out_off, int max_iters, double epsilon,
                       float damping, float *scores, double *err_trace) {
  /* :37-38 -- init and base are computed in float from num_nodes */
  const float init_score = 1.0f / (float)n;
  const float base_score = (1.0f - damping) / (float)n;
  float *contrib = (float *)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
  int sweeps = 0;
  for (int64_t u = 0; u < n; u++) scores[u] = init_score;        /* :39 */
  for (int iter = 0; iter < max_iters; iter++) {                    /* :41 */
    double error = 0;
    for (int64_t v = 0; v < n; v++)                                 /* :43-45 */
      contrib[v] = scores[v] / (float)deg_of(out_off, v);
    for (int64_t u = 0; u < n; u++) {                               /* :46-54 */
      float incoming_total = 0;
      for (int64_t e = in_off[u]; e < in_off[u + 1]; e++)
        incoming_total += contrib[in_nbr[e]];
      float old_score = scores[u];
      scores[u] = base_score + damping * incoming_total;
      error += fabsf(scores[u] - old_score);
    }
    if (err_trace) err_trace[iter] = error;
    sweeps = iter + 1;
    if (error < epsilon) break;                                     /* :57-58 */
  }
  free(contrib);
  return sweeps;
}

/* The reference's own rounding error per sweep: the FP32 mirror of
 * src/pr_spmv.cc:35-61 and the same Jacobi sweeps in double, run side by
 * side from the same start for exactly nsweeps sweeps (no stop test);
 * l1[k] = sum_u |s32_k[u] - s64_k[u]| after sweep k. */
void oracle_pr_rounding_f32(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                            const int64_t *out_off, int nsweeps, float damping, double *l1) {
  const float init32 = 1.0f / (float)n, base32 = (1.0f - damping) / (float)n;
  const double init64 = 1.0 / (double)n, base64 = (1.0 - (double)damping) / (double)n;
  const size_t cap = (size_t)(n > 0 ? n : 1);
  float *s32 = (float *)malloc(sizeof(float) * cap), *c32 = (float *)malloc(sizeof(float) * cap);
  double *s64 = (double *)malloc(sizeof(double) * cap), *c64 = (double *)malloc(sizeof(double) * cap);
  for (int64_t u = 0; u < n; u++) {
    s32[u] = init32;
    s64[u] = init64;
  }
  for (int k = 0; k < nsweeps; k++) {
    for (int64_t v = 0; v < n; v++) {
      const int64_t d = deg_of(out_off, v);
      c32[v] = s32[v] / (float)d;
      c64[v] = d ? s64[v] / (double)d : 0.0;
    }
    double acc = 0;
    for (int64_t u = 0; u < n; u++) {
      float t32 = 0;
      double t64 = 0;
      for (int64_t e = in_off[u]; e < in_off[u + 1]; e++) {
        t32 += c32[in_nbr[e]];
        t64 += c64[in_nbr[e]];
      }
      s32[u] = base32 + damping * t32;
      s64[u] = base64 + (double)damping * t64;
      acc += fabs((double)s32[u] - s64[u]);
    }
    l1[k] = acc;
  }
  free(s32);
  free(c32);
  free(s64);
  free(c64);
}

/* src/pr_spmv.cc:35-61 with double everywhere */
int oracle_pr_pull_f64(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                       const int64_t *out_off, int max_iters, double epsilon,
                       double damping, double *scores, double *err_trace) {
  const double init_score = 1.0 / (double)n;
  const double base_score = (1.0 - damping) / (double)n;
  double *contrib = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  int sweeps = 0;
  for (int64_t u = 0; u < n; u++) scores[u] = init_score;
  for (int iter = 0; iter < max_iters; iter++) {
    double error = 0;
    for (int64_t v = 0; v < n; v++) {
      int64_t d = deg_of(out_off, v);
      contrib[v] = d ? scores[v] / (double)d : 0.0;
    }
    for (int64_t u = 0; u < n; u++) {
      double incoming_total = 0;
      for (int64_t e = in_off[u]; e < in_off[u + 1]; e++)
        incoming_total += contrib[in_nbr[e]];
      double old_score = scores[u];
      scores[u] = base_score + damping * incoming_total;
      error += fabs(scores[u] - old_score);
    }
    if (err_trace) err_trace[iter] = error;
    sweeps = iter + 1;
    if (error < epsilon) break;
  }
  free(contrib);
  return sweeps;
}

/* src/pr_spmv.cc:78-94 */
double oracle_pr_verify_f32(int64_t n, const int64_t *out_off,
                            const int32_t *out_nbr, float damping,
                            const float *scores) {
  const float base_score = (1.0f - damping) / (float)n;
  float *incoming = (float *)calloc((size_t)(n > 0 ? n : 1), sizeof(float));
  double error = 0;
  for (int64_t u = 0; u < n; u++) {                                 /* :82-87 */
    float outgoing_contrib = scores[u] / (float)deg_of(out_off, u);
    for (int64_t e = out_off[u]; e < out_off[u + 1]; e++)
      incoming[out_nbr[e]] += outgoing_contrib;
  }
  for (int64_t v = 0; v < n; v++)                                   /* :88-91 */
    error += fabsf(base_score + damping * incoming[v] - scores[v]);
  free(incoming);
  return error;
}

double oracle_pr_residual_f64(int64_t n, const int64_t *in_off,
                              const int32_t *in_nbr, const int64_t *out_off,
                              float damping, const float *scores) {
  const double base = (double)((1.0f - damping) / (float)n);
  const double d = (double)damping;
  double error = 0;
  #pragma omp parallel for reduction(+ : error) schedule(dynamic, 4096)
  for (int64_t u = 0; u < n; u++) {
    double acc = 0;
    for (int64_t e = in_off[u]; e < in_off[u + 1]; e++) {
      int32_t v = in_nbr[e];
      acc += (double)scores[v] / (double)deg_of(out_off, v);
    }
    error += fabs(base + d * acc - (double)scores[u]);
  }
  return error;
}

double oracle_ppr_residual_f64(int64_t n, const int64_t *in_off,
                               const int32_t *in_nbr, const int64_t *out_off,
                               float damping, const float *t, const float *s) {
  const double d = (double)damping;
  double error = 0;
  #pragma omp parallel for reduction(+ : error) schedule(dynamic, 4096)
  for (int64_t u = 0; u < n; u++) {
    double acc = 0;
    for (int64_t e = in_off[u]; e < in_off[u + 1]; e++) {
      int32_t v = in_nbr[e];
      acc += (double)s[v] / (double)deg_of(out_off, v);
    }
    error += fabs((1.0 - d) * (double)t[u] + d * acc - (double)s[u]);
  }
  return error;
}

/* Row sums S_v: explicit or out-degree. */
static inline double rowsum_of(const double *rowsum, const int64_t *out_off,
                               int64_t v) {
  return rowsum ? rowsum[v] : (double)deg_of(out_off, v);
}

int oracle_ppr_f64_from(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                        const double *in_w, const double *rowsum,
                        const int64_t *out_off, double damping, const double *t,
                        const double *s_init, int max_iters, double epsilon,
                        double *s, double *err_trace) {
  double *contrib = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  int sweeps = 0;
  if (s != s_init) memcpy(s, s_init, sizeof(double) * (size_t)n);
  for (int iter = 0; iter < max_iters; iter++) {
    double error = 0;
    for (int64_t v = 0; v < n; v++) {
      double sv = rowsum_of(rowsum, out_off, v);
      contrib[v] = sv != 0.0 ? s[v] / sv : 0.0;
    }
    #pragma omp parallel for reduction(+ : error) schedule(dynamic, 4096)
    for (int64_t u = 0; u < n; u++) {
      double acc = 0;
      for (int64_t e = in_off[u]; e < in_off[u + 1]; e++)
        acc += (in_w ? in_w[e] : 1.0) * contrib[in_nbr[e]];
      double nv = (1.0 - damping) * t[u] + damping * acc;
      error += fabs(nv - s[u]);
      s[u] = nv;
    }
    if (err_trace) err_trace[iter] = error;
    sweeps = iter + 1;
    if (error < epsilon) break;
  }
  free(contrib);
  return sweeps;
}

int oracle_ppr_f64(int64_t n, const int64_t *in_off, const int32_t *in_nbr,
                   const double *in_w, const double *rowsum,
                   const int64_t *out_off, double damping, const double *t,
                   int max_iters, double epsilon, double *s, double *err_trace) {
  return oracle_ppr_f64_from(n, in_off, in_nbr, in_w, rowsum, out_off, damping,
                             t, t, max_iters, epsilon, s, err_trace);
}

int oracle_ppr_adjoint_f64(int64_t n, const int64_t *out_off,
                           const int32_t *out_nbr, const double *out_w,
                           double damping, const double *loss_w,
                           const double *s, int max_iters, double epsilon,
                           double *lambda, double *grad_t, double *grad_ew) {
  double *next = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *plam = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double wnorm = 0;
  for (int64_t v = 0; v < n; v++) wnorm += fabs(loss_w[v]);
  const double tol = epsilon * wnorm;
  int sweeps = 0;
  memcpy(lambda, loss_w, sizeof(double) * (size_t)n);
  for (int iter = 0; iter < max_iters; iter++) {
    double error = 0;
    #pragma omp parallel for reduction(+ : error) schedule(dynamic, 4096)
    for (int64_t v = 0; v < n; v++) {
      double acc = 0, sv = 0;
      for (int64_t e = out_off[v]; e < out_off[v + 1]; e++) {
        double w = out_w ? out_w[e] : 1.0;
        acc += w * lambda[out_nbr[e]];
        sv += w;
      }
      double pl = sv != 0.0 ? acc / sv : 0.0;
      next[v] = loss_w[v] + damping * pl;
      error += fabs(next[v] - lambda[v]);
    }
    memcpy(lambda, next, sizeof(double) * (size_t)n);
    sweeps = iter + 1;
    if (error < tol) break;
  }
  /* P lambda at the final lambda, for the edge-weight gradient */
  #pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < n; v++) {
    double acc = 0, sv = 0;
    for (int64_t e = out_off[v]; e < out_off[v + 1]; e++) {
      double w = out_w ? out_w[e] : 1.0;
      acc += w * lambda[out_nbr[e]];
      sv += w;
    }
    plam[v] = sv != 0.0 ? acc / sv : 0.0;
    if (grad_ew) {
      for (int64_t e = out_off[v]; e < out_off[v + 1]; e++)
        grad_ew[e] = sv != 0.0
            ? damping * s[v] / sv * (lambda[out_nbr[e]] - plam[v]) : 0.0;
    }
  }
  if (grad_t)
    for (int64_t u = 0; u < n; u++) grad_t[u] = (1.0 - damping) * lambda[u];
  free(next);
  free(plam);
  return sweeps;
}

/* ---- connected components (src/cc.cc) ---------------------------------- */

/* :40-55, serial: hook the larger root under the smaller one. */
static void cc_link(int32_t u, int32_t v, int32_t *comp) {
  int32_t p1 = comp[u], p2 = comp[v];
  while (p1 != p2) {
    int32_t high = p1 > p2 ? p1 : p2;
    int32_t low = p1 + (p2 - high);
    int32_t p_high = comp[high];
    if (p_high == low) break;
    if (p_high == high) {
      comp[high] = low;
      break;
    }
    p1 = comp[comp[high]];
    p2 = comp[low];
  }
}

/* :58-66 */
static void cc_compress(int64_t n, int32_t *comp) {
  for (int64_t v = 0; v < n; v++)
    while (comp[v] != comp[comp[v]]) comp[v] = comp[comp[v]];
}

void oracle_cc_afforest(int64_t n, const int64_t *out_off, const int32_t *out_nbr,
                        const int64_t *in_off, const int32_t *in_nbr, int directed,
                        int32_t *comp) {
  const int rounds = 2; /* :92 */
  for (int64_t v = 0; v < n; v++) comp[v] = (int32_t)v;
  for (int r = 0; r < rounds; r++) { /* :100-110 */
    for (int64_t u = 0; u < n; u++)
      if (out_off[u] + r < out_off[u + 1]) cc_link((int32_t)u, out_nbr[out_off[u] + r], comp);
    cc_compress(n, comp);
  }
  /* :69-87: the most frequent label among a sample; the final labels do not
   * depend on which component is skipped, so a fixed stride sample serves */
  int32_t giant = 0;
  if (n > 0) {
    int64_t best = 0;
    const int64_t step = n > 1024 ? n / 1024 : 1;
    for (int64_t a = 0; a < n; a += step) {
      int64_t count = 0;
      for (int64_t b = 0; b < n; b += step)
        if (comp[b] == comp[a]) count++;
      if (count > best) {
        best = count;
        giant = comp[a];
      }
    }
  }
  for (int64_t u = 0; u < n; u++) { /* :116-146 */
    if (comp[u] == giant) continue;
    for (int64_t e = out_off[u] + rounds; e < out_off[u + 1]; e++)
      cc_link((int32_t)u, out_nbr[e], comp);
    if (directed)
      for (int64_t e = in_off[u]; e < in_off[u + 1]; e++) cc_link((int32_t)u, in_nbr[e], comp);
  }
  cc_compress(n, comp);
}

/* ---- breadth-first search (src/bfs.cc) ---------------------------------- */

void oracle_bfs_depths(int64_t n, const int64_t *out_off, const int32_t *out_nbr,
                       int32_t source, int32_t *depth) {
  int32_t *queue = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  for (int64_t v = 0; v < n; v++) depth[v] = -1;
  int64_t head = 0, tail = 0;
  depth[source] = 0;
  queue[tail++] = source;
  while (head < tail) {
    const int32_t u = queue[head++];
    for (int64_t e = out_off[u]; e < out_off[u + 1]; e++) {
      const int32_t v = out_nbr[e];
      if (depth[v] == -1) {
        depth[v] = depth[u] + 1;
        queue[tail++] = v;
      }
    }
  }
  free(queue);
}

int oracle_bfs_verify(int64_t n, const int64_t *out_off, const int32_t *out_nbr,
                      const int64_t *in_off, const int32_t *in_nbr, int32_t source,
                      const int32_t *parent) {
  int32_t *depth = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  oracle_bfs_depths(n, out_off, out_nbr, source, depth);
  int ok = 1;
  for (int64_t u = 0; u < n && ok; u++) {
    if (depth[u] != -1 && parent[u] != -1) {
      if (u == source) {
        if (!(parent[u] == u && depth[u] == 0)) ok = 0;
        continue;
      }
      int found = 0;
      for (int64_t e = in_off[u]; e < in_off[u + 1]; e++) {
        if (in_nbr[e] == parent[u]) {
          if (depth[in_nbr[e]] != depth[u] - 1) ok = 0;
          found = 1;
          break;
        }
      }
      if (!found) ok = 0;
    } else if (depth[u] != parent[u]) {
      ok = 0;
    }
  }
  free(depth);
  return ok;
}
