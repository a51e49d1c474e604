// ref_shim.cc -- TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own PageRankPull / PRVerifier / Builder through a
// small C ABI so that tests and the CPU baseline can run the UNMODIFIED
// reference code on the same graphs the GPU engine sees.  This file is
// compiled (by oracle/Makefile) against the reference sources where they lie;
// the result goes to oracle/_ref/ only and is never linked into the product.
//
// Entry points wrap: src/pr_spmv.cc PageRankPull (:35-61), PRVerifier
// (:78-94); src/pr.cc PageRankPullGS (:34-61); src/builder.h
// BuilderBase::MakeGraph (:343-364);
// src/graph.h CSRGraph constructors (:131-151) and GenIndex (:242-249).

#include <chrono>
#include <cstring>

#define main gapbs_reference_pr_spmv_main
#include "pr_spmv.cc"
#undef main

// The reference's Gauss-Seidel PageRank (src/pr.cc:34-61).  pr.cc defines
// the same names as pr_spmv.cc (ScoreT, kDamp, PrintTopScores, PRVerifier,
// main), so it is compiled inside a namespace of its own (the headers it
// includes are already in, behind their include guards, so only its own
// definitions land there), with its two functions over Graph renamed so
// that argument-dependent lookup from its main cannot also find the global
// ones.
#define main gapbs_reference_pr_main
#define PRVerifier PRVerifierGS
#define PrintTopScores PrintTopScoresGS
namespace gs {
#include "pr.cc"
}  // namespace gs
#undef PrintTopScores
#undef PRVerifier
#undef main

namespace {

struct RefGraph {
  Graph g;
};

void FillOffsets(pvector<SGOffset> *dst, int64_t n, const int64_t *off) {
  for (int64_t i = 0; i <= n; i++) (*dst)[i] = off[i];
}

}  // namespace

extern "C" {

// Builds a graph exactly as the reference binary does for the given argv
// (e.g. {"pr_spmv", "-g", "10"}).  Returns nullptr when parsing fails.
void *ref_make_graph(int argc, char **argv) {
  CLPageRank cli(argc, argv, "pagerank", 1e-4, 20);
  optind = 1;  // getopt state is process-global
  if (!cli.ParseArgs()) return nullptr;
  Builder b(cli);
  RefGraph *rg = new RefGraph();
  rg->g = b.MakeGraph();
  return rg;
}

// Wraps caller CSR arrays (copied) into a reference CSRGraph.
void *ref_graph_from_csr(int64_t n, int directed, const int64_t *out_off,
                         const int32_t *out_nbr, const int64_t *in_off,
                         const int32_t *in_nbr) {
  RefGraph *rg = new RefGraph();
  int64_t m_out = out_off[n];
  pvector<SGOffset> offs(n + 1);
  FillOffsets(&offs, n, out_off);
  NodeID *oneigh = new NodeID[m_out > 0 ? m_out : 1];
  if (m_out) std::memcpy(oneigh, out_nbr, sizeof(NodeID) * m_out);
  NodeID **oindex = Graph::GenIndex(offs, oneigh);
  if (!directed) {
    rg->g = Graph(n, oindex, oneigh);
  } else {
    int64_t m_in = in_off[n];
    pvector<SGOffset> ioffs(n + 1);
    FillOffsets(&ioffs, n, in_off);
    NodeID *ineigh = new NodeID[m_in > 0 ? m_in : 1];
    if (m_in) std::memcpy(ineigh, in_nbr, sizeof(NodeID) * m_in);
    NodeID **iindex = Graph::GenIndex(ioffs, ineigh);
    rg->g = Graph(n, oindex, oneigh, iindex, ineigh);
  }
  return rg;
}

void ref_free_graph(void *h) { delete static_cast<RefGraph *>(h); }

int64_t ref_num_nodes(void *h) { return static_cast<RefGraph *>(h)->g.num_nodes(); }
int64_t ref_num_edges(void *h) { return static_cast<RefGraph *>(h)->g.num_edges(); }
int64_t ref_num_edges_directed(void *h) {
  return static_cast<RefGraph *>(h)->g.num_edges_directed();
}
int ref_directed(void *h) { return static_cast<RefGraph *>(h)->g.directed(); }

// Copies the CSR out: offsets relative to the first neighbour (as
// CSRGraph::VertexOffsets does, src/graph.h:251-259).  in_* may be null.
void ref_export_csr(void *h, int64_t *out_off, int32_t *out_nbr,
                    int64_t *in_off, int32_t *in_nbr) {
  const Graph &g = static_cast<RefGraph *>(h)->g;
  pvector<SGOffset> o = g.VertexOffsets(false);
  for (int64_t i = 0; i <= g.num_nodes(); i++) out_off[i] = o[i];
  if (o[g.num_nodes()])
    std::memcpy(out_nbr, g.out_neigh(0).begin(),
                sizeof(int32_t) * o[g.num_nodes()]);
  if (in_off) {
    pvector<SGOffset> io = g.VertexOffsets(true);
    for (int64_t i = 0; i <= g.num_nodes(); i++) in_off[i] = io[i];
    if (in_nbr && io[g.num_nodes()])
      std::memcpy(in_nbr, g.in_neigh(0).begin(),
                  sizeof(int32_t) * io[g.num_nodes()]);
  }
}

// Runs the reference PageRankPull; logging prints the per-sweep lines.
void ref_pagerank_pull(void *h, int max_iters, double epsilon, int logging,
                       float *scores_out) {
  const Graph &g = static_cast<RefGraph *>(h)->g;
  pvector<ScoreT> s = PageRankPull(g, max_iters, epsilon, logging != 0);
  std::memcpy(scores_out, s.data(), sizeof(float) * g.num_nodes());
  std::fflush(stdout);
}

// Wall-clock seconds of `trials` back-to-back PageRankPull calls (the same
// timing BenchmarkKernel applies, src/benchmark.h:104-111).  Fills
// per_trial (nullable) with each trial's seconds.
double ref_time_pagerank_pull(void *h, int max_iters, double epsilon,
                              int trials, double *per_trial) {
  const Graph &g = static_cast<RefGraph *>(h)->g;
  double total = 0;
  for (int t = 0; t < trials; t++) {
    auto t0 = std::chrono::steady_clock::now();
    pvector<ScoreT> s = PageRankPull(g, max_iters, epsilon, false);
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    if (per_trial) per_trial[t] = sec;
    total += sec;
  }
  return total;
}

// Runs the reference Gauss-Seidel PageRankPullGS; logging prints the
// per-iteration lines.
void ref_pagerank_gs(void *h, int max_iters, double epsilon, int logging, float *scores_out) {
  const Graph &g = static_cast<RefGraph *>(h)->g;
  pvector<gs::ScoreT> s = gs::PageRankPullGS(g, max_iters, epsilon, logging != 0);
  std::memcpy(scores_out, s.data(), sizeof(float) * g.num_nodes());
  std::fflush(stdout);
}

// Wall-clock seconds of `trials` back-to-back PageRankPullGS calls, as
// ref_time_pagerank_pull does for the Jacobi kernel.
double ref_time_pagerank_gs(void *h, int max_iters, double epsilon, int trials,
                            double *per_trial) {
  const Graph &g = static_cast<RefGraph *>(h)->g;
  double total = 0;
  for (int t = 0; t < trials; t++) {
    auto t0 = std::chrono::steady_clock::now();
    pvector<gs::ScoreT> s = gs::PageRankPullGS(g, max_iters, epsilon, false);
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    if (per_trial) per_trial[t] = sec;
    total += sec;
  }
  return total;
}

// Runs the reference PRVerifier (prints "Total Error:"); returns PASS (1).
int ref_pr_verifier(void *h, const float *scores, double tolerance) {
  const Graph &g = static_cast<RefGraph *>(h)->g;
  pvector<ScoreT> s(g.num_nodes());
  std::memcpy(s.data(), scores, sizeof(float) * g.num_nodes());
  bool ok = PRVerifier(g, s, tolerance);
  std::fflush(stdout);
  return ok ? 1 : 0;
}

}  // extern "C"
