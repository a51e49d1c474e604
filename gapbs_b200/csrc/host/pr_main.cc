// pr_main.cc -- pr_gpu: the pr_spmv command line with the B200 engine behind
// PageRankPull.
//
// Same options, defaults and stdout lines as the reference binary
// (src/pr_spmv.cc:97-111 + src/benchmark.h:97-123), so the reference's test
// harness (test/test.mk:73-86: `./pr_gpu -g10 -vn1` must print
// "Verification:           PASS") runs unchanged against it.  Synthetic
// graphs (-g / -u) are generated and built on the GPU, identical to the
// reference's (pr_gpu_generate; "Generate Time:" covers the host permutation
// and the device build, "Build Time:" the copy of the CSR to the host graph
// the command line holds, as the other kernels' verifiers need it).  Graphs
// read from files are built on the host and uploaded once before the timed
// trials, on their own "Upload Time:" line.  -v runs the reference's check
// on the device (pr_gpu_verify).
#include <cstdio>
#include <iostream>
#include <vector>

#include "benchmark.h"
#include "builder.h"
#include "command_line.h"
#include "device_graph.h"
#include "graph.h"
#include "pr_gpu.h"
#include "util.h"

using namespace gapbs_b200;

typedef float ScoreT;
static const float kDamp = 0.85f;  // src/pr_spmv.cc:33

namespace {

pr_gpu_t *g_engine = nullptr;

// src/pr_spmv.cc:35-61, computed by the engine.
std::vector<ScoreT> PageRankPull(const HostGraph &g, int max_iters, double epsilon = 0,
                                 bool logging_enabled = false) {
  std::vector<ScoreT> scores(g.num_nodes());
  std::vector<double> trace(max_iters > 0 ? max_iters : 1);
  int32_t sweeps = 0;
  int rc = pr_gpu_run(g_engine, max_iters, epsilon, kDamp, 1, nullptr, scores.data(), &sweeps,
                      trace.data());
  if (rc) Die(rc, std::string("pr_gpu_run failed: ") + pr_gpu_last_error(g_engine));
  if (logging_enabled)
    for (int i = 0; i < sweeps; i++) PrintStep(i, trace[i]);
  return scores;
}

// src/pr_spmv.cc:64-73
void PrintTopScores(const HostGraph &g, const std::vector<ScoreT> &scores) {
  std::vector<std::pair<NodeID, ScoreT>> kv(g.num_nodes());
  for (NodeID n = 0; n < g.num_nodes(); n++) kv[n] = std::make_pair(n, scores[n]);
  for (const auto &p : TopK(kv, 5)) std::cout << p.second << ":" << p.first << std::endl;
}

// src/pr_spmv.cc:78-94: one serial push-direction sweep with float sums; the
// L1 residual, accumulated in double, must be below the tolerance.  Computed
// by the engine (pr_gpu_verify) on the graph it holds, which is this one: the
// same error bit for bit on the builder's sorted rows, in milliseconds where
// the serial loop takes seconds on the largest graphs.
bool PRVerifier(const HostGraph &g, const std::vector<ScoreT> &scores, double target_error) {
  (void)g;
  double error = 0;
  const int rc = pr_gpu_verify(g_engine, scores.data(), kDamp, &error);
  if (rc) Die(rc, std::string("pr_gpu_verify failed: ") + pr_gpu_last_error(g_engine));
  PrintTime("Total Error", error);
  return error < target_error;
}

}  // namespace

int main(int argc, char *argv[]) {
  PageRankCLI cli("pagerank", 1e-4, 20);
  if (!cli.Parse(argc, argv)) return -1;
  HostGraph g = AcquireGraph(cli.source(), &g_engine);
  auto PRBound = [&cli](const HostGraph &graph) {
    return PageRankPull(graph, cli.max_iters(), cli.tolerance(), cli.logging_en());
  };
  auto VerifierBound = [&cli](const HostGraph &graph, const std::vector<ScoreT> &scores) {
    return PRVerifier(graph, scores, cli.tolerance());
  };
  BenchmarkKernel<std::vector<ScoreT>>(cli, g, PRBound, PrintTopScores, VerifierBound);
  pr_gpu_destroy(g_engine);
  return 0;
}
