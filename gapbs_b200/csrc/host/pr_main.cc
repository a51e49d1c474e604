// pr_main.cc -- pr_gpu: the pr_spmv command line with the B200 engine behind
// PageRankPull.
//
// Same options, defaults and stdout lines as the reference binary
// (src/pr_spmv.cc:97-111 + src/benchmark.h:97-123), so the reference's test
// harness (test/test.mk:73-86: `./pr_gpu -g10 -vn1` must print
// "Verification:           PASS") runs unchanged against it.  Synthetic
// graphs (-g / -u) are generated and built on the GPU, identical to the
// reference's (pr_gpu_generate; "Generate Time:" covers the host permutation
// and the device build, "Build Time:" the copy of the CSR to the host for
// the verifier).  Graphs read from files are built on the host and uploaded
// once before the timed trials, on their own "Upload Time:" line.
#include <cmath>
#include <cstdio>
#include <iostream>
#include <vector>

#include "benchmark.h"
#include "builder.h"
#include "command_line.h"
#include "graph.h"
#include "pr_gpu.h"
#include "util.h"

using namespace gapbs_b200;

typedef float ScoreT;
static const float kDamp = 0.85f;  // src/pr_spmv.cc:33

namespace {

pr_gpu_t *g_engine = nullptr;

[[noreturn]] void Die(int code, const std::string &msg) {
  std::cout << msg << std::endl;
  std::exit(code);
}

// One-time upload of the CSR (int32 offsets) to device 0.
void UploadGraph(const HostGraph &g) {
  WallTimer t;
  t.Start();
  int rc = pr_gpu_create(&g_engine, 0);
  if (rc) Die(rc, "pr_gpu_create failed: no usable CUDA device");
  const int64_t n = g.num_nodes();
  const int64_t m = g.out_entries();
  if (m > 0x7fffffffLL - 8) Die(PR_GPU_ERANGE, "graph exceeds int32 offsets");
  std::vector<int32_t> out_off(n + 1), in_off;
  for (int64_t i = 0; i <= n; i++) out_off[i] = static_cast<int32_t>(g.out_off_ptr()[i]);
  if (g.directed()) {
    in_off.resize(n + 1);
    for (int64_t i = 0; i <= n; i++) in_off[i] = static_cast<int32_t>(g.in_off_ptr()[i]);
  }
  rc = pr_gpu_upload(g_engine, n, m, out_off.data(), g.out_nbr_ptr(),
                     g.directed() ? in_off.data() : nullptr,
                     g.directed() ? g.in_nbr_ptr() : nullptr, nullptr);
  if (rc) Die(rc, std::string("pr_gpu_upload failed: ") + pr_gpu_last_error(g_engine));
  t.Stop();
  PrintTime("Upload Time", t.Seconds());
}

// -g / -u on the device: the reference's graph, uploaded as it is built.
// Returns false (host path) for sizes the device path does not cover.
bool GenerateOnDevice(const GraphSource &src, HostGraph *g) {
  if (src.scale < 1 || src.scale > 30 || src.degree < 0) return false;
  if ((int64_t(2) * src.degree) << src.scale > 0x7fffffffLL - 8) return false;
  WallTimer t;
  t.Start();
  int rc = pr_gpu_create(&g_engine, 0);
  if (rc) Die(rc, "pr_gpu_create failed: no usable CUDA device");
  std::vector<NodeID> perm;
  if (!src.uniform) {
    perm.resize(size_t(1) << src.scale);
    RMatPermutation(src.scale, perm.data());
  }
  int64_t n = 0, m = 0;
  rc = pr_gpu_generate(g_engine, src.uniform ? 1 : 0, src.scale, src.degree,
                       src.uniform ? nullptr : perm.data(), &n, &m);
  if (rc) Die(rc, std::string("pr_gpu_generate failed: ") + pr_gpu_last_error(g_engine));
  t.Stop();
  PrintTime("Generate Time", t.Seconds());
  t.Start();
  Buffer<Offset> off(static_cast<size_t>(n + 1));
  Buffer<NodeID> nbr(static_cast<size_t>(m > 0 ? m : 1));
  rc = pr_gpu_download_csr(g_engine, off.data(), nbr.data());
  if (rc) Die(rc, std::string("pr_gpu_download_csr failed: ") + pr_gpu_last_error(g_engine));
  *g = HostGraph::Undirected(n, std::move(off), std::move(nbr));
  t.Stop();
  PrintTime("Build Time", t.Seconds());
  return true;
}

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
// L1 residual, accumulated in double, must be below the tolerance.
bool PRVerifier(const HostGraph &g, const std::vector<ScoreT> &scores, double target_error) {
  const ScoreT base_score = (1.0f - kDamp) / g.num_nodes();
  std::vector<ScoreT> incoming(g.num_nodes(), 0);
  double error = 0;
  for (NodeID u = 0; u < g.num_nodes(); u++) {
    const ScoreT contrib = scores[u] / g.out_degree(u);
    for (NodeID v : g.out_neigh(u)) incoming[v] += contrib;
  }
  for (NodeID n = 0; n < g.num_nodes(); n++)
    error += std::fabs(base_score + kDamp * incoming[n] - scores[n]);
  PrintTime("Total Error", error);
  return error < target_error;
}

}  // namespace

int main(int argc, char *argv[]) {
  PageRankCLI cli("pagerank", 1e-4, 20);
  if (!cli.Parse(argc, argv)) return -1;
  HostGraph g;
  if (!GenerateOnDevice(cli.source(), &g)) {
    try {
      g = MakeGraph(cli.source(), true);
    } catch (const BuildError &e) {
      Die(e.code(), e.what());
    }
    UploadGraph(g);
  }
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
