// benchmark.h -- trial harness, top-k and verifier of the pr_gpu CLI.
//
// BenchmarkKernel keeps the reference's trial loop and output
// (src/benchmark.h:97-123): "Graph has ..." stats, one "Trial Time:" per
// trial, analysis of the last trial with -a, "Verification: PASS|FAIL" and
// "Verification Time:" per trial with -v, then "Average Time:".
// TopK keeps the reference's selection rule exactly (src/benchmark.h:72-88),
// including its tie handling.
#ifndef GAPBS_B200_HOST_BENCHMARK_H_
#define GAPBS_B200_HOST_BENCHMARK_H_

#include <algorithm>
#include <functional>
#include <utility>
#include <vector>

#include "command_line.h"
#include "graph.h"
#include "util.h"

namespace gapbs_b200 {

// The k largest values: scan in key order, insert when the buffer is not full
// or the value beats the current minimum, keep the buffer sorted descending
// by (value, key), truncate to k.
template <typename KeyT, typename ValT>
std::vector<std::pair<ValT, KeyT>> TopK(const std::vector<std::pair<KeyT, ValT>> &kv, size_t k) {
  std::vector<std::pair<ValT, KeyT>> top;
  ValT min_so_far = 0;
  for (const auto &p : kv) {
    if (top.size() < k || p.second > min_so_far) {
      top.push_back(std::make_pair(p.second, p.first));
      std::sort(top.begin(), top.end(), std::greater<std::pair<ValT, KeyT>>());
      if (top.size() > k) top.resize(k);
      min_so_far = top.back().first;
    }
  }
  return top;
}

template <typename Result, typename KernelFn, typename StatsFn, typename VerifyFn>
void BenchmarkKernel(const PageRankCLI &cli, const HostGraph &g, KernelFn kernel,
                     StatsFn stats, VerifyFn verify) {
  g.PrintStats();
  double total = 0;
  WallTimer t;
  for (int iter = 0; iter < cli.num_trials(); iter++) {
    t.Start();
    Result result = kernel(g);
    t.Stop();
    PrintTime("Trial Time", t.Seconds());
    total += t.Seconds();
    if (cli.do_analysis() && iter == cli.num_trials() - 1) stats(g, result);
    if (cli.do_verify()) {
      t.Start();
      PrintLabel("Verification", verify(g, result) ? "PASS" : "FAIL");
      t.Stop();
      PrintTime("Verification Time", t.Seconds());
    }
  }
  PrintTime("Average Time", total / cli.num_trials());
}

}  // namespace gapbs_b200

#endif  // GAPBS_B200_HOST_BENCHMARK_H_
