// bfs_main.cc -- bfs_gpu: the reference's bfs command line (direction-
// optimizing breadth-first search, src/bfs.cc:248-263) with the B200 engine
// behind DOBFS.
//
// Same options, defaults and stdout lines as the reference binary: the same
// sources (its SourcePicker, restated below), "BFS Tree has ..." under -a,
// the reference's verifier (restated) under -v, and its step lines under -l.
#include <iostream>
#include <random>
#include <type_traits>
#include <vector>

#include "benchmark.h"
#include "builder.h"
#include "command_line.h"
#include "device_graph.h"
#include "graph.h"
#include "pr_gpu.h"
#include "util.h"

using namespace gapbs_b200;

namespace {

pr_gpu_t *g_engine = nullptr;

// Sources as the reference picks them (src/benchmark.h:46-68 with UniDist,
// src/generator.h:33-61): a std::mt19937_64 seeded kRandSeed whose draws are
// cut to the 32-bit unsigned node type, redrawn above the cutoff, reduced
// modulo N, until a vertex with out-edges comes up.  The cutoff is computed
// in 64 bits and stored in the 32-bit type, as there.
class SourcePicker {
 public:
  SourcePicker(const HostGraph &g, int64_t given) : g_(g), given_(given), rng_(kRandSeed) {
    typedef uint32_t U;
    const U max_value = static_cast<U>(g.num_nodes() - 1);
    no_mod_ = rng_.max() == static_cast<U>(max_value);
    mod_ = max_value + 1;
    const U remainder_sub_1 = static_cast<U>(rng_.max() % mod_);
    cutoff_ = (remainder_sub_1 == mod_ - 1) ? 0 : static_cast<U>(rng_.max() - remainder_sub_1);
  }

  NodeID PickNext() {
    if (given_ != -1) return static_cast<NodeID>(given_);
    NodeID source;
    do {
      source = Draw();
    } while (g_.out_degree(source) == 0);
    return source;
  }

 private:
  NodeID Draw() {
    uint32_t r = static_cast<uint32_t>(rng_());
    if (no_mod_) return static_cast<NodeID>(r);
    if (cutoff_ != 0)
      while (r >= cutoff_) r = static_cast<uint32_t>(rng_());
    return static_cast<NodeID>(r % mod_);
  }

  const HostGraph &g_;
  int64_t given_;
  std::mt19937_64 rng_;
  bool no_mod_;
  uint32_t mod_;
  uint32_t cutoff_;
};

// src/bfs.cc:99-174, computed by the engine.
std::vector<NodeID> DOBFS(const HostGraph &g, NodeID source, bool logging_enabled) {
  if (logging_enabled) PrintStep("Source", static_cast<int64_t>(source));
  std::vector<NodeID> parent(g.num_nodes());
  std::vector<pr_gpu_bfs_step_t> steps(1024);
  int nsteps = 0;
  int rc = pr_gpu_bfs(g_engine, source, parent.data(), steps.data(),
                      static_cast<int>(steps.size()), &nsteps);
  if (rc) Die(rc, std::string("pr_gpu_bfs failed: ") + pr_gpu_last_error(g_engine));
  if (logging_enabled)
    for (int i = 0; i < nsteps && i < static_cast<int>(steps.size()); i++)
      PrintStep(steps[i].kind, steps[i].seconds, steps[i].count);
  return parent;
}

// src/bfs.cc:177-189
void PrintBFSStats(const HostGraph &g, const std::vector<NodeID> &bfs_tree) {
  int64_t tree_size = 0, n_edges = 0;
  for (NodeID n = 0; n < g.num_nodes(); n++) {
    if (bfs_tree[n] >= 0) {
      n_edges += g.out_degree(n);
      tree_size++;
    }
  }
  std::cout << "BFS Tree has " << tree_size << " nodes and ";
  std::cout << n_edges << " edges" << std::endl;
}

// src/bfs.cc:201-245: a serial search for the depths, then every reached
// vertex's parent must be an in-neighbour one level up, the source its own
// parent, every unreached vertex -1.
bool BFSVerifier(const HostGraph &g, NodeID source, const std::vector<NodeID> &parent) {
  std::vector<int> depth(g.num_nodes(), -1);
  depth[source] = 0;
  std::vector<NodeID> to_visit;
  to_visit.reserve(g.num_nodes());
  to_visit.push_back(source);
  for (size_t i = 0; i < to_visit.size(); i++) {
    const NodeID u = to_visit[i];
    for (NodeID v : g.out_neigh(u)) {
      if (depth[v] == -1) {
        depth[v] = depth[u] + 1;
        to_visit.push_back(v);
      }
    }
  }
  for (NodeID u = 0; u < g.num_nodes(); u++) {
    if ((depth[u] != -1) && (parent[u] != -1)) {
      if (u == source) {
        if (!((parent[u] == u) && (depth[u] == 0))) {
          std::cout << "Source wrong" << std::endl;
          return false;
        }
        continue;
      }
      bool parent_found = false;
      for (NodeID v : g.in_neigh(u)) {
        if (v == parent[u]) {
          if (depth[v] != depth[u] - 1) {
            std::cout << "Wrong depths for " << u << " & " << v << std::endl;
            return false;
          }
          parent_found = true;
          break;
        }
      }
      if (!parent_found) {
        std::cout << "Couldn't find edge from " << parent[u] << " to " << u << std::endl;
        return false;
      }
    } else if (depth[u] != parent[u]) {
      std::cout << "Reachability mismatch" << std::endl;
      return false;
    }
  }
  return true;
}

}  // namespace

int main(int argc, char *argv[]) {
  PageRankCLI cli("breadth-first search", 1e-4, 20, false);
  if (!cli.Parse(argc, argv)) return -1;
  HostGraph g = AcquireGraph(cli.source(), &g_engine);
  SourcePicker sp(g, cli.start_vertex());
  auto BFSBound = [&sp, &cli](const HostGraph &graph) {
    return DOBFS(graph, sp.PickNext(), cli.logging_en());
  };
  SourcePicker vsp(g, cli.start_vertex());
  auto VerifierBound = [&vsp](const HostGraph &graph, const std::vector<NodeID> &parent) {
    return BFSVerifier(graph, vsp.PickNext(), parent);
  };
  BenchmarkKernel<std::vector<NodeID>>(cli, g, BFSBound, PrintBFSStats, VerifierBound);
  pr_gpu_destroy(g_engine);
  return 0;
}
