// cc_main.cc -- cc_gpu: the reference's cc command line (Afforest connected
// components, src/cc.cc:219-229) with the B200 engine behind Afforest.
//
// Same options, defaults and stdout lines as the reference binary; the
// labels are the reference's (every vertex labelled with the smallest id of
// its component), so -a prints the same clusters and -v runs the reference's
// verifier, restated below.
#include <iostream>
#include <unordered_map>
#include <utility>
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

// src/cc.cc:89-150, computed by the engine.
std::vector<NodeID> Afforest(const HostGraph &g) {
  std::vector<NodeID> comp(g.num_nodes());
  int rc = pr_gpu_connected_components(g_engine, comp.data());
  if (rc) Die(rc, std::string("pr_gpu_connected_components failed: ") + pr_gpu_last_error(g_engine));
  return comp;
}

// src/cc.cc:153-170: a blank line, the (at most) five largest components
// as "label:size" lines, then the number of components.  Sizes are tallied
// in a hash map and given to TopK in that map's iteration order, as the
// reference's are: which of several equally large components make the list
// depends on that order, so the same container and insertion sequence keep
// the printed lines identical.
void PrintCompStats(const HostGraph &, const std::vector<NodeID> &comp) {
  std::unordered_map<NodeID, NodeID> size_of;
  for (size_t v = 0; v < comp.size(); v++) ++size_of[comp[v]];
  const std::vector<std::pair<NodeID, NodeID>> sizes(size_of.begin(), size_of.end());
  const auto largest = TopK(sizes, 5);
  std::cout << '\n' << largest.size() << " biggest clusters\n";
  for (const auto &entry : largest) std::cout << entry.second << ':' << entry.first << '\n';
  std::cout << "There are " << size_of.size() << " components" << std::endl;
}

// src/cc.cc:173-216: one search per label, as if undirected; every vertex
// must be reached and every reached vertex must carry the search's label.
bool CCVerifier(const HostGraph &g, const std::vector<NodeID> &comp) {
  std::unordered_map<NodeID, NodeID> label_to_source;
  for (NodeID n = 0; n < g.num_nodes(); n++) label_to_source[comp[n]] = n;
  std::vector<bool> visited(g.num_nodes(), false);
  std::vector<NodeID> frontier;
  frontier.reserve(g.num_nodes());
  for (auto label_source : label_to_source) {
    const NodeID label = label_source.first;
    frontier.clear();
    frontier.push_back(label_source.second);
    visited[label_source.second] = true;
    for (size_t i = 0; i < frontier.size(); i++) {
      const NodeID u = frontier[i];
      for (NodeID v : g.out_neigh(u)) {
        if (comp[v] != label) return false;
        if (!visited[v]) {
          visited[v] = true;
          frontier.push_back(v);
        }
      }
      if (g.directed()) {
        for (NodeID v : g.in_neigh(u)) {
          if (comp[v] != label) return false;
          if (!visited[v]) {
            visited[v] = true;
            frontier.push_back(v);
          }
        }
      }
    }
  }
  for (NodeID n = 0; n < g.num_nodes(); n++)
    if (!visited[n]) return false;
  return true;
}

}  // namespace

int main(int argc, char *argv[]) {
  PageRankCLI cli("connected-components-afforest", 1e-4, 20, false);
  if (!cli.Parse(argc, argv)) return -1;
  HostGraph g = AcquireGraph(cli.source(), &g_engine);
  auto CCBound = [](const HostGraph &graph) { return Afforest(graph); };
  BenchmarkKernel<std::vector<NodeID>>(cli, g, CCBound, PrintCompStats, CCVerifier);
  pr_gpu_destroy(g_engine);
  return 0;
}
