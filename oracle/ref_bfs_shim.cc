// ref_bfs_shim.cc -- TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own direction-optimizing BFS (src/bfs.cc:99-174)
// and its SourcePicker (src/benchmark.h:46-68) through a C ABI, for golden
// fixtures and the CPU baseline.  Compiled by oracle/Makefile against the
// reference sources where they lie; the result goes to oracle/_ref/ only and
// is never linked into the product.

#include <chrono>
#include <cstring>

#define main gapbs_reference_bfs_main
#include "bfs.cc"
#undef main

extern "C" {

// Builds the graph for argv as the reference's bfs binary does; writes the
// first k sources its SourcePicker yields (given_source -1) into sources,
// and, when parent_out is non-null, the DOBFS parents from `source` (or from
// the first picked source when source < 0).  Returns num_nodes, or -1 when
// the arguments do not parse.
int64_t ref_bfs(int argc, char **argv, int k, int32_t *sources, int64_t source,
                int32_t *parent_out, int64_t cap, double *seconds) {
  CLApp cli(argc, argv, "breadth-first search");
  optind = 1;  // getopt state is process-global
  if (!cli.ParseArgs()) return -1;
  Builder b(cli);
  Graph g = b.MakeGraph();
  SourcePicker<Graph> sp(g, -1);
  for (int i = 0; i < k; i++) sources[i] = sp.PickNext();
  if (parent_out && cap >= g.num_nodes()) {
    NodeID src = source >= 0 ? static_cast<NodeID>(source) : sources[0];
    auto t0 = std::chrono::steady_clock::now();
    pvector<NodeID> parent = DOBFS(g, src);
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    std::memcpy(parent_out, parent.data(), sizeof(int32_t) * g.num_nodes());
  }
  return g.num_nodes();
}

}  // extern "C"

namespace {

void CopyOffsetsBfs(pvector<SGOffset> *dst, int64_t n, const int64_t *off) {
  for (int64_t i = 0; i <= n; i++) (*dst)[i] = off[i];
}

}  // namespace

extern "C" {

// The reference's DOBFS on a CSR given by the caller, from each of the
// nsrc sources in turn; returns the total kernel time in seconds and copies
// the last search's parents into parent_out.
double ref_bfs_csr(int64_t n, int directed, const int64_t *out_off, const int32_t *out_nbr,
                   const int64_t *in_off, const int32_t *in_nbr, int nsrc,
                   const int32_t *sources, int32_t *parent_out) {
  pvector<SGOffset> offs(n + 1);
  CopyOffsetsBfs(&offs, n, out_off);
  NodeID *oneigh = new NodeID[out_off[n] > 0 ? out_off[n] : 1];
  if (out_off[n]) std::memcpy(oneigh, out_nbr, sizeof(NodeID) * out_off[n]);
  NodeID **oindex = Graph::GenIndex(offs, oneigh);
  Graph g;
  if (!directed) {
    g = Graph(n, oindex, oneigh);
  } else {
    pvector<SGOffset> ioffs(n + 1);
    CopyOffsetsBfs(&ioffs, n, in_off);
    NodeID *ineigh = new NodeID[in_off[n] > 0 ? in_off[n] : 1];
    if (in_off[n]) std::memcpy(ineigh, in_nbr, sizeof(NodeID) * in_off[n]);
    NodeID **iindex = Graph::GenIndex(ioffs, ineigh);
    g = Graph(n, oindex, oneigh, iindex, ineigh);
  }
  double total = 0;
  for (int i = 0; i < nsrc; i++) {
    auto t0 = std::chrono::steady_clock::now();
    pvector<NodeID> parent = DOBFS(g, sources[i]);
    auto t1 = std::chrono::steady_clock::now();
    total += std::chrono::duration<double>(t1 - t0).count();
    if (i == nsrc - 1 && parent_out) std::memcpy(parent_out, parent.data(), sizeof(int32_t) * n);
  }
  return total;
}

}  // extern "C"
