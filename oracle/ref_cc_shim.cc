// ref_cc_shim.cc -- TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own Afforest connected components (src/cc.cc
// :89-150) and its graph Builder through a C ABI, for golden fixtures and the
// CPU baseline.  Compiled by oracle/Makefile against the reference sources
// where they lie; the result goes to oracle/_ref/ only and is never linked
// into the product.

#include <chrono>
#include <cstring>

#define main gapbs_reference_cc_main
#include "cc.cc"
#undef main

extern "C" {

// Builds the graph for argv (e.g. {"cc", "-g", "10"}) as the reference's cc
// binary does, runs Afforest once, and copies the labels into comp_out when
// it holds at least num_nodes entries.  Returns num_nodes (or -1 when the
// arguments do not parse); *seconds receives the kernel's wall time.
int64_t ref_cc_afforest(int argc, char **argv, int32_t *comp_out, int64_t cap,
                        double *seconds) {
  CLApp cli(argc, argv, "connected-components-afforest");
  optind = 1;  // getopt state is process-global
  if (!cli.ParseArgs()) return -1;
  Builder b(cli);
  Graph g = b.MakeGraph();
  auto t0 = std::chrono::steady_clock::now();
  pvector<NodeID> comp = Afforest(g);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if (comp_out && cap >= g.num_nodes())
    std::memcpy(comp_out, comp.data(), sizeof(int32_t) * g.num_nodes());
  return g.num_nodes();
}

}  // extern "C"

namespace {

void CopyOffsets(pvector<SGOffset> *dst, int64_t n, const int64_t *off) {
  for (int64_t i = 0; i <= n; i++) (*dst)[i] = off[i];
}

}  // namespace

extern "C" {

// The reference's Afforest on a CSR given by the caller (the graph the GPU
// engine sees), `trials` times; returns the fastest kernel time in seconds
// and copies the last labels into comp_out.
double ref_cc_afforest_csr(int64_t n, int directed, const int64_t *out_off,
                           const int32_t *out_nbr, const int64_t *in_off,
                           const int32_t *in_nbr, int trials, int32_t *comp_out) {
  pvector<SGOffset> offs(n + 1);
  CopyOffsets(&offs, n, out_off);
  NodeID *oneigh = new NodeID[out_off[n] > 0 ? out_off[n] : 1];
  if (out_off[n]) std::memcpy(oneigh, out_nbr, sizeof(NodeID) * out_off[n]);
  NodeID **oindex = Graph::GenIndex(offs, oneigh);
  Graph g;
  if (!directed) {
    g = Graph(n, oindex, oneigh);
  } else {
    pvector<SGOffset> ioffs(n + 1);
    CopyOffsets(&ioffs, n, in_off);
    NodeID *ineigh = new NodeID[in_off[n] > 0 ? in_off[n] : 1];
    if (in_off[n]) std::memcpy(ineigh, in_nbr, sizeof(NodeID) * in_off[n]);
    NodeID **iindex = Graph::GenIndex(ioffs, ineigh);
    g = Graph(n, oindex, oneigh, iindex, ineigh);
  }
  double best = 1e300;
  for (int t = 0; t < trials; t++) {
    auto t0 = std::chrono::steady_clock::now();
    pvector<NodeID> comp = Afforest(g);
    auto t1 = std::chrono::steady_clock::now();
    best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
    if (t == trials - 1 && comp_out) std::memcpy(comp_out, comp.data(), sizeof(int32_t) * n);
  }
  return best;
}

}  // extern "C"
