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
