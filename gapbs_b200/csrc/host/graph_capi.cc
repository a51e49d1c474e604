// graph_capi.cc -- C ABI over the host graph builder (include/gapbs_graph.h).
#include "gapbs_graph.h"

#include <cstdio>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "benchmark.h"
#include "builder.h"
#include "command_line.h"

struct gapbs_graph {
  gapbs_b200::HostGraph g;
};

namespace {

thread_local std::string g_last_error;

int Fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code < 0 ? code : -1;
}

}  // namespace

extern "C" {

int gapbs_graph_build(gapbs_graph_t **out, const char *args, int verbose) {
  if (!out || !args) return Fail(-1, "null argument");
  *out = nullptr;
  std::vector<std::string> toks;
  toks.push_back("gapbs_graph");
  std::istringstream is(args);
  std::string t;
  while (is >> t) toks.push_back(t);
  std::vector<char *> argv;
  for (std::string &s : toks) argv.push_back(&s[0]);
  gapbs_b200::PageRankCLI cli("pagerank", 1e-4, 20);
  if (!cli.Parse(static_cast<int>(argv.size()), argv.data()))
    return Fail(-1, "No graph input specified");
  try {
    gapbs_graph *h = new gapbs_graph();
    h->g = gapbs_b200::MakeGraph(cli.source(), verbose != 0);
    std::fflush(stdout);
    *out = h;
    return 0;
  } catch (const gapbs_b200::BuildError &e) {
    return Fail(e.code(), e.what());
  } catch (const std::bad_alloc &) {
    return Fail(-12, "out of host memory while building the graph");
  }
}

int gapbs_graph_from_edges(gapbs_graph_t **out, const int32_t *u,
                           const int32_t *v, int64_t m, int symmetrize) {
  if (!out || m < 0 || (m > 0 && (!u || !v))) return Fail(-1, "invalid argument");
  *out = nullptr;
  try {
    gapbs_graph *h = new gapbs_graph();
    h->g = gapbs_b200::MakeGraphFromEdges(u, v, m, symmetrize != 0);
    *out = h;
    return 0;
  } catch (const gapbs_b200::BuildError &e) {
    return Fail(e.code(), e.what());
  } catch (const std::bad_alloc &) {
    return Fail(-12, "out of host memory while building the graph");
  }
}

int gapbs_graph_new_undirected(gapbs_graph_t **out, int64_t n, int64_t m, int64_t **off,
                               int32_t **nbr) {
  if (!out || !off || !nbr || n < 1 || m < 0) return Fail(-1, "invalid argument");
  *out = nullptr;
  try {
    gapbs_b200::Buffer<gapbs_b200::Offset> o(static_cast<size_t>(n + 1));
    gapbs_b200::Buffer<gapbs_b200::NodeID> b(static_cast<size_t>(m > 0 ? m : 1));
    *off = o.data();
    *nbr = b.data();
    gapbs_graph *h = new gapbs_graph();
    h->g = gapbs_b200::HostGraph::Undirected(n, std::move(o), std::move(b));
    *out = h;
    return 0;
  } catch (const std::bad_alloc &) {
    return Fail(-12, "out of host memory for the graph");
  }
}

int gapbs_rmat_permutation(int scale, int32_t *perm) {
  if (!perm || scale < 0 || scale > 30) return Fail(-1, "invalid argument");
  gapbs_b200::RMatPermutation(scale, perm);
  return 0;
}

int gapbs_graph_write_sg(const gapbs_graph_t *g, const char *path) {
  if (!g || !path) return Fail(-1, "null argument");
  try {
    gapbs_b200::WriteSerialized(g->g, path);
    return 0;
  } catch (const gapbs_b200::BuildError &e) {
    return Fail(e.code(), e.what());
  }
}

void gapbs_graph_free(gapbs_graph_t *g) { delete g; }

int64_t gapbs_graph_num_nodes(const gapbs_graph_t *g) { return g->g.num_nodes(); }
int64_t gapbs_graph_num_edges(const gapbs_graph_t *g) { return g->g.num_edges(); }
int64_t gapbs_graph_num_edges_directed(const gapbs_graph_t *g) {
  return g->g.num_edges_directed();
}
int gapbs_graph_directed(const gapbs_graph_t *g) { return g->g.directed() ? 1 : 0; }
const int64_t *gapbs_graph_out_offsets(const gapbs_graph_t *g) { return g->g.out_off_ptr(); }
const int32_t *gapbs_graph_out_neighbors(const gapbs_graph_t *g) { return g->g.out_nbr_ptr(); }
const int64_t *gapbs_graph_in_offsets(const gapbs_graph_t *g) { return g->g.in_off_ptr(); }
const int32_t *gapbs_graph_in_neighbors(const gapbs_graph_t *g) { return g->g.in_nbr_ptr(); }

void gapbs_graph_print_stats(const gapbs_graph_t *g) {
  g->g.PrintStats();
  std::fflush(stdout);
}

int gapbs_top_scores(const float *scores, int64_t n, int k, int32_t *ids, float *values) {
  if (!scores || n < 0 || k < 0 || (k > 0 && (!ids || !values))) return Fail(-1, "invalid argument");
  std::vector<std::pair<int32_t, float>> kv(n);
  for (int64_t i = 0; i < n; i++) kv[i] = std::make_pair(static_cast<int32_t>(i), scores[i]);
  auto top = gapbs_b200::TopK(kv, static_cast<size_t>(k));
  for (size_t i = 0; i < top.size(); i++) {
    ids[i] = top[i].second;
    values[i] = top[i].first;
  }
  return static_cast<int>(top.size());
}

const char *gapbs_graph_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"
