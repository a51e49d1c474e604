/*
 * gapbs_graph.h -- C ABI of the host graph builder (libgapbs_graph.so).
 *
 * Replaces, for callers that are not C++ (the Python package, ctypes, any
 * FFI), the reference's graph construction entry point
 * BuilderBase::MakeGraph (src/builder.h:343-364) and the CSRGraph accessors
 * the PageRank kernel touches (src/graph.h:189-221, VertexOffsets :251-259).
 * The graph built for a given argument string is identical, offset for offset
 * and neighbour for neighbour, to the one the reference builds for the same
 * command line.
 *
 * All functions return 0 on success or a negative code (the reference's exit
 * code for the same condition where it has one); the message is available
 * from gapbs_graph_last_error() on the calling thread.
 */
#ifndef GAPBS_GRAPH_H_
#define GAPBS_GRAPH_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gapbs_graph gapbs_graph_t;

/* Builds from pr_spmv-style options, e.g. "-g 16", "-u 24 -k 16",
 * "-f graph.el -s", "-f graph.sg" (src/command_line.h:28-94 option
 * semantics: -g/-u force symmetrisation).  verbose != 0 prints the
 * reference's "Generate Time:" / "Read Time:" / "Build Time:" lines. */
int gapbs_graph_build(gapbs_graph_t **out, const char *args, int verbose);

/* Builds from an explicit edge list u[i] -> v[i] (N = max id + 1, rows
 * sorted, de-duplicated, self-loops removed; symmetrize != 0 adds reverse
 * edges).  Mirrors BuilderBase::MakeGraphFromEL + SquishGraph
 * (src/builder.h:317-341,172-186). */
int gapbs_graph_from_edges(gapbs_graph_t **out, const int32_t *u,
                           const int32_t *v, int64_t m, int symmetrize);

/* An undirected graph of n vertices and m CSR entries whose arrays the
 * caller fills (for example from pr_gpu_download_csr): *off receives the
 * n + 1 offsets, *nbr the m neighbours, both owned by the graph (the
 * reference's CSRGraph(num_nodes, index, neighs), src/graph.h:138-143). */
int gapbs_graph_new_undirected(gapbs_graph_t **out, int64_t n, int64_t m,
                               int64_t **off, int32_t **nbr);

/* The seeded permutation the reference relabels R-MAT graphs through
 * (src/generator.h:93-103): perm[i] for i < 2^scale (input of
 * pr_gpu_generate). */
int gapbs_rmat_permutation(int scale, int32_t *perm);

/* Writes the .sg serialized layout (src/writer.h:39-69). */
int gapbs_graph_write_sg(const gapbs_graph_t *g, const char *path);

/* ~CSRGraph (src/graph.h:165-167). */
void gapbs_graph_free(gapbs_graph_t *g);

/* CSRGraph::num_nodes / num_edges / num_edges_directed / directed
 * (src/graph.h:189-203); undirected graphs count each edge once in
 * num_edges. */
int64_t gapbs_graph_num_nodes(const gapbs_graph_t *g);
int64_t gapbs_graph_num_edges(const gapbs_graph_t *g);
int64_t gapbs_graph_num_edges_directed(const gapbs_graph_t *g);
int gapbs_graph_directed(const gapbs_graph_t *g);

/* CSR views owned by the graph (valid until gapbs_graph_free): the arrays
 * behind CSRGraph::out_neigh / in_neigh (src/graph.h:214-222) and
 * VertexOffsets (src/graph.h:251-259), offsets as int64 counts.  For an undirected graph the in-views
 * return the out-arrays. */
const int64_t *gapbs_graph_out_offsets(const gapbs_graph_t *g);
const int32_t *gapbs_graph_out_neighbors(const gapbs_graph_t *g);
const int64_t *gapbs_graph_in_offsets(const gapbs_graph_t *g);
const int32_t *gapbs_graph_in_neighbors(const gapbs_graph_t *g);

/* Prints "Graph has N nodes and M [un]directed edges for degree: D"
 * (src/graph.h:223-230). */
void gapbs_graph_print_stats(const gapbs_graph_t *g);

/* The k largest scores as (id, score), in the order and with the tie rule of
 * the reference's TopK (src/benchmark.h:72-88) as used by PrintTopScores
 * (src/pr_spmv.cc:64-73).  Returns the number written (<= k). */
int gapbs_top_scores(const float *scores, int64_t n, int k, int32_t *ids, float *values);

const char *gapbs_graph_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GAPBS_GRAPH_H_ */
