// builder.h -- host graph construction for the pr_gpu engine.
//
// Produces the same CSR graph, bit for bit, that the GAP Benchmark Suite's
// BuilderBase::MakeGraph (src/builder.h:343-364) produces for the same
// command line, so that GPU results can be compared with the reference on
// identical inputs.  Identity requires the same edge stream:
//   -g  R-MAT, A/B/C = 0.57/0.19/0.19 of 2^32, one std::mt19937 per block of
//       2^18 edges seeded kRandSeed + block, then a std::shuffle vertex
//       permutation seeded kRandSeed (src/generator.h:93-155);
//   -u  uniform pairs from the same per-block seeding through a
//       rejection-sampled modulo (src/generator.h:33-64,105-120);
//   -f  .el .wel .gr .graph .mtx (1-based formats shifted to 0-based) and the
//       .sg serialized CSR (src/reader.h:50-307);
// then N = max id + 1 (src/builder.h:317-323), optional symmetrisation, and a
// per-vertex sort / de-duplicate / self-loop removal (src/builder.h:141-186).
// The CSR assembly itself is this file's own (count, scatter, squish in
// place), not the reference's pointer-array construction.
#ifndef GAPBS_B200_HOST_BUILDER_H_
#define GAPBS_B200_HOST_BUILDER_H_

#include <stdexcept>
#include <string>

#include "graph.h"

namespace gapbs_b200 {

// Failure with the reference's exit code for the same condition
// (e.g. -2 unreadable file, -3 unknown suffix, -31 NodeID too narrow).
class BuildError : public std::runtime_error {
 public:
  BuildError(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }
 private:
  int code_;
};

struct GraphSource {
  std::string filename;     // -f
  int scale = -1;           // -g / -u
  int degree = 16;          // -k
  bool symmetrize = false;  // -s (forced on for -g / -u, src/command_line.h:79-80)
  bool uniform = false;     // -u
  bool in_place = false;    // -m: accepted; yields the same graph
};

// Builds the graph; when verbose, prints "Generate Time:" / "Read Time:" and
// "Build Time:" lines in the reference's format.  Throws BuildError.
HostGraph MakeGraph(const GraphSource &src, bool verbose);

// Builds from an explicit edge list (u[i] -> v[i]); N = max id + 1.
HostGraph MakeGraphFromEdges(const NodeID *u, const NodeID *v, int64_t m,
                             bool symmetrize);

// The seeded vertex permutation R-MAT graphs are relabelled through
// (src/generator.h:93-103): perm[i] for i < 2^scale.
void RMatPermutation(int scale, NodeID *perm);

// Writes / reads the .sg layout of src/writer.h:39-69.
void WriteSerialized(const HostGraph &g, const std::string &path);
HostGraph ReadSerialized(const std::string &path);

}  // namespace gapbs_b200

#endif  // GAPBS_B200_HOST_BUILDER_H_
