// builder.cc -- host graph construction (see builder.h for the contract).
#include "builder.h"

#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <limits>
#include <random>
#include <sstream>
#include <vector>

#include "util.h"

namespace gapbs_b200 {

namespace {

// Edges are generated in blocks of 2^18, each block with its own reseeded
// generator, so that the stream is independent of the thread count
// (src/generator.h:112-113,130-131,193).
const int64_t kGenBlock = 1 << 18;

// C++ leaves the evaluation order of the two draws in the reference's
// Edge(udist(), udist()) unspecified.  It does not matter for the graphs it
// produces: -u graphs are always symmetrised, and (a, b) and (b, a) then
// yield the same rows.
const bool kUniformDrawsDestinationFirst = true;

struct EdgeList {
  Buffer<NodeID> u, v;
  int64_t m = 0;
  EdgeList() {}
  explicit EdgeList(int64_t count) : u(count), v(count), m(count) {}
};

// Exclusive prefix sum counts[0..n) -> off[0..n]; off[n] = total.
void ExclusiveScan(const int64_t *counts, int64_t n, Offset *off) {
  int nt = omp_get_max_threads();
  std::vector<int64_t> part(nt + 1, 0);
  int team = 1;
  #pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    int T = omp_get_num_threads();
    #pragma omp single
    team = T;
    int64_t lo = n * t / T, hi = n * (t + 1) / T;
    int64_t s = 0;
    for (int64_t i = lo; i < hi; i++) s += counts[i];
    part[t + 1] = s;
    #pragma omp barrier
    #pragma omp single
    {
      for (int i = 1; i <= T; i++) part[i] += part[i - 1];
    }
    int64_t run = part[t];
    for (int64_t i = lo; i < hi; i++) {
      off[i] = run;
      run += counts[i];
    }
  }
  off[n] = part[team];
}

// Rows keyed by key[e] holding val[e] (and, when both_dirs, rows keyed by
// val[e] holding key[e]); every row then sorted, de-duplicated and stripped
// of its self-loop, which is the squished form (src/builder.h:141-170).
void AssembleRows(int64_t n, const EdgeList &el, bool transpose, bool both_dirs,
                  Buffer<Offset> *off_out, Buffer<NodeID> *nbr_out) {
  const NodeID *key = transpose ? el.v.data() : el.u.data();
  const NodeID *val = transpose ? el.u.data() : el.v.data();
  const int64_t m = el.m;
  Buffer<int64_t> cnt(n);
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) cnt[i] = 0;
  #pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; e++) {
    __atomic_fetch_add(&cnt[key[e]], 1, __ATOMIC_RELAXED);
    if (both_dirs) __atomic_fetch_add(&cnt[val[e]], 1, __ATOMIC_RELAXED);
  }
  Buffer<Offset> raw(n + 1);
  ExclusiveScan(cnt.data(), n, raw.data());
  Buffer<NodeID> tmp(raw[n] > 0 ? raw[n] : 1);
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) cnt[i] = raw[i];
  #pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; e++) {
    int64_t p = __atomic_fetch_add(&cnt[key[e]], 1, __ATOMIC_RELAXED);
    tmp[p] = val[e];
    if (both_dirs) {
      int64_t q = __atomic_fetch_add(&cnt[val[e]], 1, __ATOMIC_RELAXED);
      tmp[q] = key[e];
    }
  }
  #pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t r = 0; r < n; r++) {
    NodeID *b = tmp.data() + raw[r], *e = tmp.data() + raw[r + 1];
    std::sort(b, e);
    NodeID *ue = std::unique(b, e);
    ue = std::remove(b, ue, static_cast<NodeID>(r));
    cnt[r] = ue - b;
  }
  Buffer<Offset> off(n + 1);
  ExclusiveScan(cnt.data(), n, off.data());
  Buffer<NodeID> nbr(off[n] > 0 ? off[n] : 1);
  #pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t r = 0; r < n; r++)
    std::copy(tmp.data() + raw[r], tmp.data() + raw[r] + cnt[r], nbr.data() + off[r]);
  *off_out = std::move(off);
  *nbr_out = std::move(nbr);
}

int64_t MaxNodeIdPlusOne(const EdgeList &el) {
  NodeID max_seen = 0;
  bool negative = false;
  #pragma omp parallel for reduction(max : max_seen) reduction(|| : negative)
  for (int64_t e = 0; e < el.m; e++) {
    max_seen = std::max(max_seen, std::max(el.u[e], el.v[e]));
    negative = negative || el.u[e] < 0 || el.v[e] < 0;
  }
  if (negative) throw BuildError(-40, "Edge list holds a negative vertex id");
  return static_cast<int64_t>(max_seen) + 1;
}

HostGraph BuildFromEdgeList(EdgeList &el, bool symmetrize) {
  const int64_t n = MaxNodeIdPlusOne(el);
  Buffer<Offset> out_off, in_off;
  Buffer<NodeID> out_nbr, in_nbr;
  if (symmetrize) {
    AssembleRows(n, el, false, true, &out_off, &out_nbr);
    el = EdgeList();
    return HostGraph::Undirected(n, std::move(out_off), std::move(out_nbr));
  }
  AssembleRows(n, el, false, false, &out_off, &out_nbr);
  AssembleRows(n, el, true, false, &in_off, &in_nbr);
  el = EdgeList();
  return HostGraph::Directed(n, std::move(out_off), std::move(out_nbr),
                             std::move(in_off), std::move(in_nbr));
}

// ---- synthetic generators -------------------------------------------------

void CheckScale(int scale, int degree) {
  if (scale < 0 || scale > 62) throw BuildError(-31, "Invalid scale");
  int64_t n = int64_t(1) << scale;
  if (n > std::numeric_limits<NodeID>::max()) {
    std::ostringstream os;
    os << "NodeID type (max: " << std::numeric_limits<NodeID>::max()
       << ") too small to hold " << n << std::endl
       << "Recommend changing NodeID (typedef'd in src/benchmark.h)"
       << " to a wider type and recompiling";
    throw BuildError(-31, os.str());
  }
  if (degree < 0) throw BuildError(-31, "Invalid degree");
}

// Uniform draws in [0, n-1]: a raw 32-bit draw, redrawn while it falls in the
// biased tail, then reduced modulo n (src/generator.h:33-64).
struct BoundedDraw {
  uint32_t mod;
  uint32_t cutoff;
  bool identity;
  explicit BoundedDraw(uint32_t max_value) {
    const uint32_t top = 0xFFFFFFFFu;
    identity = (top == max_value);
    mod = max_value + 1u;
    uint32_t rem = identity ? 0 : top % mod;
    cutoff = (identity || rem == mod - 1) ? 0 : top - rem;
  }
  NodeID operator()(std::mt19937 &rng) const {
    uint32_t r = static_cast<uint32_t>(rng());
    if (identity) return static_cast<NodeID>(r);
    if (cutoff != 0)
      while (r >= cutoff) r = static_cast<uint32_t>(rng());
    return static_cast<NodeID>(r % mod);
  }
};

EdgeList GenerateUniform(int scale, int degree) {
  const int64_t n = int64_t(1) << scale;
  const int64_t m = n * degree;
  EdgeList el(m);
  const BoundedDraw draw(static_cast<uint32_t>(n - 1));
  const int64_t nblocks = (m + kGenBlock - 1) / kGenBlock;
  #pragma omp parallel for schedule(dynamic, 1)
  for (int64_t b = 0; b < nblocks; b++) {
    std::mt19937 rng(static_cast<uint32_t>(kRandSeed + b));
    const int64_t lo = b * kGenBlock, hi = std::min(lo + kGenBlock, m);
    for (int64_t e = lo; e < hi; e++) {
      NodeID first = draw(rng);
      NodeID second = draw(rng);
      if (kUniformDrawsDestinationFirst) {
        el.u[e] = second;
        el.v[e] = first;
      } else {
        el.u[e] = first;
        el.v[e] = second;
      }
    }
  }
  return el;
}

// R-MAT recursive quadrant descent, one 32-bit draw per level: below A -> top
// left, below A+B -> top right, below A+B+C -> bottom left, else bottom
// right (src/generator.h:122-155; boundary draws equal to A or A+B+C stay on
// the lower side, as there).
EdgeList GenerateRMat(int scale, int degree) {
  const int64_t n = int64_t(1) << scale;
  const int64_t m = n * degree;
  EdgeList el(m);
  const uint32_t top = std::numeric_limits<uint32_t>::max();
  const uint32_t A = static_cast<uint32_t>(0.57 * top);
  const uint32_t B = static_cast<uint32_t>(0.19 * top);
  const uint32_t C = static_cast<uint32_t>(0.19 * top);
  const uint32_t AB = A + B, ABC = A + B + C;
  const int64_t nblocks = (m + kGenBlock - 1) / kGenBlock;
  #pragma omp parallel for schedule(dynamic, 1)
  for (int64_t b = 0; b < nblocks; b++) {
    std::mt19937 rng(static_cast<uint32_t>(kRandSeed + b));
    const int64_t lo = b * kGenBlock, hi = std::min(lo + kGenBlock, m);
    for (int64_t e = lo; e < hi; e++) {
      uint32_t s = 0, d = 0;
      for (int level = 0; level < scale; level++) {
        uint32_t r = static_cast<uint32_t>(rng());
        s <<= 1;
        d <<= 1;
        if (r < AB) {
          d += (r > A);
        } else {
          s += 1;
          d += (r > ABC);
        }
      }
      el.u[e] = static_cast<NodeID>(s);
      el.v[e] = static_cast<NodeID>(d);
    }
  }
  // Relabel through a seeded random permutation (src/generator.h:93-103).
  Buffer<NodeID> perm(n);
  RMatPermutation(scale, perm.data());
  #pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; e++) {
    el.u[e] = perm[el.u[e]];
    el.v[e] = perm[el.v[e]];
  }
  return el;
}

// ---- file readers -----------------------------------------------------------

std::string Suffix(const std::string &fn) {
  size_t p = fn.rfind('.');
  if (p == std::string::npos)
    throw BuildError(-1, "Couldn't find suffix of " + fn);
  return fn.substr(p);
}

struct EdgeVec {
  std::vector<NodeID> u, v;
  void add(NodeID a, NodeID b) { u.push_back(a); v.push_back(b); }
  EdgeList Take() {
    EdgeList el(static_cast<int64_t>(u.size()));
    std::copy(u.begin(), u.end(), el.u.data());
    std::copy(v.begin(), v.end(), el.v.data());
    return el;
  }
};

// "u v" per edge (src/reader.h:50-57).
void ParseEL(std::istream &in, EdgeVec *ev) {
  NodeID a, b;
  while (in >> a >> b) ev->add(a, b);
}

// "u v w" per edge, weight dropped (src/reader.h:59-67).
void ParseWEL(std::istream &in, EdgeVec *ev) {
  NodeID a, b;
  int32_t w;
  while (in >> a >> b >> w) ev->add(a, b);
}

// DIMACS: "a u v w" arc lines, 1-based; other lines skipped
// (src/reader.h:70-85).
void ParseGR(std::istream &in, EdgeVec *ev) {
  while (!in.eof()) {
    int c = in.peek();
    if (c == 'a') {
      char tag;
      NodeID a, b;
      int32_t w;
      in >> tag >> a >> b >> w;
      ev->add(a - 1, b - 1);
    } else {
      in.ignore(200, '\n');
    }
  }
}

// METIS: header "nodes edges [fmt]", then one 1-based adjacency line per
// vertex ("v w" pairs when fmt == 1); '%' lines are comments
// (src/reader.h:88-141).
void ParseMetis(std::istream &in, EdgeVec *ev) {
  int64_t nodes = 0, edges = 0;
  bool weighted = false;
  std::string line;
  while (true) {
    if (in.peek() == '%') {
      in.ignore(200, '\n');
      continue;
    }
    std::getline(in, line, '\n');
    std::istringstream hs(line);
    hs >> nodes >> edges;
    hs >> std::ws;
    if (!hs.eof()) {
      int32_t fmt;
      hs >> fmt;
      if (fmt == 1) {
        weighted = true;
      } else if (fmt != 0 && fmt != 100) {
        throw BuildError(-20, "Do not support METIS fmt type: " + std::to_string(fmt));
      }
    }
    break;
  }
  NodeID u = 0;
  while (u < nodes) {
    if (in.peek() == '%') {
      in.ignore(200, '\n');
      continue;
    }
    std::getline(in, line);
    if (!line.empty()) {
      std::istringstream es(line);
      if (weighted) {
        NodeID b;
        int32_t w;
        while (es >> b >> w >> std::ws) ev->add(u, b - 1);
      } else {
        NodeID b;
        while (es >> b >> std::ws) ev->add(u, b - 1);
      }
    }
    u++;
    if (!in && in.eof()) break;
  }
}

// MatrixMarket coordinate format, 1-based; "symmetric" adds the reverse of
// every entry (src/reader.h:145-218).
void ParseMTX(std::istream &in, EdgeVec *ev) {
  std::string start, object, format, field, symmetry, line;
  in >> start >> object >> format >> field >> symmetry >> std::ws;
  if (start != "%%MatrixMarket")
    throw BuildError(-21, ".mtx file did not start with %%MatrixMarket");
  if (object != "matrix" || format != "coordinate")
    throw BuildError(-22, "only allow matrix coordinate format for .mtx");
  if (field == "complex")
    throw BuildError(-23, "do not support complex weights for .mtx");
  bool weighted;
  if (field == "pattern") weighted = false;
  else if (field == "real" || field == "double" || field == "integer") weighted = true;
  else throw BuildError(-24, "unrecognized field type for .mtx");
  bool undirected;
  if (symmetry == "symmetric") undirected = true;
  else if (symmetry == "general" || symmetry == "skew-symmetric") undirected = false;
  else throw BuildError(-25, "unsupported symmetry type for .mtx");
  while (in.peek() == '%') in.ignore(200, '\n');
  int64_t rows, cols, nnz;
  in >> rows >> cols >> nnz >> std::ws;
  if (rows != cols) {
    std::ostringstream os;
    os << rows << " " << cols << " " << nnz << "\nmatrix must be square for .mtx";
    throw BuildError(-26, os.str());
  }
  (void)weighted;  // weights are dropped by the unweighted builder
  while (std::getline(in, line)) {
    if (line.empty()) continue;
    std::istringstream es(line);
    NodeID a, b;
    es >> a >> b;
    ev->add(a - 1, b - 1);
    if (undirected) ev->add(b - 1, a - 1);
  }
}

}  // namespace

void RMatPermutation(int scale, NodeID *perm) {
  const int64_t n = int64_t(1) << scale;
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) perm[i] = static_cast<NodeID>(i);
  std::mt19937 prng(static_cast<uint32_t>(kRandSeed));
  std::shuffle(perm, perm + n, prng);
}

// ---- serialized graphs (.sg) ---------------------------------------------

void WriteSerialized(const HostGraph &g, const std::string &path) {
  std::ofstream out(path, std::ios::out | std::ios::binary);
  if (!out) throw BuildError(-5, "Couldn't write to file " + path);
  bool directed = g.directed();
  int64_t n = g.num_nodes();
  int64_t entries = g.num_edges_directed();
  out.write(reinterpret_cast<const char *>(&directed), sizeof(bool));
  out.write(reinterpret_cast<const char *>(&entries), sizeof(int64_t));
  out.write(reinterpret_cast<const char *>(&n), sizeof(int64_t));
  out.write(reinterpret_cast<const char *>(g.out_off_ptr()), (n + 1) * sizeof(Offset));
  out.write(reinterpret_cast<const char *>(g.out_nbr_ptr()), entries * sizeof(NodeID));
  if (directed) {
    out.write(reinterpret_cast<const char *>(g.in_off_ptr()), (n + 1) * sizeof(Offset));
    out.write(reinterpret_cast<const char *>(g.in_nbr_ptr()), entries * sizeof(NodeID));
  }
  if (!out) throw BuildError(-5, "Couldn't write to file " + path);
}

HostGraph ReadSerialized(const std::string &path) {
  std::ifstream in(path, std::ios::in | std::ios::binary);
  if (!in.is_open()) throw BuildError(-6, "Couldn't open file " + path);
  bool directed = false;
  int64_t entries = 0, n = 0;
  in.read(reinterpret_cast<char *>(&directed), sizeof(bool));
  in.read(reinterpret_cast<char *>(&entries), sizeof(int64_t));
  in.read(reinterpret_cast<char *>(&n), sizeof(int64_t));
  if (!in || n < 0 || entries < 0)
    throw BuildError(-6, "Corrupt serialized graph " + path);
  Buffer<Offset> off(n + 1);
  Buffer<NodeID> nbr(entries > 0 ? entries : 1);
  in.read(reinterpret_cast<char *>(off.data()), (n + 1) * sizeof(Offset));
  in.read(reinterpret_cast<char *>(nbr.data()), entries * sizeof(NodeID));
  if (!directed) {
    if (!in) throw BuildError(-6, "Corrupt serialized graph " + path);
    return HostGraph::Undirected(n, std::move(off), std::move(nbr));
  }
  Buffer<Offset> ioff(n + 1);
  Buffer<NodeID> inbr(entries > 0 ? entries : 1);
  in.read(reinterpret_cast<char *>(ioff.data()), (n + 1) * sizeof(Offset));
  in.read(reinterpret_cast<char *>(inbr.data()), entries * sizeof(NodeID));
  if (!in) throw BuildError(-6, "Corrupt serialized graph " + path);
  return HostGraph::Directed(n, std::move(off), std::move(nbr), std::move(ioff),
                             std::move(inbr));
}

HostGraph MakeGraphFromEdges(const NodeID *u, const NodeID *v, int64_t m,
                             bool symmetrize) {
  EdgeList el(m);
  std::copy(u, u + m, el.u.data());
  std::copy(v, v + m, el.v.data());
  return BuildFromEdgeList(el, symmetrize);
}

HostGraph MakeGraph(const GraphSource &src, bool verbose) {
  EdgeList el;
  bool symmetrize = src.symmetrize;
  if (!src.filename.empty()) {
    std::string suffix = Suffix(src.filename);
    if (suffix == ".sg") {
      WallTimer t;
      t.Start();
      HostGraph g = ReadSerialized(src.filename);
      t.Stop();
      if (verbose) PrintTime("Read Time", t.Seconds());
      return g;
    }
    if (suffix == ".wsg")
      throw BuildError(-5, ".wsg only allowed for weighted graphs");
    WallTimer t;
    t.Start();
    std::ifstream file(src.filename);
    if (!file.is_open()) throw BuildError(-2, "Couldn't open file " + src.filename);
    EdgeVec ev;
    if (suffix == ".el") ParseEL(file, &ev);
    else if (suffix == ".wel") ParseWEL(file, &ev);
    else if (suffix == ".gr") ParseGR(file, &ev);
    else if (suffix == ".graph") ParseMetis(file, &ev);
    else if (suffix == ".mtx") ParseMTX(file, &ev);
    else throw BuildError(-3, "Unrecognized suffix: " + suffix);
    el = ev.Take();
    t.Stop();
    if (verbose) PrintTime("Read Time", t.Seconds());
  } else if (src.scale != -1) {
    CheckScale(src.scale, src.degree);
    symmetrize = true;
    WallTimer t;
    t.Start();
    el = src.uniform ? GenerateUniform(src.scale, src.degree)
                     : GenerateRMat(src.scale, src.degree);
    t.Stop();
    if (verbose) PrintTime("Generate Time", t.Seconds());
  } else {
    throw BuildError(-1, "No graph input specified. (Use -h for help)");
  }
  WallTimer t;
  t.Start();
  HostGraph g = BuildFromEdgeList(el, symmetrize);
  t.Stop();
  if (verbose) PrintTime("Build Time", t.Seconds());
  return g;
}

}  // namespace gapbs_b200
