// graph.h -- host CSR graph container behind the pr_gpu CLI and the graph C ABI.
//
// Same observable interface as the reference's CSRGraph<int32_t>
// (src/graph.h:98-273): num_nodes, num_edges (undirected edges are counted
// once), num_edges_directed, out_degree/in_degree, out_neigh/in_neigh
// ranges, directed(), PrintStats() with the identical stdout line.
// Storage differs: the reference keeps an array of N+1 neighbour POINTERS per
// direction; this keeps N+1 int64 OFFSETS (the .sg on-disk form,
// src/writer.h:39-69), which is what the device upload needs.  An undirected
// graph stores one CSR and serves it for both directions, as the reference
// does (src/graph.h:138-143).
#ifndef GAPBS_B200_HOST_GRAPH_H_
#define GAPBS_B200_HOST_GRAPH_H_

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <new>
#include <utility>

namespace gapbs_b200 {

// Uninitialised, move-only heap array (large arrays are filled in parallel by
// their producers, so value-initialising them first would only cost time).
template <typename T>
class Buffer {
 public:
  Buffer() : p_(nullptr), n_(0) {}
  explicit Buffer(size_t n) : p_(n ? new T[n] : nullptr), n_(n) {}
  Buffer(Buffer &&o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  Buffer &operator=(Buffer &&o) noexcept {
    if (this != &o) { delete[] p_; p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
    return *this;
  }
  Buffer(const Buffer &) = delete;
  Buffer &operator=(const Buffer &) = delete;
  ~Buffer() { delete[] p_; }
  T *data() { return p_; }
  const T *data() const { return p_; }
  size_t size() const { return n_; }
  T &operator[](size_t i) { return p_[i]; }
  const T &operator[](size_t i) const { return p_[i]; }
  void reset() { delete[] p_; p_ = nullptr; n_ = 0; }

 private:
  T *p_;
  size_t n_;
};

typedef int32_t NodeID;
typedef int64_t Offset;

class HostGraph {
 public:
  class Range {
   public:
    Range(const NodeID *b, const NodeID *e) : b_(b), e_(e) {}
    const NodeID *begin() const { return b_; }
    const NodeID *end() const { return e_; }
   private:
    const NodeID *b_, *e_;
  };

  HostGraph() : directed_(false), n_(0) {}
  HostGraph(HostGraph &&) = default;
  HostGraph &operator=(HostGraph &&) = default;

  // Undirected: one CSR serves both directions.
  static HostGraph Undirected(int64_t n, Buffer<Offset> off, Buffer<NodeID> nbr) {
    HostGraph g;
    g.directed_ = false;
    g.n_ = n;
    g.out_off_ = std::move(off);
    g.out_nbr_ = std::move(nbr);
    return g;
  }
  static HostGraph Directed(int64_t n, Buffer<Offset> out_off, Buffer<NodeID> out_nbr,
                            Buffer<Offset> in_off, Buffer<NodeID> in_nbr) {
    HostGraph g;
    g.directed_ = true;
    g.n_ = n;
    g.out_off_ = std::move(out_off);
    g.out_nbr_ = std::move(out_nbr);
    g.in_off_ = std::move(in_off);
    g.in_nbr_ = std::move(in_nbr);
    return g;
  }

  bool directed() const { return directed_; }
  int64_t num_nodes() const { return n_; }
  // Entries in the out-CSR.
  int64_t out_entries() const { return n_ ? out_off_[n_] : 0; }
  // Same convention as the reference: an undirected graph reports half its
  // CSR entries (src/graph.h:131-136,197-203).
  int64_t num_edges() const { return directed_ ? out_entries() : out_entries() / 2; }
  int64_t num_edges_directed() const { return directed_ ? num_edges() : 2 * num_edges(); }

  int64_t out_degree(NodeID v) const { return out_off_[v + 1] - out_off_[v]; }
  int64_t in_degree(NodeID v) const {
    const Offset *o = in_off_ptr();
    return o[v + 1] - o[v];
  }
  Range out_neigh(NodeID v) const {
    return Range(out_nbr_.data() + out_off_[v], out_nbr_.data() + out_off_[v + 1]);
  }
  Range in_neigh(NodeID v) const {
    const Offset *o = in_off_ptr();
    const NodeID *nb = in_nbr_ptr();
    return Range(nb + o[v], nb + o[v + 1]);
  }

  const Offset *out_off_ptr() const { return out_off_.data(); }
  const NodeID *out_nbr_ptr() const { return out_nbr_.data(); }
  const Offset *in_off_ptr() const { return directed_ ? in_off_.data() : out_off_.data(); }
  const NodeID *in_nbr_ptr() const { return directed_ ? in_nbr_.data() : out_nbr_.data(); }

  // Identical text to src/graph.h:223-230.
  void PrintStats() const {
    std::cout << "Graph has " << n_ << " nodes and " << num_edges() << " ";
    if (!directed_) std::cout << "un";
    std::cout << "directed edges for degree: ";
    std::cout << (n_ ? num_edges() / n_ : 0) << std::endl;
  }

 private:
  bool directed_;
  int64_t n_;
  Buffer<Offset> out_off_;
  Buffer<NodeID> out_nbr_;
  Buffer<Offset> in_off_;
  Buffer<NodeID> in_nbr_;
};

}  // namespace gapbs_b200

#endif  // GAPBS_B200_HOST_GRAPH_H_
