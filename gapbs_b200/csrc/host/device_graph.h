// device_graph.h -- the graph of a CLI run, on the GPU and on the host.
//
// Synthetic graphs (-g / -u) are generated and built on the GPU, identical to
// the reference's (pr_gpu_generate): "Generate Time:" covers the host
// permutation and the device build, "Build Time:" the copy of the CSR to the
// host (for verifiers and analysis).  Graphs read from files are built on the
// host and uploaded once, on an "Upload Time:" line.
#ifndef GAPBS_B200_HOST_DEVICE_GRAPH_H_
#define GAPBS_B200_HOST_DEVICE_GRAPH_H_

#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "builder.h"
#include "graph.h"
#include "pr_gpu.h"
#include "util.h"

namespace gapbs_b200 {

[[noreturn]] inline void Die(int code, const std::string &msg) {
  std::cout << msg << std::endl;
  std::exit(code);
}

inline pr_gpu_t *CreateEngine() {
  pr_gpu_t *h = nullptr;
  int rc = pr_gpu_create(&h, 0);
  if (rc) Die(rc, "pr_gpu_create failed: no usable CUDA device");
  return h;
}

// One-time upload of a host graph (int32 offsets) to the engine.
inline void UploadGraph(pr_gpu_t *h, const HostGraph &g) {
  WallTimer t;
  t.Start();
  const int64_t n = g.num_nodes();
  const int64_t m = g.out_entries();
  if (m > 0x7fffffffLL - 8) Die(PR_GPU_ERANGE, "graph exceeds int32 offsets");
  std::vector<int32_t> out_off(n + 1), in_off;
  for (int64_t i = 0; i <= n; i++) out_off[i] = static_cast<int32_t>(g.out_off_ptr()[i]);
  if (g.directed()) {
    in_off.resize(n + 1);
    for (int64_t i = 0; i <= n; i++) in_off[i] = static_cast<int32_t>(g.in_off_ptr()[i]);
  }
  int rc = pr_gpu_upload(h, n, m, out_off.data(), g.out_nbr_ptr(),
                         g.directed() ? in_off.data() : nullptr,
                         g.directed() ? g.in_nbr_ptr() : nullptr, nullptr);
  if (rc) Die(rc, std::string("pr_gpu_upload failed: ") + pr_gpu_last_error(h));
  t.Stop();
  PrintTime("Upload Time", t.Seconds());
}

// -g / -u on the device.  Returns false (host path) for sizes the device
// path does not cover.
inline bool GenerateOnDevice(pr_gpu_t *h, const GraphSource &src, HostGraph *g) {
  if (src.scale < 1 || src.scale > 30 || src.degree < 0) return false;
  if ((int64_t(2) * src.degree) << src.scale > 0x7fffffffLL - 8) return false;
  WallTimer t;
  t.Start();
  std::vector<NodeID> perm;
  if (!src.uniform) {
    perm.resize(size_t(1) << src.scale);
    RMatPermutation(src.scale, perm.data());
  }
  int64_t n = 0, m = 0;
  int rc = pr_gpu_generate(h, src.uniform ? 1 : 0, src.scale, src.degree,
                           src.uniform ? nullptr : perm.data(), &n, &m);
  if (rc) Die(rc, std::string("pr_gpu_generate failed: ") + pr_gpu_last_error(h));
  t.Stop();
  PrintTime("Generate Time", t.Seconds());
  t.Start();
  Buffer<Offset> off(static_cast<size_t>(n + 1));
  Buffer<NodeID> nbr(static_cast<size_t>(m > 0 ? m : 1));
  rc = pr_gpu_download_csr(h, off.data(), nbr.data());
  if (rc) Die(rc, std::string("pr_gpu_download_csr failed: ") + pr_gpu_last_error(h));
  *g = HostGraph::Undirected(n, std::move(off), std::move(nbr));
  t.Stop();
  PrintTime("Build Time", t.Seconds());
  return true;
}

// The run's graph: on the device in *engine (created here) and on the host.
inline HostGraph AcquireGraph(const GraphSource &src, pr_gpu_t **engine) {
  HostGraph g;
  if (src.scale != -1 && src.scale >= 1 && src.scale <= 30 && src.degree >= 0 &&
      ((int64_t(2) * src.degree) << src.scale) <= 0x7fffffffLL - 8) {
    *engine = CreateEngine();
    GenerateOnDevice(*engine, src, &g);
    return g;
  }
  try {
    g = MakeGraph(src, true);
  } catch (const BuildError &e) {
    Die(e.code(), e.what());
  }
  *engine = CreateEngine();
  UploadGraph(*engine, g);
  return g;
}

}  // namespace gapbs_b200

#endif  // GAPBS_B200_HOST_DEVICE_GRAPH_H_
