// noalloc.cu -- pr_gpu_run_noalloc: PageRankPull on a caller-owned device CSR
// without allocating any device memory.
//
// Who needs this: callers that cannot call cudaMalloc -- for example a host
// application whose GPU memory is entirely reserved up front by its own pool
// allocator, or a service that must not pay the implicit device-wide
// synchronisation cudaMalloc / cudaFree can cause in the middle of serving.
// They pass device buffers they already own (the CSR in, the scores out) and
// this entry point uses only a fixed scratch area that lives in this file as
// a static __device__ array.  The CUDA runtime loads this file's device code
// and that array onto a GPU lazily, at the first call on that GPU (the
// cudaGetSymbolAddress in ScratchFor): that one load reserves about 8.4 MB of
// device memory plus the module's code, and the GPU keeps it until the
// process exits.  Callers whose pool allocator reserves the GPU's memory
// must therefore make their first call on each device (max_iters = 0 on any
// small graph is enough) before the pool takes its memory, and before any
// stream capture; later calls load nothing and allocate nothing.
//
// Limits: at most kNoAllocMaxVertices vertices and kNoAllocMaxIters sweeps;
// larger requests are rejected.  All calls share the one scratch array, so
// calls whose GPU work overlaps (two host threads, or two streams, on the same
// device) race on it and must be serialised by the caller.  The array keeps
// whatever the last call left in it; everything that must start at zero is
// cleared by the call itself before use.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "pr_gpu.h"

namespace prgpu {
namespace {

constexpr int64_t kNoAllocMaxVertices = PR_GPU_NOALLOC_MAX_VERTICES;
constexpr int kNoAllocMaxIters = PR_GPU_NOALLOC_MAX_ITERS;
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 1024;

// Scratch layout (byte offsets into the static array, each 256-byte aligned).
constexpr size_t Align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffContrib0 = 0;
constexpr size_t kOffContrib1 = Align256(kOffContrib0 + sizeof(float) * kNoAllocMaxVertices);
constexpr size_t kOffPartial = Align256(kOffContrib1 + sizeof(float) * kNoAllocMaxVertices);
constexpr size_t kOffTrace = Align256(kOffPartial + sizeof(double) * kNoAllocMaxBlocks);
constexpr size_t kOffCtl = Align256(kOffTrace + sizeof(double) * kNoAllocMaxIters);
constexpr size_t kScratchBytes = Align256(kOffCtl + 256);

struct NoAllocCtl {
  unsigned ticket;  // blocks of the current sweep that have finished
  int done;         // set once the L1 change of a sweep is below epsilon
  int sweeps;       // sweeps completed
  unsigned bad;     // input validation flags
};

// The scratch area.  In host code this name is a host-side stand-in, not a
// device address: the host takes the device address with
// cudaGetSymbolAddress (once per device) and passes it to the kernels.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct View {
  float *c0, *c1;
  double *partial;
  double *trace;
  NoAllocCtl *ctl;
};

__host__ __device__ inline View MakeView(unsigned char *base) {
  View v;
  v.c0 = reinterpret_cast<float *>(base + kOffContrib0);
  v.c1 = reinterpret_cast<float *>(base + kOffContrib1);
  v.partial = reinterpret_cast<double *>(base + kOffPartial);
  v.trace = reinterpret_cast<double *>(base + kOffTrace);
  v.ctl = reinterpret_cast<NoAllocCtl *>(base + kOffCtl);
  return v;
}

// Checks the caller's CSR: offsets from 0 to m, monotone; ids in [0, n);
// out-degrees non-negative.  Problems are flagged in the control block,
// which noalloc_clear_kernel zeroed just before.
__global__ void noalloc_validate_kernel(unsigned char *scratch, int64_t n, int64_t m,
                                        const int32_t *in_off, const int32_t *in_nbr,
                                        const int32_t *out_deg) {
  View s = MakeView(scratch);
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  unsigned bad = 0;
  for (int64_t i = i0; i <= n; i += stride) {
    const int32_t o = in_off[i];
    if (i == 0 && o != 0) bad |= 1u;
    if (i == n && o != m) bad |= 2u;
    if (i < n && o > in_off[i + 1]) bad |= 4u;
    if (i < n && out_deg && out_deg[i] < 0) bad |= 16u;
  }
  for (int64_t e = i0; e < m; e += stride) {
    const int32_t v = in_nbr[e];
    if (v < 0 || v >= n) bad |= 8u;
  }
  if (bad) atomicOr(&s.ctl->bad, bad);
}

__global__ void noalloc_clear_kernel(unsigned char *scratch, int max_iters) {
  View s = MakeView(scratch);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    s.ctl->ticket = 0;
    s.ctl->done = 0;
    s.ctl->sweeps = 0;
    s.ctl->bad = 0;
  }
  for (int i = t; i < max_iters; i += gridDim.x * blockDim.x) s.trace[i] = 0.0;
}

__device__ __forceinline__ float noalloc_degree(const int32_t *in_off, const int32_t *out_deg,
                                                int u) {
  return __int2float_rn(out_deg ? out_deg[u] : in_off[u + 1] - in_off[u]);
}

// score = 1/N, contrib = score / out_degree (src/pr_spmv.cc:37-45).
__global__ void noalloc_init_kernel(unsigned char *scratch, int32_t n, const int32_t *in_off,
                                    const int32_t *out_deg, float init, float *score) {
  View s = MakeView(scratch);
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  score[u] = init;
  s.c0[u] = __fdiv_rn(init, noalloc_degree(in_off, out_deg, u));
}

// One sweep, one warp per row (grid-stride), contribution sums in float,
// new = base + d * sum, |new - old| summed in FP64 per block; the last block
// (ticket) adds the block sums in block order and decides convergence.
__global__ void __launch_bounds__(kNoAllocThreads)
noalloc_sweep_kernel(unsigned char *scratch, int32_t n, const int32_t *__restrict__ in_off,
                     const int32_t *__restrict__ in_nbr, const int32_t *__restrict__ out_deg,
                     float base, float damping, float *score, int iter, double epsilon) {
  View s = MakeView(scratch);
  if (*reinterpret_cast<volatile int *>(&s.ctl->done)) return;
  const float *cin = (iter & 1) ? s.c1 : s.c0;
  float *cout = (iter & 1) ? s.c0 : s.c1;
  __shared__ double sred[kNoAllocThreads / 32];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (kNoAllocThreads / 32);
  double err = 0.0;  // each |new - old| added in FP64, as src/pr_spmv.cc:53 does
  for (int u = blockIdx.x * (kNoAllocThreads / 32) + (threadIdx.x >> 5); u < n; u += warps) {
    const int rs = in_off[u], re = in_off[u + 1];
    float acc = 0.f;
    for (int e = rs + lane; e < re; e += 32) acc = __fadd_rn(acc, cin[in_nbr[e]]);
    acc = warp_sum_f(acc);
    if (lane == 0) {
      const float old = score[u];
      const float nw = __fadd_rn(base, __fmul_rn(damping, acc));
      score[u] = nw;
      cout[u] = __fdiv_rn(nw, noalloc_degree(in_off, out_deg, u));
      err += static_cast<double>(fabsf(__fsub_rn(nw, old)));
    }
  }
  const double block_err = block_sum_d<kNoAllocThreads>(err, sred);
  if (threadIdx.x == 0) {
    s.partial[blockIdx.x] = block_err;
    __threadfence();
    const unsigned t = atomicAdd(&s.ctl->ticket, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v = 0;
  for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += blockDim.x)
    v += __ldcg(s.partial + i);
  const double total = block_sum_d<kNoAllocThreads>(v, sred);
  if (threadIdx.x == 0) {
    s.trace[iter] = total;
    s.ctl->sweeps = iter + 1;
    s.ctl->ticket = 0;
    if (total < epsilon) s.ctl->done = 1;
    __threadfence();
  }
}

// Device address of the scratch array, taken once per device by the first
// call on that device (with that device current); taking it loads the
// module onto that device.  The address is cached per device index, so it
// belongs to the device's primary context (the one the runtime API uses);
// a caller that switches the device to another driver-API context gets the
// primary context's array.  That first call should be made before any stream
// capture begins.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_ptr[kMaxDevices] = {};

cudaError_t ScratchFor(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = p;
  }
  *out = static_cast<unsigned char *>(g_scratch_ptr[device]);
  return cudaSuccess;
}

int Fail(char *err_msg, size_t err_len, int code, const char *text) {
  if (err_msg && err_len) std::snprintf(err_msg, err_len, "%s", text);
  return code;
}

}  // namespace
}  // namespace prgpu

extern "C" int pr_gpu_run_noalloc(int device, int64_t n, int64_t m, const int32_t *in_off_dev,
                                  const int32_t *in_nbr_dev, const int32_t *out_deg_dev,
                                  int max_iters, double epsilon, float damping,
                                  float *scores_out_dev, int32_t *sweeps_out, double *err_trace,
                                  void *stream, char *err_msg, size_t err_len) {
  using namespace prgpu;
  if (err_msg && err_len) err_msg[0] = '\0';
  if (device < 0 || device >= kMaxDevices)
    return Fail(err_msg, err_len, PR_GPU_EINVAL, "device index out of range");
  if (n < 1 || m < 0)
    return Fail(err_msg, err_len, PR_GPU_EINVAL, "need n >= 1 and m >= 0");
  if (n > kNoAllocMaxVertices)
    return Fail(err_msg, err_len, PR_GPU_ERANGE,
                "pr_gpu_run_noalloc: n exceeds PR_GPU_NOALLOC_MAX_VERTICES (its fixed scratch "
                "holds at most that many vertices); use pr_gpu_upload + pr_gpu_run");
  if (m > 0x7fffffffLL)
    return Fail(err_msg, err_len, PR_GPU_ERANGE, "m exceeds int32 offsets");
  if (max_iters < 0 || max_iters > kNoAllocMaxIters)
    return Fail(err_msg, err_len, PR_GPU_ERANGE,
                "pr_gpu_run_noalloc: max_iters must be in [0, PR_GPU_NOALLOC_MAX_ITERS]");
  if (!in_off_dev || (m > 0 && !in_nbr_dev) || !scores_out_dev)
    return Fail(err_msg, err_len, PR_GPU_EINVAL, "null device buffer");
  cudaError_t e = cudaSetDevice(device);
  unsigned char *scratch = nullptr;
  if (e == cudaSuccess) e = ScratchFor(device, &scratch);
  if (e != cudaSuccess) return Fail(err_msg, err_len, PR_GPU_ECUDA, cudaGetErrorString(e));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int T = kNoAllocThreads;
  const int n32 = static_cast<int>(n);
  noalloc_clear_kernel<<<4, T, 0, s>>>(scratch, max_iters);
  noalloc_validate_kernel<<<kNoAllocMaxBlocks, T, 0, s>>>(scratch, n, m, in_off_dev, in_nbr_dev,
                                                          out_deg_dev);
  NoAllocCtl ctl;
  View host_view = MakeView(scratch);
  e = cudaMemcpyAsync(&ctl, host_view.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return Fail(err_msg, err_len, PR_GPU_ECUDA, cudaGetErrorString(e));
  if (ctl.bad)
    return Fail(err_msg, err_len, PR_GPU_EGRAPH,
                "invalid CSR (offsets not 0..m and monotone, or an id outside [0, n))");
  const float n_f = static_cast<float>(n);
  const float init = 1.0f / n_f;                  // src/pr_spmv.cc:37
  const float base = (1.0f - damping) / n_f;      // src/pr_spmv.cc:38
  noalloc_init_kernel<<<(n32 + T - 1) / T, T, 0, s>>>(scratch, n32, in_off_dev, out_deg_dev, init,
                                                      scores_out_dev);
  const int blocks = static_cast<int>(std::min<int64_t>((n + 7) / 8, kNoAllocMaxBlocks));
  for (int it = 0; it < max_iters; it++)
    noalloc_sweep_kernel<<<blocks, T, 0, s>>>(scratch, n32, in_off_dev, in_nbr_dev, out_deg_dev,
                                              base, damping, scores_out_dev, it, epsilon);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&ctl, host_view.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && err_trace && max_iters > 0)
    e = cudaMemcpyAsync(err_trace, host_view.trace, sizeof(double) * max_iters,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return Fail(err_msg, err_len, PR_GPU_ECUDA, cudaGetErrorString(e));
  if (sweeps_out) *sweeps_out = max_iters ? ctl.sweeps : 0;
  return PR_GPU_OK;
}
