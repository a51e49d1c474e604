// gather_roofline.cu -- measures the random-gather ceiling that bounds a pull
// sweep (pr_gpu_measure_gather_rate in include/pr_gpu.h).
//
// A pull sweep issues one 4-byte load per edge at an unpredictable address.
// Each such load that misses L1 costs one 32-byte sector request on the
// SM-to-L2 path, whatever the HBM bandwidth; this kernel issues only such
// loads (hashed addresses masked into an array of the requested size, eight
// independent loads in flight per thread) and reports how many complete per
// second.  With an array far larger than L1 nearly every load misses L1; with
// one that fits in L2 the result is the gather roofline of the sweep kernels.
//
// pr_gpu_measure_row_gather_rate does the same for whole rows of row_bytes
// (a batched sweep gathers one row of its contrib tile per edge): groups of
// row_bytes / 16 lanes read a hashed row with 16-byte loads, four rows in
// flight per lane.
#include <cuda_runtime.h>

#include <cstdint>

#include "pr_gpu.h"

namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

__global__ void gather_probe_kernel(const float *__restrict__ a, uint32_t mask, int iters,
                                    float *out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  float acc = 0.f;
  uint32_t h = mix32(tid * 0x9E3779B9u + 1u);
  for (int k = 0; k < iters; k++) {
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      h = mix32(h + q + 1);
      const float *p = a + (h & mask);
      asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v[q]) : "l"(p));
    }
#pragma unroll
    for (int q = 0; q < 8; q++) acc += v[q];
  }
  out[tid] = acc;
}

// rows of 16 * L bytes, L lanes per row
__global__ void row_gather_probe_kernel(const float4 *__restrict__ a, uint32_t row_mask, int L,
                                        int iters, float *out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int gl = lane % L, grp = lane / L;
  uint32_t h = mix32((tid >> 5) * 0x9E3779B9u + 11u + grp * 7919u);
  float acc = 0.f;
  for (int k = 0; k < iters; k++) {
    float4 v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      h = mix32(h + q + 1);
      const float4 *p = a + static_cast<size_t>(h & row_mask) * L + gl;
      asm volatile("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];"
                   : "=f"(v[q].x), "=f"(v[q].y), "=f"(v[q].z), "=f"(v[q].w)
                   : "l"(p));
    }
#pragma unroll
    for (int q = 0; q < 4; q++) acc += v[q].x + v[q].y + v[q].z + v[q].w;
  }
  out[tid] = acc;
}

}  // namespace

extern "C" int pr_gpu_measure_row_gather_rate(int device, int64_t array_bytes, int row_bytes,
                                              double *bytes_per_s) {
  if (!bytes_per_s || array_bytes < 4096 || row_bytes < 16 || row_bytes > 512 ||
      (row_bytes & (row_bytes - 1)) != 0)
    return PR_GPU_EINVAL;
  int64_t rows = 1;
  while (rows * 2 * row_bytes <= array_bytes) rows *= 2;  // power of two rows
  if (cudaSetDevice(device) != cudaSuccess) return PR_GPU_ECUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return PR_GPU_ECUDA;
  const int threads = 256, blocks = sms * 8, iters = 64, L = row_bytes / 16;
  float4 *a = nullptr;
  float *out = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = PR_GPU_OK;
  if (cudaMalloc(&a, rows * row_bytes) != cudaSuccess ||
      cudaMalloc(&out, sizeof(float) * blocks * threads) != cudaSuccess) {
    rc = PR_GPU_ENOMEM;
  } else if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
             cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
             cudaMemsetAsync(a, 0, rows * row_bytes, s) != cudaSuccess) {
    rc = PR_GPU_ECUDA;
  } else {
    const uint32_t mask = static_cast<uint32_t>(rows - 1);
    row_gather_probe_kernel<<<blocks, threads, 0, s>>>(a, mask, L, iters, out);  // warm-up
    const int reps = 5;
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; r++)
      row_gather_probe_kernel<<<blocks, threads, 0, s>>>(a, mask, L, iters, out);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      rc = PR_GPU_ECUDA;
    } else {
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      const double row_loads = static_cast<double>(reps) * blocks * threads / L * 4 * iters;
      *bytes_per_s = row_loads * row_bytes / (ms / 1e3);
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (a) cudaFree(a);
  if (out) cudaFree(out);
  return rc;
}

extern "C" int pr_gpu_measure_gather_rate(int device, int64_t array_bytes, double *gathers_per_s) {
  if (!gathers_per_s || array_bytes < 4096) return PR_GPU_EINVAL;
  int64_t floats = 1;
  while (floats * 2 * 4 <= array_bytes) floats *= 2;  // power of two <= array_bytes
  if (cudaSetDevice(device) != cudaSuccess) return PR_GPU_ECUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return PR_GPU_ECUDA;
  const int threads = 256, blocks = sms * 8, iters = 64;
  float *a = nullptr, *out = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = PR_GPU_OK;
  if (cudaMalloc(&a, floats * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&out, sizeof(float) * blocks * threads) != cudaSuccess) {
    rc = PR_GPU_ENOMEM;
  } else if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
             cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
             cudaMemsetAsync(a, 0, floats * sizeof(float), s) != cudaSuccess) {
    rc = PR_GPU_ECUDA;
  } else {
    const uint32_t mask = static_cast<uint32_t>(floats - 1);
    gather_probe_kernel<<<blocks, threads, 0, s>>>(a, mask, iters, out);  // warm-up
    const int reps = 5;
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; r++) gather_probe_kernel<<<blocks, threads, 0, s>>>(a, mask, iters, out);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      rc = PR_GPU_ECUDA;
    } else {
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      const double loads = static_cast<double>(reps) * blocks * threads * iters * 8;
      *gathers_per_s = loads / (ms / 1e3);
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (a) cudaFree(a);
  if (out) cudaFree(out);
  return rc;
}
