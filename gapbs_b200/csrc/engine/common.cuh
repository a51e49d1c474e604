// common.cuh -- memory-access helpers and reductions for the sm_100a kernels.
//
// Cache policy of the sweep:
//   * neighbour-index / edge-weight / old-score streams are read once per
//     sweep: non-coherent loads that do not allocate in L1 and are marked
//     evict-first in L2, so they do not push the contrib array out of L2;
//   * contrib gathers are random: non-coherent loads, L1-allocating (hub
//     entries repeat within an SM), evict-last in L2;
//   * new scores are streamed out (evict-first); new contribs are written
//     with evict-last because the next sweep gathers them.
// The L2 priorities use per-instruction cache policies (createpolicy), which
// leave no state behind on the device.
#ifndef GAPBS_B200_ENGINE_COMMON_CUH_
#define GAPBS_B200_ENGINE_COMMON_CUH_

#include <cuda_runtime.h>
#include <cstdint>

namespace prgpu {

__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ int4 ld_stream_v4(const int4 *p, uint64_t pol) {
  int4 r;
  asm volatile(
      "ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ float4 ld_stream_v4f(const float4 *p, uint64_t pol) {
  float4 r;
  asm volatile(
      "ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
      : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
      : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ int ld_stream_s32(const int *p, uint64_t pol) {
  int r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
               : "=r"(r) : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ float ld_stream_f32(const float *p, uint64_t pol) {
  float r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(r) : "l"(p), "l"(pol));
  return r;
}

// Score arrays are read and then rewritten by the same thread within one
// sweep; the read uses the coherent path.
__device__ __forceinline__ float ld_score(const float *p, uint64_t pol) {
  float r;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(r) : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ float ld_gather(const float *p, uint64_t pol) {
  float r;
  asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(r) : "l"(p), "l"(pol));
  return r;
}

// Gather that does not allocate in L1 (cold rows must not evict the hubs).
__device__ __forceinline__ float ld_gather_cold(const float *p, uint64_t pol) {
  float r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(r) : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ float4 ld_gather_v4(const float4 *p, uint64_t pol) {
  float4 r;
  asm("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
      : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
      : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ float4 ld_gather_v4_cold(const float4 *p, uint64_t pol) {
  float4 r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
      : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
      : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ float4 ld_score_v4(const float4 *p, uint64_t pol) {
  float4 r;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
               : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
               : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ void st_hint_v4(float4 *p, float4 v, uint64_t pol) {
  asm volatile("st.global.L1::no_allocate.L2::cache_hint.v4.f32 [%0], {%1,%2,%3,%4}, %5;"
               :: "l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol) : "memory");
}

__device__ __forceinline__ void st_hint_f32(float *p, float v, uint64_t pol) {
  asm volatile("st.global.L1::no_allocate.L2::cache_hint.f32 [%0], %1, %2;"
               :: "l"(p), "f"(v), "l"(pol) : "memory");
}

// Warp-wide sums over lane groups of G consecutive lanes (fixed xor order,
// so the result is deterministic).
template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; every thread of the block must call it.  Result valid in
// thread 0.  Deterministic: fixed per-warp tree, then warps in order.
template <int THREADS>
__device__ __forceinline__ double block_sum_d(double v, double *smem) {
  constexpr int W = THREADS / 32;
  v = warp_sum_d(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < W; i++) r += smem[i];
  }
  __syncthreads();
  return r;
}

template <int THREADS>
__device__ __forceinline__ float block_sum_f(float v, float *smem) {
  constexpr int W = THREADS / 32;
  v = warp_sum_f(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  float r = 0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < W; i++) r += smem[i];
  }
  __syncthreads();
  return r;
}

}  // namespace prgpu

#endif  // GAPBS_B200_ENGINE_COMMON_CUH_
