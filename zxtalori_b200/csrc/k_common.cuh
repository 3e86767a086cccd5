// Small device utilities shared by the kernel files: warp reductions, ordered float bits,
// last-block-done tickets and a device-wide exclusive scan.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "qvm_device.cuh"

namespace zo {

__device__ __forceinline__ float warp_min(float v) {
  for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Float bits that order like the values (shaders/shell.wgsl:17) and back (src/near.zig:198).
__device__ __forceinline__ unsigned int ordered_bits(float x) {
  const unsigned int b = __float_as_uint(x);
  return (b >> 31) ? ~b : (b ^ 0x80000000u);
}
__device__ __forceinline__ float unordered_bits(unsigned int k) {
  return __uint_as_float((k & 0x80000000u) ? (k ^ 0x80000000u) : ~k);
}

// Returns true in exactly one thread of the last block to arrive (after a fence), which may
// then read every block's published partials. Resets the counter for the next launch.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int total = gridDim.x * gridDim.y;
    const unsigned int got = atomicAdd(ticket, 1u);
    is_last = (got == total - 1);
    if (is_last) *ticket = 0;
  }
  __syncthreads();
  return is_last;
}

// Stereographic chart position of a unit quaternion near the identity (src/near.zig:3-11).
__device__ __forceinline__ float3 chart(float4 q) {
  const float s = 1.0f / (1.0f + q.x);
  return make_float3(q.y * s, q.z * s, q.w * s);
}
__device__ __forceinline__ float3 chart(double4 q) {
  const double s = 1.0 / (1.0 + q.x);
  return make_float3((float)(q.y * s), (float)(q.z * s), (float)(q.w * s));
}

}  // namespace zo
