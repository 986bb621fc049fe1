// Packed FP32 arithmetic for the tree walks: two lanes' values per
// instruction on sm_100 (FFMA2 / FADD2 / FMUL2, through the float2
// intrinsics of the CUDA 12.8+ runtime headers). Each component rounds as the
// scalar round-to-nearest operation does. The scalar overloads let one
// template body serve a packed pair of target slots and a single leftover
// slot; every fused multiply-add is written out, so the two forms round the
// same way.
#pragma once

#include <cuda_runtime.h>

namespace sbh {

__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float vrsqrt(float a) { return rsqrtf(a); }
__device__ __forceinline__ float2 vrsqrt(float2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }

template <typename V>
__device__ __forceinline__ V vsplat(float s);
template <>
__device__ __forceinline__ float vsplat<float>(float s) {
  return s;
}
template <>
__device__ __forceinline__ float2 vsplat<float2>(float s) {
  return make_float2(s, s);
}

}  // namespace sbh
