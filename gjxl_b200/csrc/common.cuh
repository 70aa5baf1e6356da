// Shared device helpers for the gjxl B200 analysis kernels.
//
// Every translation unit is compiled with --fmad=false: a multiply followed by
// an add stays two IEEE-rounded operations, exactly like the reference's x86
// build (which has no FMA contraction). Where the reference calls std::fma,
// the kernels call fmaf explicitly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gjxl_b200.h"

namespace gjxl_b200 {

constexpr int kBlockDim = 8;

// Device error-word bits (atomicOr into a caller-provided uint32).
constexpr uint32_t kErrorNonFiniteInput = 1u << 0;
constexpr uint32_t kErrorNonFiniteOutput = 1u << 1;
constexpr uint32_t kErrorRange = 1u << 2;
constexpr uint32_t kErrorInternal = 1u << 3;

__device__ __forceinline__ bool IsFinite(float v) {
  return (__float_as_uint(v) & 0x7F800000u) != 0x7F800000u;
}

__device__ __forceinline__ void RaiseError(uint32_t* error, uint32_t bit) {
  if (error != nullptr) atomicOr(error, bit);
}

// Max over non-negative floats through their ordered bit patterns.
__device__ __forceinline__ void AtomicMaxNonNegative(float* address, float v) {
  atomicMax(reinterpret_cast<unsigned int*>(address), __float_as_uint(v));
}

__device__ __forceinline__ float WarpSum(float v) {
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, offset);
  }
  return v;
}

__device__ __forceinline__ float WarpMax(float v) {
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) {
    v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, offset));
  }
  return v;
}

// libjxl's CubeRootAndAdd (three reciprocal-cube-root Newton steps and one
// refinement), as pinned in the reference's codec/color_transform.cpp:54.
__device__ __forceinline__ float CubeRootAndAdd(float value, float add) {
  const float kOneThird = 1.0f / 3.0f;
  const float kFourThirds = 4.0f / 3.0f;
  const uint32_t bits = __float_as_uint(value);
  const uint32_t estimate =
    bits == 0 ? 0u : 0x54800000u - (bits >> 23) * 0x002AAAAAu;
  float r = __uint_as_float(estimate);
  const float divided = kOneThird * value;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float sq = r * r;
    r = fmaf(-divided, sq * sq, kFourThirds * r);
  }
  float sq = r * r;
  r = fmaf(kOneThird, fmaf(-value, sq * sq, r), r);
  sq = r * r;
  return fmaf(sq, value, add);
}

// libjxl's rational log2 / exp2 approximations (reference util/fast_math.h).
__device__ __forceinline__ float FastLog2(float value) {
  if (!IsFinite(value) || value <= 0.0f) return __int_as_float(0x7fc00000);
  const uint32_t bits = __float_as_uint(value);
  const int32_t e = static_cast<int32_t>(bits - 0x3f2aaaabu) >> 23;
  const uint32_t m = bits - (static_cast<uint32_t>(e) << 23);
  const float x = __uint_as_float(m) - 1.0f;
  float num = fmaf(0.74245873327820566f, x, 1.4287160470083755f);
  num = fmaf(num, x, -1.8503833400518310e-06f);
  float den = fmaf(0.17409343003366853f, x, 1.0096718572241148f);
  den = fmaf(den, x, 0.99032814277590719f);
  return num / den + static_cast<float>(e);
}

__device__ __forceinline__ float FastPow2(float value) {
  if (!IsFinite(value) || value < -126.0f || value > 127.0f) {
    return __int_as_float(0x7fc00000);
  }
  const float fl = floorf(value);
  const int32_t e = static_cast<int32_t>(fl) + 127;
  const float ev = __uint_as_float(static_cast<uint32_t>(e) << 23);
  const float f = value - fl;
  float num = f + 1.01749063e+01f;
  num = fmaf(num, f, 4.88687798e+01f);
  num = fmaf(num, f, 9.85506591e+01f);
  num *= ev;
  float den = fmaf(f, 2.10242958e-01f, -2.22328856e-02f);
  den = fmaf(den, f, -1.94414990e+01f);
  den = fmaf(den, f, 9.85506633e+01f);
  return num / den;
}

}  // namespace gjxl_b200
