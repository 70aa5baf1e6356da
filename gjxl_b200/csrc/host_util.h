// Host-side helpers shared by the C-ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>

#include "gjxl_b200.h"

namespace gjxl_b200 {

// Thread-local last-error message (mirrors gjxl_get_last_error's contract).
void ClearLastError();
int SetError(int code, const char* message);

// Maps a pending CUDA launch error to DEVICE_ERROR / SUBMISSION_FAILED.
int CheckLaunch(const char* what);
int CheckCuda(cudaError_t error, const char* what);

// Deterministic failure injection for tests (gjxl_b200_test_arm_failure):
// returns true, once, when the calling thread's countdown for `kind` reaches
// its armed check point.
enum InjectedFailure : int {
  kInjectAllocation = 1,
  kInjectGraph = 2,
  kInjectSubmission = 3,
  kInjectKinds = 4,
};
bool InjectFailure(int kind);

// Device / pinned host allocations of the handle constructors; both are
// allocation check points of the failure injection.
cudaError_t DeviceMalloc(void** ptr, size_t bytes);
cudaError_t HostMalloc(void** ptr, size_t bytes);

inline bool Aligned16(const void* p) {
  return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

// sRGB transfer decode in double precision, rounded to float
// (src/c_api/image_conversion.cpp:18-31).
inline float SrgbToLinear(int i) {
  const double encoded = static_cast<double>(i) / 255.0;
  const double linear = encoded <= 0.04045 ? encoded / 12.92
                                           : std::pow((encoded + 0.055) / 1.055, 2.4);
  return static_cast<float>(linear);
}

// Host copy of CubeRootAndAdd for constants (src/codec/color_transform.cpp:54).
inline float HostCubeRootAndAdd(float value, float add) {
  const float kOneThird = 1.0f / 3.0f;
  const float kFourThirds = 4.0f / 3.0f;
  uint32_t bits;
  std::memcpy(&bits, &value, 4);
  const uint32_t est = bits == 0 ? 0u : 0x54800000u - (bits >> 23) * 0x002AAAAAu;
  float r;
  std::memcpy(&r, &est, 4);
  const float divided = kOneThird * value;
  for (int i = 0; i < 3; ++i) {
    const float sq = r * r;
    r = std::fma(-divided, sq * sq, kFourThirds * r);
  }
  float sq = r * r;
  r = std::fma(kOneThird, std::fma(-value, sq * sq, r), r);
  sq = r * r;
  return std::fma(sq, value, add);
}

}  // namespace gjxl_b200
