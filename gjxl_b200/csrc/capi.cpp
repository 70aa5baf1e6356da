// Library-wide C-ABI plumbing: error reporting and version.
#include <string>

#include "host_util.h"

namespace gjxl_b200 {
namespace {
thread_local std::string g_last_error;
// Armed check point per failure kind (0 = disarmed), counted down per thread.
thread_local int g_inject_countdown[kInjectKinds] = {};
}  // namespace

bool InjectFailure(int kind) {
  if (kind <= 0 || kind >= kInjectKinds || g_inject_countdown[kind] == 0) return false;
  return --g_inject_countdown[kind] == 0;
}

cudaError_t DeviceMalloc(void** ptr, size_t bytes) {
  if (InjectFailure(kInjectAllocation)) return cudaErrorMemoryAllocation;
  return cudaMalloc(ptr, bytes);
}

cudaError_t HostMalloc(void** ptr, size_t bytes) {
  if (InjectFailure(kInjectAllocation)) return cudaErrorMemoryAllocation;
  return cudaMallocHost(ptr, bytes);
}

void ClearLastError() { g_last_error.clear(); }

int SetError(int code, const char* message) {
  g_last_error = message;
  return code;
}

int CheckCuda(cudaError_t error, const char* what) {
  if (error == cudaSuccess) return GJXL_B200_OK;
  g_last_error = std::string(what) + ": " + cudaGetErrorString(error);
  switch (error) {
    case cudaErrorMemoryAllocation:
      return GJXL_B200_OUT_OF_MEMORY;
    case cudaErrorInvalidValue:
    case cudaErrorInvalidConfiguration:
    case cudaErrorInvalidDevicePointer:
      return GJXL_B200_SUBMISSION_FAILED;
    case cudaErrorNoDevice:
    case cudaErrorInsufficientDriver:
    case cudaErrorNoKernelImageForDevice:
      return GJXL_B200_UNAVAILABLE;
    default:
      return GJXL_B200_DEVICE_ERROR;
  }
}

int CheckLaunch(const char* what) { return CheckCuda(cudaGetLastError(), what); }

}  // namespace gjxl_b200

extern "C" const char* gjxl_b200_last_error(void) {
  return gjxl_b200::g_last_error.c_str();
}

extern "C" int gjxl_b200_version(void) { return 100; }

extern "C" int gjxl_b200_test_arm_failure(int kind, int check_point) {
  gjxl_b200::ClearLastError();
  if (kind <= 0 || kind >= gjxl_b200::kInjectKinds || check_point < 0) {
    return gjxl_b200::SetError(GJXL_B200_INVALID_ARGUMENT, "test_arm_failure: invalid kind");
  }
  gjxl_b200::g_inject_countdown[kind] = check_point;
  return GJXL_B200_OK;
}

extern "C" int gjxl_b200_check_device_error(const uint32_t* device_error, size_t words,
                                            void* stream) {
  using namespace gjxl_b200;
  ClearLastError();
  if (device_error == nullptr || words == 0 || words > 64) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "check_device_error: 1..64 words");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t host[64] = {};
  int status = CheckCuda(cudaStreamSynchronize(s), "check_device_error: synchronize");
  if (status != GJXL_B200_OK) return status;
  status = CheckCuda(cudaMemcpy(host, device_error, words * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost),
                     "check_device_error: read");
  if (status != GJXL_B200_OK) return status;
  for (size_t i = 0; i < words; ++i) {
    if (host[i] != 0) {
      g_last_error = "device error word " + std::to_string(i) + " = " + std::to_string(host[i]) +
                     " (1 non-finite input, 2 non-finite output, 4 range, 8 internal)";
      return GJXL_B200_DEVICE_ERROR;
    }
  }
  return GJXL_B200_OK;
}
