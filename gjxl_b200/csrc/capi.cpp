// Library-wide C-ABI plumbing: error reporting and version.
#include <string>

#include "host_util.h"

namespace gjxl_b200 {
namespace {
thread_local std::string g_last_error;
}  // namespace

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
