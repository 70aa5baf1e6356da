// Device calibration for roofline reporting (no counterpart in the
// reference): the FP64 multiply/add throughput of the current device.
//
// The bit-exact transform kernels (the candidate costs, CfL fits and
// reconstructions) restate the reference's double-precision DCT with every
// multiply and add rounded separately, so their ceiling is the rate at
// which the FP64 pipe retires DMUL and DADD instructions, one operation each.
// The calibration kernel runs that mix: eight independent chains per thread
// of x = x * a + b, built with --fmad=false like the library, on a grid of
// eight 256-thread CTAs per SM.

#include <cuda_runtime.h>

#include "gjxl_b200.h"
#include "host_util.h"

namespace gjxl_b200 {
namespace {

constexpr int kChains = 8;
constexpr int kCalibrationThreads = 256;

__global__ void __launch_bounds__(kCalibrationThreads)
Fp64ChainKernel(double* sink, int iterations, double a, double b) {
  double x[kChains];
#pragma unroll
  for (int j = 0; j < kChains; ++j) x[j] = 1e-3 * threadIdx.x + j;
  for (int i = 0; i < iterations; ++i) {
#pragma unroll
    for (int j = 0; j < kChains; ++j) x[j] = x[j] * a + b;
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < kChains; ++j) s += x[j];
  // Never true for the constants used; keeps the chains live.
  if (s != s) sink[0] = s;
}

}  // namespace
}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" int gjxl_b200_fp64_throughput(double* device_sink, double* ops_per_second,
                                         void* stream) {
  ClearLastError();
  if (device_sink == nullptr || ops_per_second == nullptr) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "fp64_throughput: null argument");
  }
  int device = 0, sms = 0;
  int status = CheckCuda(cudaGetDevice(&device), "fp64_throughput: cudaGetDevice");
  if (status != GJXL_B200_OK) return status;
  status = CheckCuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device),
                     "fp64_throughput: SM count");
  if (status != GJXL_B200_OK) return status;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int blocks = sms * 8, iterations = 100000;
  cudaEvent_t start = nullptr, stop = nullptr;
  status = CheckCuda(cudaEventCreate(&start), "fp64_throughput: event");
  if (status == GJXL_B200_OK) status = CheckCuda(cudaEventCreate(&stop), "fp64_throughput: event");
  float best_ms = 0.0f;
  for (int rep = 0; rep < 4 && status == GJXL_B200_OK; ++rep) {
    cudaEventRecord(start, st);
    Fp64ChainKernel<<<blocks, kCalibrationThreads, 0, st>>>(device_sink, iterations,
                                                            0.9999999, 1e-7);
    status = CheckLaunch("fp64_throughput: launch");
    cudaEventRecord(stop, st);
    if (status == GJXL_B200_OK) {
      status = CheckCuda(cudaEventSynchronize(stop), "fp64_throughput: synchronize");
    }
    float ms = 0.0f;
    if (status == GJXL_B200_OK) {
      status = CheckCuda(cudaEventElapsedTime(&ms, start, stop), "fp64_throughput: elapsed");
    }
    // The first repetition warms the clocks up; keep the fastest of the rest.
    if (rep > 0 && (best_ms == 0.0f || ms < best_ms)) best_ms = ms;
  }
  if (start != nullptr) cudaEventDestroy(start);
  if (stop != nullptr) cudaEventDestroy(stop);
  if (status != GJXL_B200_OK) return status;
  const double ops = static_cast<double>(blocks) * kCalibrationThreads * kChains * 2.0 *
                     iterations;
  *ops_per_second = ops / (static_cast<double>(best_ms) * 1e-3);
  return GJXL_B200_OK;
}
