// Entry point over the reference's own CUDA path, compiled for sm_100a from
// its sources by oracle/Makefile (target `cuda`) into
// oracle/_ref/libgjxl_ref_cuda.so.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY: bench.py times it as the
// reference's GPU baseline and the parity tests compare against its
// codestreams. The product library never links or loads it.
//
// It runs the reference's whole encode with its CUDA backend in the
// fully-resident adaptive-quantization mode, exactly as its
// cuda_encoding_benchmark does (benchmarks/cuda_encoding_benchmark.cpp:425-470):
// EncodeLinearRgbVarDctCodestreamProfiledWithBackendForTesting with an
// explicitly created CudaBackend, reporting the workflow's own phase timing
// (VarDctEncodingProfile::quantization_pipeline_nanoseconds, the analysis
// half).

#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "codestream/workflow.h"
#include "codestream/workflow_internal.h"
#include "gpu/cuda/cuda_backend.h"

#define GJXL_REF_API extern "C" __attribute__((visibility("default")))

namespace {

using namespace gjxl;

thread_local std::string g_last_error;
std::unique_ptr<GpuBackend> g_backend;

int Fail(const Status& status) {
  g_last_error = std::string(status.message());
  const int code = static_cast<int>(status.code());
  return code == 0 ? -1 : code;
}

}  // namespace

GJXL_REF_API const char* gjxl_ref_cuda_last_error(void) { return g_last_error.c_str(); }

// Creates the CUDA backend on device 0 once per process.
GJXL_REF_API int gjxl_ref_cuda_init(void) {
  if (g_backend) return 0;
  Status status = CreateCudaBackend(&g_backend);
  return status.ok() ? 0 : Fail(status);
}

GJXL_REF_API void gjxl_ref_cuda_release(void) { g_backend.reset(); }

// One encode of planar linear RGB (3 x height x width floats) at the given
// distance and effort. Outputs: the codestream (capacity bytes; -2 when it
// does not fit), its size, the final Butteraugli score and the analysis
// ("quantization pipeline") and total wall times in nanoseconds.
GJXL_REF_API int gjxl_ref_cuda_encode(const float* linear, size_t width, size_t height,
                                      float target, int effort, uint8_t* out,
                                      size_t capacity, size_t* size, double* score,
                                      uint64_t* analysis_ns, uint64_t* total_ns) {
  if (!g_backend) {
    g_last_error = "gjxl_ref_cuda_init was not called";
    return -1;
  }
  ConstImage3FView view;
  for (size_t c = 0; c < 3; ++c) {
    view.plane[c] = {linear + c * width * height, {width, height}, width};
  }
  VarDctEncodingOptions options;
  options.butteraugli_target = target;
  options.effort = effort;
  options.backend = VarDctBackendPreference::kCuda;
  options.gpu_aq_mode = GpuAdaptiveQuantizationMode::kFullyResident;
  options.collect_final_butteraugli_score = true;
  std::vector<uint8_t> bytes;
  VarDctEncodingSummary summary;
  codestream_internal::VarDctEncodingProfile profile;
  Status status = codestream_internal::EncodeLinearRgbVarDctCodestreamProfiledWithBackendForTesting(
    view, options, g_backend.get(), false, &bytes, &summary, &profile);
  if (!status.ok()) return Fail(status);
  *size = bytes.size();
  *score = summary.score_history.empty() ? 0.0 : summary.score_history.back();
  *analysis_ns = profile.quantization_pipeline_nanoseconds;
  *total_ns = profile.total_nanoseconds;
  if (bytes.size() > capacity) {
    g_last_error = "codestream capacity exceeded";
    return -2;
  }
  std::memcpy(out, bytes.data(), bytes.size());
  return 0;
}
