// Initial quantization field with library-owned scratch: the one entry point
// of this library that allocates no device memory when it is called.
//
// gjxl_b200_initial_quant_field needs scratch device memory (the raw pixel
// mask and the 4x4 pre-erosion grid, 4.25 bytes per padded pixel) that its
// caller allocates. Some callers cannot allocate:
//  - an encoder service that reserves all of its device memory at start-up
//    under a fixed budget: cudaMalloc / cudaFree in the per-image path can
//    synchronize the whole device (stalling the other streams' work) and an
//    out-of-memory failure half-way through an image cannot be recovered;
//  - a plug-in host that hands the analysis only its own image planes and
//    has no device allocator to draw scratch from.
// This variant takes the scratch from a fixed, statically sized device array
// instead. It has no counterpart in the reference.
//
// Set-up: the first call in each CUDA context (normally a device's primary
// context) looks up the array's address there with cudaGetSymbolAddress
// (which also loads this module's device memory in that context); make that
// first call before any stream capture. The address belongs to that context:
// it is cached under the context's unique id, so a call in another context,
// or after cudaDeviceReset replaced the primary context, looks it up again
// instead of using a stale address. Later calls only launch the three
// kernels of the initial quantization field.
//
// Like every __device__ array, the 16 MiB are held on each device whose
// context loads this library's module, whether or not this entry point is
// ever called, until the context is destroyed.
//
// Every scratch element is written before it is read (the pre-erosion kernel
// writes every pixel of the raw mask and every 4x4 cell of the grid), so
// nothing in the scratch has to start at zero and nothing is cleared.
// `device_error` is the caller's word, OR'ed into as by the caller-scratch
// entry point.
//
// There is one scratch array per device: calls that overlap on one device
// (on different streams, or from different host threads without ordering)
// race on it. Callers serialize them, e.g. by using one stream.

#include <cuda.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "host_util.h"
#include "session.h"

// 16 MiB of scratch: padded images of at most 3,947,580 pixels
// (4 Mi floats / 1.0625 floats per padded pixel), e.g. 2048 x 1920.
constexpr size_t kNoAllocScratchFloats = size_t{4} << 20;
static __device__ __align__(256) float g_initial_quant_scratch[kNoAllocScratchFloats];

namespace gjxl_b200 {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
struct ScratchAddress {
  unsigned long long context_id = 0;  // 0: not looked up yet
  float* address = nullptr;
};
ScratchAddress g_scratch_address[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (never reused within a
// process, unlike the CUcontext handle), through the runtime's driver entry
// points so the library needs no link against the driver library. Returns
// false (and *id = 0) when no context is current.
bool CurrentContextId(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult found;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &found) ==
            cudaSuccess && found == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    fn = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &found) == cudaSuccess &&
        found == cudaDriverEntryPointSuccess) {
      get_id = reinterpret_cast<CtxGetIdFn>(fn);
    }
    cudaGetLastError();
  });
  *id = 0;
  CUcontext context = nullptr;
  if (get_current == nullptr || get_id == nullptr || get_current(&context) != CUDA_SUCCESS ||
      context == nullptr || get_id(context, id) != CUDA_SUCCESS) {
    *id = 0;
  }
  return *id != 0;
}

// Address of the static scratch in the current context, looked up once per
// context. With no context current yet, the lookup itself makes the device's
// primary context current (as any runtime call does), and the address is
// cached under that context's id.
int NoAllocScratch(float** out) {
  int device = -1;
  int status = CheckCuda(cudaGetDevice(&device), "initial_quant_field_noalloc: cudaGetDevice");
  if (status != GJXL_B200_OK) return status;
  if (device < 0 || device >= kMaxDevices) {
    return SetError(GJXL_B200_UNSUPPORTED, "initial_quant_field_noalloc: device ordinal >= 64");
  }
  unsigned long long context_id = 0;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  ScratchAddress& cached = g_scratch_address[device];
  if (!CurrentContextId(&context_id) || cached.context_id != context_id) {
    float* address = nullptr;
    status = CheckCuda(cudaGetSymbolAddress(reinterpret_cast<void**>(&address),
                                            g_initial_quant_scratch),
                       "initial_quant_field_noalloc: cudaGetSymbolAddress");
    if (status != GJXL_B200_OK) return status;
    if (!CurrentContextId(&context_id)) {
      return SetError(GJXL_B200_UNAVAILABLE,
                      "initial_quant_field_noalloc: no current CUDA context id");
    }
    cached.context_id = context_id;
    cached.address = address;
  }
  *out = cached.address;
  return GJXL_B200_OK;
}

}  // namespace
}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" int gjxl_b200_initial_quant_field_noalloc(
  const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch, size_t padded_width,
  size_t padded_height, float butteraugli_target, float rescale, float* quant_field,
  float* strategy_mask, float* pixel_mask, size_t pixel_mask_stride, uint32_t* device_error,
  void* stream) {
  ClearLastError();
  if (opsin == nullptr || quant_field == nullptr || strategy_mask == nullptr ||
      pixel_mask == nullptr || padded_width % 8 != 0 || padded_height % 8 != 0 ||
      padded_width == 0 || padded_height == 0 || padded_width > (size_t{1} << 20) ||
      padded_height > (size_t{1} << 20) || opsin_stride % 4 != 0 ||
      opsin_plane_pitch % 4 != 0 || opsin_stride < padded_width || !Aligned16(opsin) ||
      opsin_plane_pitch < opsin_stride * padded_height || pixel_mask_stride < padded_width ||
      !std::isfinite(butteraugli_target) || butteraugli_target <= 0.0f ||
      !std::isfinite(rescale) || rescale <= 0.0f) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "initial_quant_field_noalloc: invalid arguments");
  }
  if (InitialQuantScratchFloats(padded_width, padded_height) > kNoAllocScratchFloats) {
    return SetError(GJXL_B200_INVALID_ARGUMENT,
                    "initial_quant_field_noalloc: the padded image needs more scratch than the "
                    "16 MiB static array holds (at most 3,947,580 padded pixels); use "
                    "gjxl_b200_initial_quant_field with caller scratch");
  }
  float* scratch = nullptr;
  const int status = NoAllocScratch(&scratch);
  if (status != GJXL_B200_OK) return status;
  return LaunchInitialQuantField(opsin, opsin_stride, opsin_plane_pitch, padded_width,
                                 padded_height, butteraugli_target, rescale, quant_field,
                                 strategy_mask, pixel_mask, pixel_mask_stride, scratch,
                                 device_error, static_cast<cudaStream_t>(stream));
}
