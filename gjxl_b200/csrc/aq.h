// Device structures and launchers of the adaptive-quantization evaluation.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "fan.h"

namespace gjxl_b200 {

// Device copy of the reference's Quantizer (src/core/quantizer.h:24-120).
struct AqQuantizer {
  uint32_t global_scale;
  uint32_t quant_dc;
  float scale;
  float inverse_global_scale;
  float dc_steps[3];
  float inverse_dc_steps[3];
};

// ButteraugliPolicySetup (src/codec/adaptive_quantization_internal.h).
struct AqPolicy {
  float lower_bound;
  float upper_bound;
  float quant_dc;
  float pad;
};

void UploadDcTables();
void UploadDcReconTables();
int AqMatrixScales(const float* stats, bool have_stats, float target, float* multipliers,
                   int* scales, cudaStream_t stream);
int AqBuildAnchors(const uint8_t* cells, size_t bx, size_t by, int2* lists, uint32_t* counts,
                   cudaStream_t stream);
int AqForwardCoefficients(const float* opsin, size_t stride, size_t pitch, size_t bx, size_t by,
                          const int2* lists, const uint32_t* counts, float* coef,
                          cudaStream_t stream, const StreamFan* fan = nullptr);
int AqAdjustField(const uint8_t* cells, size_t bx, size_t by, const float* in, float* out,
                  float target, cudaStream_t stream);
int AqPolicySetup(const float* field, size_t blocks, float target, float* range,
                  AqPolicy* policy, uint32_t* error, cudaStream_t stream);
// Device state of the quantizer's median / deviation selection.
size_t AqSelectStateBytes();
int AqQuantizer_(const float* field, size_t blocks, const AqPolicy* policy, AqQuantizer* q,
                 int32_t* raw, void* select_state, uint32_t* error, cudaStream_t stream);
int AqFinalCfl(const uint8_t* cells, size_t bx, size_t by, const float* coef, size_t stride,
               size_t pitch, const int32_t* raw, const AqQuantizer* q, int8_t* y_to_x,
               int8_t* y_to_b, cudaStream_t stream);
int AqCoding(const int2* lists, const uint32_t* counts, size_t bx, size_t by, const float* coef,
             size_t stride, size_t pitch, int32_t* qac, float* dc, int32_t* raw,
             const AqQuantizer* q, const int8_t* y_to_x, const int8_t* y_to_b,
             const float* matrix_multiplier, uint32_t* error, cudaStream_t stream,
             const StreamFan* fan = nullptr);
// Prediction-aware DC quantization; with `tokens`, also the weighted-predictor
// DC token stream (DcTokenOffset layout), residual range errors to `error`.
int AqDcQuantize(const float* dc, size_t bx, size_t by, const AqQuantizer* q, int32_t* quantized,
                 float* reconstructed, int extra_precision, uint2* tokens, uint32_t* error,
                 cudaStream_t stream);
// The weighted-predictor DC tokens of quantized DC (3 planes of `pitch`).
int DcWeightedTokens(const int32_t* quantized, size_t pitch, size_t bx, size_t by, uint2* tokens,
                     uint32_t* error, cudaStream_t stream);
int AqInverseSigma(const uint8_t* cells, size_t bx, size_t by, const int32_t* raw,
                   const AqQuantizer* q, float* inverse_sigma, cudaStream_t stream);

// Reconstruction side (aq_recon.cu).
int AqSmoothDc(const float* dc, size_t bx, size_t by, const AqQuantizer* q, float* out,
               cudaStream_t stream);
int AqReconstruct(const int2* lists, const uint32_t* counts, size_t bx, size_t by,
                  const int32_t* qac, size_t stride, size_t pitch, const float* dc,
                  const int32_t* raw, const AqQuantizer* q, const int8_t* y_to_x,
                  const int8_t* y_to_b, const float* matrix_multiplier, float* recon,
                  cudaStream_t stream, const StreamFan* fan = nullptr);
// With `linear` non-null the last pass writes OpsinToLinear of the filtered
// image (at intensity_target) there instead of the filtered planes.
int AqLoopFilters(const float* recon, size_t recon_stride, size_t recon_pitch, size_t width,
                  size_t height, const float* inverse_sigma, size_t bx, float* scratch_a,
                  float* scratch_b, float* filtered, uint32_t* error, cudaStream_t stream,
                  float* linear = nullptr, float intensity_target = 80.0f);
int AqOpsinToLinear(const float* opsin, size_t width, size_t height, float intensity_target,
                    float* linear, uint32_t* error, cudaStream_t stream);
int AqBlockReduce(const uint8_t* cells, size_t bx, size_t by, const float* distance_map,
                  size_t width, size_t height, float* block_distance, cudaStream_t stream);
int AqPolicyUpdate(float* field, const float* adjusted_initial, const float* block_distance,
                   size_t blocks, int iteration, float target, const AqPolicy* policy,
                   const AqQuantizer* q, uint32_t* error, cudaStream_t stream);

}  // namespace gjxl_b200
