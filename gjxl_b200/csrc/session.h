// Host-side analysis session: the B200 counterpart of the reference's
// PreparedQuantizationPipeline + PreparedResidentInput
// (src/codec/quantization_pipeline_internal.h:77-118,
// src/gpu/ops/resident_input.h:34-57). Owns every device buffer for one image
// extent and enqueues the analysis stages on the caller's stream.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "fan.h"
#include "gjxl_b200.h"

namespace gjxl_b200 {

// Entry points of the stage translation units.
int LaunchInitialQuantField(const float* opsin, size_t stride, size_t pitch, size_t pw,
                            size_t ph, float target, float rescale, float* quant_field,
                            float* strategy_mask, float* pixel_mask, size_t mask_stride,
                            float* scratch, uint32_t* error, cudaStream_t stream);
size_t InitialQuantScratchFloats(size_t padded_width, size_t padded_height);
int LaunchGaborishInverse(const float* input, size_t in_stride, size_t in_pitch, float* output,
                          size_t out_stride, size_t out_pitch, size_t width, size_t height,
                          const float multipliers[3], uint32_t* error, cudaStream_t stream);
// DC-group token streams (dc_tokens.cu).
size_t DcTokenScratchBytes(size_t blocks_x, size_t blocks_y);
size_t MetaTokenCapacity(size_t blocks_x, size_t blocks_y);
int LaunchMetaTokens(const uint8_t* cells, const int32_t* raw_quant, const uint8_t* sharpness,
                     const int8_t* y_to_x, const int8_t* y_to_b, size_t blocks_x, size_t blocks_y,
                     const uint2* dc_tokens, uint2* meta_tokens, uint32_t* info,
                     uint32_t* histogram, void* scratch, uint32_t* error, cudaStream_t stream);
int LaunchInitialCfl(const float* opsin, size_t stride, size_t pitch, size_t pw, size_t ph,
                     int8_t* y_to_x, int8_t* y_to_b, cudaStream_t stream);
size_t AcStrategyCostFloats(size_t blocks_x, size_t blocks_y);
int LaunchAcStrategyCosts(const float* opsin, size_t stride, size_t pitch, size_t pw, size_t ph,
                          const float* quant_field, const float* pixel_mask, size_t mask_stride,
                          const int8_t* y_to_x, const int8_t* y_to_b, float target, bool dense,
                          int precision, float* costs, uint32_t* error, cudaStream_t stream,
                          const StreamFan* fan = nullptr, const uint32_t* kept_tiles = nullptr,
                          const uint32_t* kept_counts = nullptr);
int LaunchAcStrategySearch(const float* costs, size_t pw, size_t ph, float target, bool dense,
                           uint8_t* cells, uint32_t* error, cudaStream_t stream);

struct ButteraugliState;
// Planes of one Butteraugli state; `external` (nullable) lends them.
size_t ButteraugliArenaBytes(size_t width, size_t height);
int ButteraugliCreate(size_t width, size_t height, float intensity_target, void* external,
                      ButteraugliState** out);
void ButteraugliDestroy(ButteraugliState* state);
int ButteraugliPrepare(ButteraugliState* st, const float* linear, size_t stride, size_t pitch,
                       cudaStream_t stream);
int ButteraugliCompare(ButteraugliState* st, const float* linear, size_t stride, size_t pitch,
                       float* map, size_t map_stride, double* score, cudaStream_t stream);
uint32_t* ButteraugliErrorWord(ButteraugliState* st);

// FP64 global Butteraugli p-norm of a distance map (pnorm.cu).
size_t PnormScratchBytes();
int LaunchPnorm(const float* map, size_t stride, size_t width, size_t height, double p,
                double* scratch, double* out, cudaStream_t stream);

}  // namespace gjxl_b200
