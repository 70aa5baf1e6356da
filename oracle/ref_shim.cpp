// Stage-level C entry points over the gjxl reference's own CPU analysis code.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the
// reference's sources (src/core, src/codec, part of src/codestream) into
// oracle/_ref/libgjxl_ref.so by oracle/Makefile. The parity tests call it as
// the checker, and bench.py's reference arm times it as the CPU baseline.
// The product library never links or loads it.
//
// Every function takes planar float images (plane-major, rows contiguous,
// stride == width) and returns 0 on success or the reference's StatusCode
// value on failure (the message is kept for gjxl_ref_last_error()).

#include <algorithm>
#include <array>
#include <memory>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <optional>
#include <string>
#include <vector>

#include "c_api/image_conversion.h"
#include "codec/ac_strategy.h"
#include "codec/adaptive_quantization.h"
#include "codec/butteraugli.h"
#include "codec/chroma_from_luma.h"
#include "codec/chroma_from_luma_internal.h"
#include "codec/color_transform.h"
#include "codec/color_transform_internal.h"
#include "codec/gaborish.h"
#include "codec/quantization.h"
#include "codec/quantization_pipeline.h"
#include "codec/quantization_pipeline_internal.h"
#include "codec/vardct_frame.h"
#include "codestream/ac_group.h"
#include "codestream/block_context_map.h"
#include "codestream/coefficient_order.h"
#include "codestream/dc_group.h"
#include "codestream/ans_internal.h"
#include "codestream/bit_writer.h"
#include "codestream/entropy.h"
#include "codestream/entropy_internal.h"
#include "codestream/weighted_dc.h"
#include "codestream/encoder.h"
#include "codestream/workflow.h"
#include "codestream/workflow_internal.h"
#include "codec/vardct_frame_view_internal.h"
#include "core/ac_strategy.h"
#include "core/image.h"
#include "core/publication_vector.h"
#include "core/thread_budget.h"

#define GJXL_REF_API extern "C" __attribute__((visibility("default")))

namespace {

using namespace gjxl;

thread_local std::string g_last_error;

int Fail(const Status& status) {
  g_last_error = std::string(status.message());
  int code = static_cast<int>(status.code());
  return code == 0 ? -1 : code;
}

ConstImage3FView ConstPlanar(const float* data, size_t width, size_t height) {
  ConstImage3FView view;
  for (size_t c = 0; c < 3; ++c) {
    view.plane[c] = {data + c * width * height, {width, height}, width};
  }
  return view;
}

Image3FView Planar(float* data, size_t width, size_t height) {
  Image3FView view;
  for (size_t c = 0; c < 3; ++c) {
    view.plane[c] = {data + c * width * height, {width, height}, width};
  }
  return view;
}

Status MakeColorCorrelation(const int8_t* y_to_x, const int8_t* y_to_b,
                            size_t padded_width, size_t padded_height,
                            ColorCorrelationMap* out) {
  const Extent2D tiles = ColorTileExtent({padded_width, padded_height});
  return chroma_from_luma_internal::CreateColorCorrelationMap(
    {y_to_x, tiles, tiles.width}, {y_to_b, tiles, tiles.width}, out);
}

void ExportColorCorrelation(const ColorCorrelationMap& map, int8_t* y_to_x,
                            int8_t* y_to_b) {
  const ConstPlaneI8View x = map.y_to_x_map();
  const ConstPlaneI8View b = map.y_to_b_map();
  for (size_t y = 0; y < x.extent.height; ++y) {
    std::memcpy(y_to_x + y * x.extent.width, x.Row(y), x.extent.width);
    std::memcpy(y_to_b + y * b.extent.width, b.Row(y), b.extent.width);
  }
}

Status ExportGrid(const AcStrategyGrid& grid, uint8_t* cells) {
  const Extent2D extent = grid.extent();
  for (size_t y = 0; y < extent.height; ++y) {
    for (size_t x = 0; x < extent.width; ++x) {
      AcStrategyCell cell;
      Status status = grid.Get(x, y, &cell);
      if (!status.ok()) return status;
      cells[y * extent.width + x] = static_cast<uint8_t>(
        (static_cast<uint8_t>(cell.strategy) << 1) | (cell.is_anchor ? 1 : 0));
    }
  }
  return Status::Ok();
}

}  // namespace

GJXL_REF_API const char* gjxl_ref_last_error(void) {
  return g_last_error.c_str();
}

// CPU thread budget installed around the pipeline entry points, as the
// workflow installs options.cpu_thread_count (src/codestream/workflow.cpp:1640).
// 0 leaves the calling thread's budget untouched (serial outside an encode).
static size_t g_threads = 0;

GJXL_REF_API int gjxl_ref_set_threads(size_t threads) {
  g_threads = threads;
  return 0;
}

// c_api/image_conversion.cpp: packed 8-bit sRGB (3 or 4 bytes per pixel) to
// planar linear RGB through the reference's double-precision table.
GJXL_REF_API int gjxl_ref_srgb8_to_linear(const uint8_t* pixels, size_t width,
                                          size_t height, size_t row_stride,
                                          int channels, float* linear) {
  c_api_internal::PackedSrgbImageView image{};
  image.pixels = pixels;
  image.pixels_size = row_stride * (height - 1) + width * channels;
  image.width = static_cast<uint32_t>(width);
  image.height = static_cast<uint32_t>(height);
  image.row_stride_bytes = row_stride;
  image.format = channels == 4 ? c_api_internal::PackedPixelFormat::kRgba8Srgb
                               : c_api_internal::PackedPixelFormat::kRgb8Srgb;
  Status status = c_api_internal::ConvertValidatedPackedSrgbInto(
    image, Planar(linear, width, height));
  return status.ok() ? 0 : Fail(status);
}

// codec/color_transform.cpp LinearRgbToPaddedOpsin at the workflow's
// intensity target of 255.
GJXL_REF_API int gjxl_ref_linear_to_padded_opsin(
  const float* linear, size_t width, size_t height, float* opsin,
  size_t padded_width, size_t padded_height, float intensity_target) {
  Status status = color_transform_internal::LinearRgbToPaddedOpsin(
    ConstPlanar(linear, width, height), intensity_target,
    Planar(opsin, padded_width, padded_height));
  return status.ok() ? 0 : Fail(status);
}

GJXL_REF_API int gjxl_ref_opsin_to_linear(const float* opsin, size_t width,
                                          size_t height, float intensity_target,
                                          float* linear) {
  Status status = OpsinToLinearRgb(ConstPlanar(opsin, width, height),
                                   intensity_target,
                                   Planar(linear, width, height));
  return status.ok() ? 0 : Fail(status);
}

// codec/adaptive_quantization.cpp ComputeInitialQuantField.
GJXL_REF_API int gjxl_ref_initial_quant_field(
  const float* opsin, size_t padded_width, size_t padded_height,
  float butteraugli_target, float rescale, int uniform, float* quant_field,
  float* strategy_mask, float* pixel_mask) {
  const Extent2D blocks{padded_width / 8, padded_height / 8};
  const Extent2D pixels{padded_width, padded_height};
  InitialQuantFieldOutput output{
    .quant_field = {quant_field, blocks, blocks.width},
    .strategy_mask = {strategy_mask, blocks, blocks.width},
    .pixel_mask = {pixel_mask, pixels, pixels.width},
  };
  Status status = ComputeInitialQuantField(
    ConstPlanar(opsin, padded_width, padded_height),
    {.butteraugli_target = butteraugli_target,
     .rescale = rescale,
     .uniform = uniform != 0},
    output);
  return status.ok() ? 0 : Fail(status);
}

// codec/gaborish.cpp ApplyGaborishInverse.
GJXL_REF_API int gjxl_ref_gaborish_inverse(const float* input, size_t width,
                                           size_t height,
                                           const float* multipliers,
                                           float* output) {
  Status status = ApplyGaborishInverse(
    ConstPlanar(input, width, height),
    {multipliers[0], multipliers[1], multipliers[2]},
    Planar(output, width, height));
  return status.ok() ? 0 : Fail(status);
}

// codec/gaborish.cpp ApplyGaborish with default weights.
GJXL_REF_API int gjxl_ref_gaborish(const float* input, size_t width,
                                   size_t height, float* output) {
  Status status = ApplyGaborish(ConstPlanar(input, width, height),
                                GaborishOptions{},
                                Planar(output, width, height));
  return status.ok() ? 0 : Fail(status);
}

// codec/chroma_from_luma.cpp initial CfL maps (fast or regression form).
GJXL_REF_API int gjxl_ref_initial_cfl(const float* opsin, size_t padded_width,
                                      size_t padded_height, int fast,
                                      int8_t* y_to_x, int8_t* y_to_b) {
  ColorCorrelationMap map;
  Status status =
    fast ? chroma_from_luma_internal::ComputeInitialColorCorrelationMapFast(
             ConstPlanar(opsin, padded_width, padded_height), &map)
         : ComputeInitialColorCorrelationMap(
             ConstPlanar(opsin, padded_width, padded_height), &map);
  if (!status.ok()) return Fail(status);
  ExportColorCorrelation(map, y_to_x, y_to_b);
  return 0;
}

// codec/ac_strategy.cpp EstimateAcStrategyCost for one candidate.
GJXL_REF_API int gjxl_ref_ac_strategy_cost(
  const float* opsin, size_t padded_width, size_t padded_height,
  const float* quant_field, const float* pixel_mask, int strategy,
  size_t block_x, size_t block_y, float butteraugli_target,
  float entropy_multiplier, const float* cfl_factors, float* cost) {
  const Extent2D blocks{padded_width / 8, padded_height / 8};
  AcStrategyCostOptions options{
    .butteraugli_target = butteraugli_target,
    .entropy_multiplier = entropy_multiplier,
    .cfl_factors = {cfl_factors[0], cfl_factors[1], cfl_factors[2]},
  };
  Status status = EstimateAcStrategyCost(
    static_cast<AcStrategyType>(strategy), block_x, block_y,
    ConstPlanar(opsin, padded_width, padded_height),
    {quant_field, blocks, blocks.width},
    {pixel_mask, {padded_width, padded_height}, padded_width}, options, cost);
  return status.ok() ? 0 : Fail(status);
}

// codec/ac_strategy.cpp FindAcStrategyGrid. Cells use the reference's
// encoding (strategy << 1) | anchor.
GJXL_REF_API int gjxl_ref_ac_strategy_search(
  const float* opsin, size_t padded_width, size_t padded_height,
  const float* quant_field, const float* pixel_mask, const int8_t* y_to_x,
  const int8_t* y_to_b, float butteraugli_target, int dense_dct32,
  uint8_t* cells) {
  const Extent2D blocks{padded_width / 8, padded_height / 8};
  ColorCorrelationMap cfl;
  Status status =
    MakeColorCorrelation(y_to_x, y_to_b, padded_width, padded_height, &cfl);
  if (!status.ok()) return Fail(status);
  AcStrategyGrid grid;
  status = FindAcStrategyGrid(
    ConstPlanar(opsin, padded_width, padded_height),
    {quant_field, blocks, blocks.width},
    {pixel_mask, {padded_width, padded_height}, padded_width}, cfl,
    {.butteraugli_target = butteraugli_target,
     .dense_dct32_search = dense_dct32 != 0},
    &grid);
  if (!status.ok()) return Fail(status);
  status = ExportGrid(grid, cells);
  return status.ok() ? 0 : Fail(status);
}

// codec/butteraugli.cpp ComputeButteraugliDistance (default options).
GJXL_REF_API int gjxl_ref_butteraugli(const float* reference_linear,
                                      const float* distorted_linear,
                                      size_t width, size_t height,
                                      float intensity_target,
                                      float* distance_map, double* score) {
  ButteraugliOptions options;
  options.intensity_target = intensity_target;
  Status status = ComputeButteraugliDistance(
    ConstPlanar(reference_linear, width, height),
    ConstPlanar(distorted_linear, width, height), options,
    {distance_map, {width, height}, width}, score);
  return status.ok() ? 0 : Fail(status);
}

// codec/quantization.cpp GetDefaultQuantizationMatrix.
GJXL_REF_API int gjxl_ref_quant_matrix(int strategy, int channel, float* dequant,
                                       float* inverse_dequant, size_t capacity) {
  QuantizationMatrixView view;
  Status status = GetDefaultQuantizationMatrix(static_cast<AcStrategyType>(strategy),
                                               static_cast<XybChannel>(channel), &view);
  if (!status.ok()) return Fail(status);
  if (capacity < view.dequant.size()) return -1;
  std::memcpy(dequant, view.dequant.data(), view.dequant.size() * sizeof(float));
  std::memcpy(inverse_dequant, view.inverse_dequant.data(),
              view.inverse_dequant.size() * sizeof(float));
  return static_cast<int>(view.dequant.size());
}

// Cost table of every candidate the search can ask for: for each of the seven
// searched families (candidate-stage order DCT8, 16x8, 8x16, 16x16, 32x16,
// 16x32, 32x32), EstimateAcStrategyCost at every anchor that fits inside its
// 64x64 tile on the family's anchor step, with the stage's entropy multiplier
// and the tile's CfL factors. Other entries are left untouched.
GJXL_REF_API int gjxl_ref_ac_strategy_cost_table(
  const float* opsin, size_t padded_width, size_t padded_height, const float* quant_field,
  const float* pixel_mask, const int8_t* y_to_x, const int8_t* y_to_b,
  float butteraugli_target, int dense_dct32, float* costs) {
  const Extent2D blocks{padded_width / 8, padded_height / 8};
  ColorCorrelationMap cfl;
  Status status =
    MakeColorCorrelation(y_to_x, y_to_b, padded_width, padded_height, &cfl);
  if (!status.ok()) return Fail(status);
  const int strategies[7] = {0, 6, 7, 4, 10, 11, 5};
  const float entropy[7] = {1.0f, 1.21f, 1.21f, 1.34f, 1.49f, 1.49f, 1.48f};
  const int steps[7] = {1, 1, 1, 1, 2, 2, 2};
  for (int f = 0; f < 7; ++f) {
    const AcStrategyInfo* info = GetAcStrategyInfo(static_cast<AcStrategyType>(strategies[f]));
    const size_t cw = info->covered_blocks.width, ch = info->covered_blocks.height;
    const size_t step = (dense_dct32 && f >= 4) ? 1 : steps[f];
    for (size_t by = 0; by < blocks.height; ++by) {
      for (size_t bx = 0; bx < blocks.width; ++bx) {
        const size_t lx = bx % 8, ly = by % 8;
        const size_t tile_w = std::min<size_t>(8, blocks.width - (bx - lx));
        const size_t tile_h = std::min<size_t>(8, blocks.height - (by - ly));
        if (lx % step || ly % step || lx + cw > tile_w || ly + ch > tile_h) continue;
        float cost = 0.0f;
        status = EstimateAcStrategyCost(
          static_cast<AcStrategyType>(strategies[f]), bx, by,
          ConstPlanar(opsin, padded_width, padded_height),
          {quant_field, blocks, blocks.width},
          {pixel_mask, {padded_width, padded_height}, padded_width},
          {.butteraugli_target = butteraugli_target,
           .entropy_multiplier = entropy[f],
           .cfl_factors = cfl.AcFactors(bx / 8, by / 8)},
          &cost);
        if (!status.ok()) return Fail(status);
        costs[f * blocks.width * blocks.height + by * blocks.width + bx] = cost;
      }
    }
  }
  return 0;
}

// Butteraugli golden vectors of the reference's own test suite
// (tests/butteraugli_goldens_generated.h, generated there from libjxl
// e8ff0976 scalar Butteraugli) and the fixture pairs they were computed on
// (tests/butteraugli_fixtures.cpp MakeFixture).
#include "butteraugli_fixtures.h"
#include "butteraugli_goldens_generated.h"

GJXL_REF_API int gjxl_ref_butteraugli_fixture(int kind, size_t width, size_t height,
                                              uint32_t seed, size_t impulse_channel,
                                              float* reference, float* distorted,
                                              float* options3) {
  namespace bt = gjxl::butteraugli_test;
  bt::FixtureSpec spec;
  spec.name = "fixture";
  spec.extent = {width, height};
  spec.kind = static_cast<bt::FixtureKind>(kind);
  spec.impulse_channel = impulse_channel;
  spec.random_seed = seed;
  spec.options = {options3[0], options3[1], options3[2]};
  const bt::FixturePair pair = bt::MakeFixture(spec);
  for (size_t c = 0; c < 3; ++c) {
    for (size_t y = 0; y < height; ++y) {
      for (size_t x = 0; x < width; ++x) {
        reference[(c * height + y) * width + x] =
          pair.reference.planes()[c][y * pair.reference.stride() + x];
        distorted[(c * height + y) * width + x] =
          pair.distorted.planes()[c][y * pair.distorted.stride() + x];
      }
    }
  }
  return 0;
}

GJXL_REF_API int gjxl_ref_butteraugli_golden_full_map(size_t index, uint32_t* map_bits,
                                                      uint64_t* score_bits) {
  namespace golden = gjxl::butteraugli_test::golden;
  if (index >= golden::kFullMapCount) return -1;
  std::memcpy(map_bits, golden::kFullMapBits[index].data(), golden::kFullMapArea * 4);
  *score_bits = golden::kFullMapScoreBits[index];
  return static_cast<int>(golden::kFullMapArea);
}

// Butteraugli with explicit options (hf_asymmetry, x_multiplier, intensity).
GJXL_REF_API int gjxl_ref_butteraugli_options(const float* reference_linear,
                                              const float* distorted_linear, size_t width,
                                              size_t height, const float* options3,
                                              float* distance_map, double* score) {
  ButteraugliOptions options;
  options.hf_asymmetry = options3[0];
  options.x_multiplier = options3[1];
  options.intensity_target = options3[2];
  Status status = ComputeButteraugliDistance(
    ConstPlanar(reference_linear, width, height), ConstPlanar(distorted_linear, width, height),
    options, {distance_map, {width, height}, width}, score);
  return status.ok() ? 0 : Fail(status);
}

// codec/quantization_pipeline.cpp RunCpuQuantizationPipeline with the
// settings the reference workflow uses for an ordinary effort-`effort`
// Butteraugli-target encode (src/codestream/workflow.cpp:885-945,
// workflow_internal.h:17-130): Gaborish on, spatial initial field, adjusted
// shared AC quantization, prediction-aware DC with one extra bit and the
// weighted predictor, adaptive DC smoothing, fast final CfL, neutral EPF
// sharpness, and the given quantization-matrix scales.
struct RefPipelineOutputs {
  float* initial_quant;        // blocks
  float* strategy_mask;        // blocks
  float* pixel_mask;           // padded pixels
  float* final_quant;          // blocks
  float* block_distance;       // blocks
  float* reconstructed;        // 3 x width x height
  uint8_t* cells;              // blocks
  int32_t* raw_quant;          // blocks
  uint32_t* quantizer_params;  // global_scale, quant_dc
  int8_t* y_to_x;              // tiles
  int8_t* y_to_b;              // tiles
  int32_t* quantized_dc;       // 3 x blocks
  float* dc;                   // 3 x blocks
  int32_t* ac;                 // group order: per group 3 x used count
  size_t* group_used;          // per group used coefficient count
  double* score_history;       // iterations + 1
};

// Token request for the frame the pipeline produced: the coefficient orders
// (codestream/coefficient_order.cpp ComputeSimpleCoefficientOrdersForEncoder;
// order_mode 0 = natural scans, 1 = full counts, 2 = effort-7 sampled DCT8),
// then TokenizeSimpleAcGroupForEncoder (codestream/ac_group.cpp:1245) for every
// group with the given block-context map, collecting fixed populations.
struct RefTokenRequest {
  const uint32_t* qf_thresholds;   // threshold_count entries
  size_t threshold_count;
  const uint8_t* context_map;      // 3 * 13 * (threshold_count + 1)
  uint32_t num_contexts;
  int order_mode;
  uint32_t* orders;                // [13][3][1024]: scan used per family/channel
  uint32_t* used_order_mask;
  size_t* group_tokens;            // per group token count
  uint32_t* values;                // capacity entries, groups back to back
  uint16_t* contexts;
  size_t capacity;
  uint32_t* histogram;             // [num_contexts * 495][128] symbol counts
  int fixed_dct8;                  // pipeline option: DCT8 everywhere
};

static int RunPipeline(
  const float* linear, size_t width, size_t height, const float* opsin, size_t padded_width,
  size_t padded_height, float target, int effort, int x_qm_scale, int b_qm_scale,
  RefPipelineOutputs* out, const RefTokenRequest* tokens) {
  const Extent2D blocks{padded_width / 8, padded_height / 8};
  const Extent2D pixels{padded_width, padded_height};
  CpuQuantizationPipelineOptions options;
  options.butteraugli_target = target;
  options.uniform_initial_quantization = false;
  options.fixed_dct8 = tokens != nullptr && tokens->fixed_dct8 != 0;
  options.dense_dct32_search = effort == 10;
  auto& aq = options.adaptive_quantization;
  aq.profile.loop_filter.gaborish = true;
  aq.iterations = effort <= 5 ? 0 : effort == 6 ? 1 : effort == 7 ? 2 : effort == 8 ? 3 : 4;
  aq.coefficient_decision_mode = AcCoefficientDecisionMode::kAdjustedSharedQuant;
  aq.dc_quantization = DcQuantizationMode::kPredictionAware;
  aq.dc_prediction = VarDctDcPrediction::kWeighted;
  aq.profile.extra_dc_precision = 1;
  aq.profile.adaptive_dc_smoothing = true;
  aq.profile.x_qm_scale = static_cast<uint8_t>(x_qm_scale);
  aq.profile.b_qm_scale = static_cast<uint8_t>(b_qm_scale);
  aq.search_epf_sharpness = false;

  std::optional<thread_budget_internal::EncodeScope> budget;
  if (g_threads != 0) budget.emplace(g_threads);
  std::vector<double> history;
  VarDctEncoderFrame frame;
  MaximumErrorResult max_error;
  resource_budget_internal::PublicationVector<double> scores;
  CpuQuantizationPipelineOutput output{
    .initial_quantization = {
      .quant_field = {out->initial_quant, blocks, blocks.width},
      .strategy_mask = {out->strategy_mask, blocks, blocks.width},
      .pixel_mask = {out->pixel_mask, pixels, pixels.width},
    },
    .adaptive_quantization = {
      .quant_field = {out->final_quant, blocks, blocks.width},
      .block_distance_map = {out->block_distance, blocks, blocks.width},
      .reconstructed_linear_rgb = Planar(out->reconstructed, width, height),
      .frame = &frame,
      .score_history = &scores,
      .maximum_error_result = &max_error,
    },
  };
  Status status = RunCpuQuantizationPipeline(ConstPlanar(linear, width, height),
                                             ConstPlanar(opsin, padded_width, padded_height),
                                             options, output);
  if (!status.ok()) return Fail(status);
  status = ExportGrid(frame.strategies(), out->cells);
  if (!status.ok()) return Fail(status);
  const ConstPlaneI32View raw = frame.raw_quant_field();
  for (size_t y = 0; y < blocks.height; ++y)
    std::memcpy(out->raw_quant + y * blocks.width, raw.Row(y), blocks.width * 4);
  out->quantizer_params[0] = frame.quantizer().params().global_scale;
  out->quantizer_params[1] = frame.quantizer().params().quant_dc;
  ExportColorCorrelation(frame.color_correlation(), out->y_to_x, out->y_to_b);
  const ConstImage3I32View qdc = frame.quantized_dc();
  const ConstImage3FView dc = frame.dc();
  for (size_t c = 0; c < 3; ++c) {
    for (size_t y = 0; y < blocks.height; ++y) {
      std::memcpy(out->quantized_dc + (c * blocks.height + y) * blocks.width,
                  qdc.plane[c].Row(y), blocks.width * 4);
      std::memcpy(out->dc + (c * blocks.height + y) * blocks.width, dc.plane[c].Row(y),
                  blocks.width * 4);
    }
  }
  size_t offset = 0;
  for (size_t g = 0; g < frame.ac_group_count(); ++g) {
    VarDctAcGroupView group;
    status = frame.GetAcGroup(g, &group);
    if (!status.ok()) return Fail(status);
    out->group_used[g] = group.used_coefficient_count;
    for (size_t c = 0; c < 3; ++c) {
      std::memcpy(out->ac + offset, group.coefficients[c].data(),
                  group.used_coefficient_count * 4);
      offset += group.used_coefficient_count;
    }
  }
  for (size_t i = 0; i < scores.size(); ++i) out->score_history[i] = scores[i];
  if (tokens == nullptr) return 0;

  SimpleCoefficientOrders orders;
  if (tokens->order_mode != 0) {
    status = codestream_internal::ComputeSimpleCoefficientOrdersForEncoder(
      vardct_frame_internal::BorrowFrame(frame),
      tokens->order_mode == 2 ? VarDctCoefficientOrderBehavior::kEffort7Dct8Sampled
                              : VarDctCoefficientOrderBehavior::kFull,
      &orders);
    if (!status.ok()) return Fail(status);
  }
  codestream_internal::SimpleAcNaturalOrders natural;
  status = codestream_internal::PrepareSimpleAcNaturalOrders(&natural);
  if (!status.ok()) return Fail(status);
  *tokens->used_order_mask = orders.used_order_mask;
  // Scan per order family and channel: custom where used, else the natural
  // scan of the family's representative strategy.
  const AcStrategyType representative[13] = {
    AcStrategyType::kDct8, AcStrategyType::kCount, AcStrategyType::kDct16x16,
    AcStrategyType::kDct32x32, AcStrategyType::kDct16x8, AcStrategyType::kCount,
    AcStrategyType::kDct32x16, AcStrategyType::kCount, AcStrategyType::kCount,
    AcStrategyType::kCount, AcStrategyType::kCount, AcStrategyType::kCount,
    AcStrategyType::kCount};
  for (size_t family = 0; family < 13; ++family) {
    for (size_t c = 0; c < 3; ++c) {
      uint32_t* dst = tokens->orders + (family * 3 + c) * 1024;
      if (orders.used_order_mask & (1u << family)) {
        const auto& o = orders.orders[family][c];
        std::copy(o.begin(), o.end(), dst);
      } else if (representative[family] != AcStrategyType::kCount) {
        const auto& o = natural.orders[static_cast<size_t>(representative[family])];
        std::copy(o.begin(), o.end(), dst);
      }
    }
  }
  SimpleBlockContextMap map;
  map.qf_thresholds.assign(tokens->qf_thresholds, tokens->qf_thresholds + tokens->threshold_count);
  map.context_map.assign(tokens->context_map,
                         tokens->context_map + 3 * 13 * (tokens->threshold_count + 1));
  map.num_contexts = static_cast<uint8_t>(tokens->num_contexts);
  const auto view = vardct_frame_internal::BorrowFrame(frame);
  codestream_internal::SimpleAcTokenizationScratch scratch;
  size_t written = 0;
  for (size_t g = 0; g < frame.ac_group_count(); ++g) {
    codestream_internal::SimpleAcGroupTokenData data;
    status = codestream_internal::TokenizeSimpleAcGroupForEncoder(
      view, orders, natural, map, g, /*collect_fixed_populations=*/true, &scratch, &data);
    if (!status.ok()) return Fail(status);
    if (written + data.values.size() > tokens->capacity) {
      g_last_error = "token capacity exceeded";
      return -1;
    }
    std::copy(data.values.begin(), data.values.end(), tokens->values + written);
    std::copy(data.contexts.begin(), data.contexts.end(), tokens->contexts + written);
    tokens->group_tokens[g] = data.values.size();
    written += data.values.size();
    for (const auto& population : data.context_populations) {
      for (size_t k = 0; k < population.symbol_count; ++k) {
        const auto& symbol = data.symbol_populations[population.symbol_offset + k];
        tokens->histogram[static_cast<size_t>(population.context) * 128 + symbol.symbol] +=
          symbol.count;
      }
    }
  }
  return 0;
}

GJXL_REF_API int gjxl_ref_quantization_pipeline(
  const float* linear, size_t width, size_t height, const float* opsin, size_t padded_width,
  size_t padded_height, float target, int effort, int x_qm_scale, int b_qm_scale,
  RefPipelineOutputs* out) {
  return RunPipeline(linear, width, height, opsin, padded_width, padded_height, target, effort,
                     x_qm_scale, b_qm_scale, out, nullptr);
}

GJXL_REF_API int gjxl_ref_pipeline_tokens(
  const float* linear, size_t width, size_t height, const float* opsin, size_t padded_width,
  size_t padded_height, float target, int effort, int x_qm_scale, int b_qm_scale,
  RefPipelineOutputs* out, const RefTokenRequest* tokens) {
  return RunPipeline(linear, width, height, opsin, padded_width, padded_height, target, effort,
                     x_qm_scale, b_qm_scale, out, tokens);
}


// codestream/workflow.cpp:1318 ComputeQuantizationMatrixScaleStatsFromFiniteOpsin
// over the unpadded width x height region of the padded opsin image, as the
// workflow calls it (workflow.cpp:719-724, cropped_view of the frame).
// Writes {x_edge, b_edge, exposed_blue}.
GJXL_REF_API int gjxl_ref_matrix_scale_stats(const float* opsin, size_t padded_width,
                                             size_t padded_height, size_t width,
                                             size_t height, float* stats) {
  ConstImage3FView view;
  for (size_t c = 0; c < 3; ++c) {
    view.plane[c] = {opsin + c * padded_width * padded_height, {width, height},
                     padded_width};
  }
  codestream_internal::QuantizationMatrixScaleStats out;
  Status status =
    codestream_internal::ComputeQuantizationMatrixScaleStatsFromFiniteOpsin(view, &out);
  if (!status.ok()) return Fail(status);
  stats[0] = out.x_edge;
  stats[1] = out.b_edge;
  stats[2] = out.exposed_blue;
  return 0;
}

// codestream/workflow.cpp:1435 SelectQuantizationMatrixScales for a
// Butteraugli-target encode. Writes {x, b}.
GJXL_REF_API int gjxl_ref_select_matrix_scales(const float* stats, float target,
                                               int* scales) {
  codestream_internal::QuantizationMatrixScaleStats in;
  in.x_edge = stats[0];
  in.b_edge = stats[1];
  in.exposed_blue = stats[2];
  codestream_internal::QuantizationMatrixScales out;
  Status status = codestream_internal::SelectQuantizationMatrixScales(
    in, VarDctRateControlMode::kButteraugliTarget, target, &out);
  if (!status.ok()) return Fail(status);
  scales[0] = out.x;
  scales[1] = out.b;
  return 0;
}

// The whole reference encode on the CPU backend
// (codestream/workflow.h:281 EncodeLinearRgbVarDctCodestream): analysis,
// tokenization, entropy coding and bitstream assembly. Writes the codestream
// into `out` (capacity bytes), its size into *size and the final Butteraugli
// score into *score. Returns -2 when the capacity is too small.
GJXL_REF_API int gjxl_ref_encode_cpu(const float* linear, size_t width, size_t height,
                                     float target, int effort, uint8_t* out,
                                     size_t capacity, size_t* size, double* score) {
  VarDctEncodingOptions options;
  options.butteraugli_target = target;
  options.effort = effort;
  options.backend = VarDctBackendPreference::kCpu;
  options.cpu_thread_count = g_threads;
  std::vector<uint8_t> bytes;
  VarDctEncodingSummary summary;
  Status status = EncodeLinearRgbVarDctCodestream(ConstPlanar(linear, width, height), options,
                                                  &bytes, &summary);
  if (!status.ok()) return Fail(status);
  *size = bytes.size();
  *score = summary.score_history.empty() ? 0.0 : summary.score_history.back();
  if (bytes.size() > capacity) {
    g_last_error = "codestream capacity exceeded";
    return -2;
  }
  std::memcpy(out, bytes.data(), bytes.size());
  return 0;
}

// The reference's whole CPU encode under target-size rate control
// (VarDctRateControlMode::kTargetBytes: the bounded search of
// src/codestream/rate_control.cpp over complete encodes, workflow.cpp:1686).
// Writes the selected codestream, its Butteraugli target, the attempt count
// and whether the size met the tolerance.
GJXL_REF_API int gjxl_ref_encode_cpu_target_size(const float* linear, size_t width,
                                                 size_t height, size_t target_bytes,
                                                 double tolerance, size_t maximum_attempts,
                                                 int effort, uint8_t* out, size_t capacity,
                                                 size_t* size, float* selected_target,
                                                 size_t* attempts, int* target_met) {
  VarDctEncodingOptions options;
  options.effort = effort;
  options.backend = VarDctBackendPreference::kCpu;
  options.cpu_thread_count = g_threads;
  options.rate_control_mode = VarDctRateControlMode::kTargetBytes;
  options.target_bytes = target_bytes;
  options.target_size_tolerance = tolerance;
  options.target_size_maximum_attempts = maximum_attempts;
  std::vector<uint8_t> bytes;
  VarDctEncodingSummary summary;
  Status status = EncodeLinearRgbVarDctCodestream(ConstPlanar(linear, width, height), options,
                                                  &bytes, &summary);
  if (!status.ok()) return Fail(status);
  *size = bytes.size();
  *selected_target = summary.selected_butteraugli_target;
  *attempts = summary.encode_attempt_count;
  *target_met = summary.target_size_met ? 1 : 0;
  if (bytes.size() > capacity) {
    g_last_error = "codestream capacity exceeded";
    return -2;
  }
  std::memcpy(out, bytes.data(), bytes.size());
  return 0;
}

// DC-group token streams of a frame (codestream/vardct/dc_group.cpp:469-546,
// TokenizeSimpleDcGroupsForEncoder): every 256x256-block group in row-major
// order, its DC residual tokens (TokenizeWeightedDcGroup for prediction 1,
// TokenizeSimpleDcGroup for 0) and its AC-metadata tokens
// (TokenizeSimpleAcMetadata) over the same slices the encoder takes.
// Inputs: quantized DC as 3 planes of blocks_x x blocks_y (X, Y, B), the
// encoded strategy cells ((strategy << 1) | anchor), raw quant field, EPF
// sharpness, and the y_to_x / y_to_b maps (ceil(blocks/8) per side).
// Outputs, tokens as (context, value) pairs: all groups' DC tokens in group
// order into dc_out, all metadata tokens into meta_out, and per group
// {dc_offset, dc_count, meta_offset, meta_count, anchor_count}.
GJXL_REF_API int gjxl_ref_dc_group_tokens(const int32_t* quantized_dc, const uint8_t* cells,
                                          const int32_t* raw_quant, const uint8_t* sharpness,
                                          const int8_t* y_to_x, const int8_t* y_to_b,
                                          size_t blocks_x, size_t blocks_y, int prediction,
                                          uint32_t* dc_out, size_t dc_capacity,
                                          uint32_t* meta_out, size_t meta_capacity,
                                          uint32_t* group_info) {
  const Extent2D blocks{blocks_x, blocks_y};
  AcStrategyGrid grid;
  Status status = AcStrategyGrid::CreateFromEncodedCells(
    blocks, std::span<const uint8_t>(cells, blocks_x * blocks_y), &grid);
  if (!status.ok()) return Fail(status);
  const size_t tiles_x = (blocks_x + 7) / 8, tiles_y = (blocks_y + 7) / 8;
  const size_t pitch = blocks_x * blocks_y;
  const size_t groups_x = (blocks_x + 255) / 256, groups_y = (blocks_y + 255) / 256;
  size_t dc_used = 0, meta_used = 0;
  for (size_t gy = 0; gy < groups_y; ++gy) {
    for (size_t gx = 0; gx < groups_x; ++gx) {
      const size_t bx = gx * 256, by = gy * 256;
      const Extent2D extent{std::min<size_t>(256, blocks_x - bx),
                            std::min<size_t>(256, blocks_y - by)};
      ConstImage3I32View dc;
      for (size_t c = 0; c < 3; ++c)
        dc.plane[c] = {quantized_dc + c * pitch + by * blocks_x + bx, extent, blocks_x};
      codestream_internal::Storage<EntropyToken> dc_tokens, meta_tokens;
      status = prediction == 1 ? codestream_internal::TokenizeWeightedDcGroup(dc, &dc_tokens)
                               : TokenizeSimpleDcGroup(dc, &dc_tokens);
      if (!status.ok()) return Fail(status);
      const Extent2D tile_extent{(extent.width + 7) / 8, (extent.height + 7) / 8};
      const size_t tx = bx / 8, ty = by / 8;
      const SimpleAcMetadataInput metadata{
        .y_to_x_map = {y_to_x + ty * tiles_x + tx, tile_extent, tiles_x},
        .y_to_b_map = {y_to_b + ty * tiles_x + tx, tile_extent, tiles_x},
        .strategies = &grid,
        .block_x = bx,
        .block_y = by,
        .raw_quant_field = {raw_quant + by * blocks_x + bx, extent, blocks_x},
        .epf_sharpness = {sharpness + by * blocks_x + bx, extent, blocks_x},
      };
      size_t anchors = 0;
      status = TokenizeSimpleAcMetadata(metadata, &meta_tokens, &anchors);
      if (!status.ok()) return Fail(status);
      if (dc_used + dc_tokens.size() > dc_capacity ||
          meta_used + meta_tokens.size() > meta_capacity) {
        g_last_error = "token capacity exceeded";
        return -2;
      }
      uint32_t* info = group_info + 5 * (gy * groups_x + gx);
      info[0] = static_cast<uint32_t>(dc_used);
      info[1] = static_cast<uint32_t>(dc_tokens.size());
      info[2] = static_cast<uint32_t>(meta_used);
      info[3] = static_cast<uint32_t>(meta_tokens.size());
      info[4] = static_cast<uint32_t>(anchors);
      for (const EntropyToken& t : dc_tokens) {
        dc_out[2 * dc_used] = t.context;
        dc_out[2 * dc_used + 1] = t.value;
        ++dc_used;
      }
      for (const EntropyToken& t : meta_tokens) {
        meta_out[2 * meta_used] = t.context;
        meta_out[2 * meta_used + 1] = t.value;
        ++meta_used;
      }
    }
  }
  (void)tiles_y;
  return 0;
}

// EncodeHybridUint (codestream/entropy.cpp) with the given configuration:
// writes {symbol, extra_bit_count, extra_bits} per value.
GJXL_REF_API int gjxl_ref_hybrid_uint(const uint32_t* values, size_t count, int split_exponent,
                                      int msb_in_token, int lsb_in_token, uint32_t* out) {
  const HybridUintConfig config{static_cast<uint8_t>(split_exponent),
                                static_cast<uint8_t>(msb_in_token),
                                static_cast<uint8_t>(lsb_in_token)};
  for (size_t i = 0; i < count; ++i) {
    HybridUintToken token;
    Status status = EncodeHybridUint(values[i], config, &token);
    if (!status.ok()) return Fail(status);
    out[3 * i] = token.symbol;
    out[3 * i + 1] = token.extra_bit_count;
    out[3 * i + 2] = token.extra_bits;
  }
  return 0;
}

// ---- Entropy-coded sections: the reference's model builders, section
// writers and bit counters over split (value, context) token streams.

namespace {

std::vector<EntropyTokenStreamView> SplitSections(const uint32_t* values,
                                                  const uint16_t* contexts,
                                                  const uint32_t* offsets, size_t count) {
  std::vector<EntropyTokenStreamView> views;
  views.reserve(count);
  for (size_t s = 0; s < count; ++s) {
    const size_t begin = offsets[s], n = offsets[s + 1] - offsets[s];
    views.push_back(EntropyTokenStreamView::Split({values + begin, n}, {contexts + begin, n}));
  }
  return views;
}

}  // namespace

// Builds an EntropyCode over the sections: kind 0 the fast prefix code
// (OptimizeFastPrefixEntropyCode), 1/2/3 direct ANS in the balanced,
// high-density and rate-optimized modes (OptimizeDirectAnsEntropyCode) with
// at most `max_clusters` clusters.
GJXL_REF_API int gjxl_ref_entropy_build(int kind, const uint32_t* values,
                                        const uint16_t* contexts, const uint32_t* offsets,
                                        size_t count, uint32_t context_count,
                                        uint32_t max_clusters, void** handle) {
  if (handle == nullptr || offsets == nullptr || count == 0 || kind < 0 || kind > 3) {
    return Fail(Status::InvalidArgument("entropy_build: invalid arguments"));
  }
  const auto views = SplitSections(values, contexts, offsets, count);
  EntropyCodeOptions options;
  options.context_count = context_count;
  options.maximum_ans_clusters = max_clusters;
  auto code = std::make_unique<EntropyCode>();
  Status status = Status::Ok();
  if (kind == 0) {
    status = codestream_internal::OptimizeFastPrefixEntropyCode(views, options, code.get());
  } else {
    const auto mode = kind == 1 ? codestream_internal::DirectAnsEntropyMode::kBalanced
                      : kind == 2 ? codestream_internal::DirectAnsEntropyMode::kHighDensity
                                  : codestream_internal::DirectAnsEntropyMode::kRateOptimized;
    status = codestream_internal::OptimizeDirectAnsEntropyCode(views, options, mode, code.get());
  }
  if (!status.ok()) return Fail(status);
  *handle = code.release();
  return 0;
}

GJXL_REF_API void gjxl_ref_entropy_free(void* handle) {
  delete static_cast<EntropyCode*>(handle);
}

// mode (0 prefix, 1 ANS), context and cluster counts of a built code.
GJXL_REF_API int gjxl_ref_entropy_info(void* handle, int* mode, uint32_t* context_count,
                                       uint32_t* cluster_count) {
  const auto& code = *static_cast<const EntropyCode*>(handle);
  *mode = code.mode == EntropyCodingMode::kAns ? 1 : 0;
  *context_count = code.context_count;
  *cluster_count = static_cast<uint32_t>(code.mode == EntropyCodingMode::kAns
                                           ? code.ans_histograms.size()
                                           : code.prefix_codes.size());
  return 0;
}

// The code flattened: context map, HybridUint configs (3 bytes per
// cluster), prefix depths/bits [cluster][128] and degenerate symbols, ANS
// frequencies/reverse offsets [cluster][256] and reverse maps
// [cluster][4096] (absent entries zero).
GJXL_REF_API int gjxl_ref_entropy_tables(void* handle, uint8_t* context_map, uint8_t* configs,
                                         uint8_t* depths, uint16_t* bits, uint16_t* degenerate,
                                         uint16_t* frequencies, uint16_t* reverse_offsets,
                                         uint16_t* reverse_map) {
  const auto& code = *static_cast<const EntropyCode*>(handle);
  std::copy(code.context_map.begin(), code.context_map.end(), context_map);
  for (size_t c = 0; c < code.uint_configs.size(); ++c) {
    configs[3 * c] = code.uint_configs[c].split_exponent;
    configs[3 * c + 1] = code.uint_configs[c].msb_in_token;
    configs[3 * c + 2] = code.uint_configs[c].lsb_in_token;
  }
  if (code.mode == EntropyCodingMode::kAns) {
    for (size_t c = 0; c < code.ans_histograms.size(); ++c) {
      const AnsHistogram& h = code.ans_histograms[c];
      std::fill_n(frequencies + 256 * c, 256, uint16_t{0});
      std::fill_n(reverse_offsets + 256 * c, 256, uint16_t{0});
      std::fill_n(reverse_map + 4096 * c, 4096, uint16_t{0});
      std::copy(h.frequencies.begin(), h.frequencies.end(), frequencies + 256 * c);
      std::copy(h.reverse_offsets.begin(), h.reverse_offsets.end(), reverse_offsets + 256 * c);
      std::copy(h.reverse_map.begin(), h.reverse_map.end(), reverse_map + 4096 * c);
    }
  } else {
    for (size_t c = 0; c < code.prefix_codes.size(); ++c) {
      const PrefixCode& p = code.prefix_codes[c];
      std::copy(p.depths.begin(), p.depths.end(), depths + 128 * c);
      std::copy(p.bits.begin(), p.bits.end(), bits + 128 * c);
      degenerate[c] = p.degenerate_symbol;
    }
  }
  return 0;
}

// Every section written by WriteValidatedTokenStream into its own
// BitWriter (as WriteAcSections does): bits_written per section, the padded
// bytes concatenated into `out`, and each section's first byte.
GJXL_REF_API int gjxl_ref_entropy_write(void* handle, const uint32_t* values,
                                        const uint16_t* contexts, const uint32_t* offsets,
                                        size_t count, uint8_t* out, size_t capacity,
                                        uint64_t* bit_counts, uint64_t* byte_offsets) {
  const auto& code = *static_cast<const EntropyCode*>(handle);
  const auto views = SplitSections(values, contexts, offsets, count);
  size_t at = 0;
  for (size_t s = 0; s < count; ++s) {
    BitWriter writer;
    Status status = codestream_internal::WriteValidatedTokenStream(views[s], code, &writer);
    if (!status.ok()) return Fail(status);
    const auto bytes = writer.padded_bytes();
    if (at + bytes.size() > capacity) {
      return Fail(Status::InvalidArgument("entropy_write: output too small"));
    }
    std::copy(bytes.begin(), bytes.end(), out + at);
    byte_offsets[s] = at;
    bit_counts[s] = writer.bits_written();
    at += bytes.size();
  }
  byte_offsets[count] = at;
  return 0;
}

// Exact token bits per section: CountAnsTokenStreamBits for ANS,
// CountTokenStreamBits for prefix codes.
GJXL_REF_API int gjxl_ref_entropy_count(void* handle, const uint32_t* values,
                                        const uint16_t* contexts, const uint32_t* offsets,
                                        size_t count, uint64_t* bit_counts) {
  const auto& code = *static_cast<const EntropyCode*>(handle);
  const auto views = SplitSections(values, contexts, offsets, count);
  for (size_t s = 0; s < count; ++s) {
    Status status = code.mode == EntropyCodingMode::kAns
                      ? codestream_internal::CountAnsTokenStreamBits(views[s], code, &bit_counts[s])
                      : codestream_internal::CountTokenStreamBits(views[s], code, &bit_counts[s]);
    if (!status.ok()) return Fail(status);
  }
  return 0;
}
