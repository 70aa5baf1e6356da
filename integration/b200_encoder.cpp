// The binding a maintainer adds to the gjxl encoder to run its analysis half
// on a B200 through libgjxl_b200, with the encoder's own CPU back half
// (block-context and coefficient-order selection, DC tokenization, entropy
// coding, bitstream assembly) left unchanged.
//
// It is compiled against the reference's headers and linked with the
// reference's own codestream and codec sources (integration/Makefile), as it
// would be inside the reference tree. Three pieces:
//
//  * ResolveEncodeOptions: the workflow's option resolution for one ordinary
//    Butteraugli-target encode attempt (EncodePreparedAttempt,
//    src/codestream/workflow.cpp:886-921 and :1069-1076), through the
//    reference's own policy helpers, so the frame profile and serializer
//    options are exactly the ones the CPU path would use.
//  * AssembleB200Frame: a VarDctEncoderFrame from a session's results
//    (strategy cells, raw quant field, quantizer, final CfL maps, quantized DC
//    and AC), through the reference's AssembleVarDctEncoderFrame
//    (src/codec/vardct_frame_internal.h:59), as the reference's CUDA path
//    does with its readbacks (src/gpu/cuda/cuda_aq_resident.cpp:2785-2830).
//  * B200AcTokenizer: an AcTokenizationProvider
//    (src/codestream/ac_tokenization_provider_internal.h:20-31) that
//    tokenizes the frame's AC on the device with gjxl_b200_ac_tokenize for the
//    block-context map and coefficient orders the serializer chose, checks the
//    device's scans against the serializer's, and hands back split token
//    streams and the fixed-ANS populations.
//
//  * DeviceEntropyCode / WriteAcSectionsOnDevice: an EntropyCode the
//    serializer built, flattened into device tables, and the per-group body
//    of WriteAcSections (src/codestream/vardct/encoder.cpp:756-775) run on the
//    device by gjxl_b200_entropy_write_sections: every AC group's section,
//    byte for byte as WriteValidatedTokenStream writes it, without the token
//    streams coming back to the host.
//
// The C entry point gjxl_b200_encode_image runs a session on packed 8-bit
// sRGB, assembles the frame, validates it (ValidateSimpleCodestreamFrame,
// src/codec/codestream.h:87) and writes the codestream with
// EncodeVarDctCodestreamToBuffer (src/codestream/encoder_internal.h:168).

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <span>
#include <string>
#include <vector>

#include "codec/codestream.h"
#include "codec/epf.h"
#include "codec/vardct_frame.h"
#include "codec/vardct_frame_internal.h"
#include "codec/vardct_frame_view_internal.h"
#include "codestream/ac_tokenization_provider_internal.h"
#include "codestream/ans_internal.h"
#include "codestream/bit_writer.h"
#include "codestream/entropy_internal.h"
#include "codestream/encoder_internal.h"
#include "codestream/rate_control_internal.h"
#include "codestream/workflow.h"
#include "codestream/workflow_internal.h"
#include "core/ac_strategy.h"
#include "core/frame_geometry.h"
#include "core/quantizer.h"
#include "gjxl_b200.h"

#define GJXL_INTEGRATION_API extern "C" __attribute__((visibility("default")))

namespace gjxl::b200_integration {
namespace {

thread_local std::string g_last_error;

int Fail(const Status& status) {
  g_last_error = std::string(status.message());
  const int code = static_cast<int>(status.code());
  return code == 0 ? 8 : code;
}

Status FromB200(int code, const char* what) {
  if (code == GJXL_B200_OK) return Status::Ok();
  const std::string message = std::string(what) + ": " + gjxl_b200_last_error();
  switch (code) {
    case GJXL_B200_INVALID_ARGUMENT: return Status::InvalidArgument(message);
    case GJXL_B200_UNSUPPORTED: return Status::Unsupported(message);
    case GJXL_B200_UNAVAILABLE: return Status::Unavailable(message);
    case GJXL_B200_OUT_OF_MEMORY: return Status::OutOfMemory(message);
    case GJXL_B200_FAILED_PRECONDITION: return Status::FailedPrecondition(message);
    case GJXL_B200_SUBMISSION_FAILED: return Status::SubmissionFailed(message);
    case GJXL_B200_DEVICE_ERROR: return Status::DeviceError(message);
    default: return Status::Internal(message);
  }
}

Status FromCuda(cudaError_t error, const char* what) {
  if (error == cudaSuccess) return Status::Ok();
  return Status::DeviceError(std::string(what) + ": " + cudaGetErrorString(error));
}

// The pieces of one encode attempt's options that the frame and the
// serializer depend on.
struct ResolvedEncode {
  CpuQuantizationPipelineOptions pipeline;
  VarDctCodestreamOptions codestream;
};

// EncodePreparedAttempt's resolution (src/codestream/workflow.cpp:886-921),
// through the reference's own helpers, for a Butteraugli-target encode.
Status ResolveEncodeOptions(const VarDctEncodingOptions& options,
                            const codestream_internal::QuantizationMatrixScaleStats& stats,
                            ResolvedEncode* out) {
  ResolvedEncode r;
  codestream_internal::ConfigureInitialQuantizationPolicy(options, &r.pipeline);
  r.pipeline.fixed_dct8 = codestream_internal::UseFixedDct8Strategy(options);
  r.pipeline.dense_dct32_search = codestream_internal::UseDenseDct32Search(options);
  r.pipeline.butteraugli_target = options.butteraugli_target;
  auto& aq = r.pipeline.adaptive_quantization;
  aq.iterations = codestream_internal::AdaptiveQuantizationIterations(options);
  aq.coefficient_decision_mode = codestream_internal::ResolveAcCoefficientDecision(options);
  aq.dc_quantization = ResolveDcQuantization(options);
  aq.dc_prediction = options.dc_prediction;
  aq.profile.extra_dc_precision =
    ResolveDcQuantization(options) == DcQuantizationMode::kPredictionAware ? 1 : 0;
  aq.profile.adaptive_dc_smoothing = ResolveAdaptiveDcSmoothing(options);
  codestream_internal::QuantizationMatrixScales scales;
  Status status = codestream_internal::SelectQuantizationMatrixScales(
    codestream_internal::ShouldComputeQuantizationMatrixScaleStats(options)
      ? stats : codestream_internal::QuantizationMatrixScaleStats{},
    options.rate_control_mode, options.butteraugli_target, &scales);
  if (!status.ok()) return status;
  aq.profile.x_qm_scale = scales.x;
  aq.profile.b_qm_scale = scales.b;
  r.codestream = VarDctCodestreamOptions{
    .entropy_behavior = codestream_internal::ResolveEntropyBehavior(options),
    .coefficient_order_behavior = codestream_internal::ResolveCoefficientOrderBehavior(options),
    .dc_prediction = options.dc_prediction,
    .dc_uint_search = codestream_internal::UseDcUintSearch(options),
  };
  *out = std::move(r);
  return Status::Ok();
}

// A session's results, read back to the host.
struct SessionResults {
  size_t width = 0, height = 0, pw = 0, ph = 0, bx = 0, by = 0, tx = 0, ty = 0;
  std::vector<uint8_t> cells;
  std::vector<int32_t> raw_quant;
  uint32_t global_scale = 0, quant_dc = 0;
  std::vector<int8_t> y_to_x, y_to_b;
  std::vector<int32_t> quantized_dc;  // X, Y, B planes of blocks
  std::vector<int32_t> quantized_ac;  // 3 padded planes, footprint layout
  std::array<int, 2> device_matrix_scales{};
  codestream_internal::QuantizationMatrixScaleStats stats;
};

Status ReadSession(const gjxl_b200_outputs& o, size_t width, size_t height,
                   SessionResults* out) {
  SessionResults r;
  r.width = width;
  r.height = height;
  r.pw = o.padded_width;
  r.ph = o.padded_height;
  r.bx = o.blocks_x;
  r.by = o.blocks_y;
  r.tx = o.tiles_x;
  r.ty = o.tiles_y;
  const size_t blocks = r.bx * r.by, tiles = r.tx * r.ty, plane = r.pw * r.ph;
  r.cells.assign(o.host_strategy_cells, o.host_strategy_cells + blocks);
  r.raw_quant.assign(o.host_raw_quant_field, o.host_raw_quant_field + blocks);
  r.global_scale = o.host_quantizer_params[0];
  r.quant_dc = o.host_quantizer_params[1];
  r.y_to_x.assign(o.host_y_to_x, o.host_y_to_x + tiles);
  r.y_to_b.assign(o.host_y_to_b, o.host_y_to_b + tiles);
  r.quantized_dc.assign(o.host_quantized_dc, o.host_quantized_dc + 3 * blocks);
  r.stats.x_edge = o.host_matrix_scale_stats[0];
  r.stats.b_edge = o.host_matrix_scale_stats[1];
  r.stats.exposed_blue = o.host_matrix_scale_stats[2];
  r.quantized_ac.resize(3 * plane);
  Status status = FromCuda(cudaMemcpy(r.quantized_ac.data(), o.quantized_ac,
                                      3 * plane * sizeof(int32_t), cudaMemcpyDeviceToHost),
                           "quantized AC readback");
  if (!status.ok()) return status;
  status = FromCuda(cudaMemcpy(r.device_matrix_scales.data(), o.matrix_scales,
                               2 * sizeof(int), cudaMemcpyDeviceToHost),
                    "matrix scale readback");
  if (!status.ok()) return status;
  *out = std::move(r);
  return Status::Ok();
}

// VarDctEncoderFrame from the session's results: the transforms in raster
// anchor order (AcStrategyGrid::ForEachAnchor), each channel's N coefficients
// gathered from their footprint (coefficient i at pixel
// (bx*8 + i % W, by*8 + i / W)) into one contiguous run.
Status AssembleB200Frame(const SessionResults& r, const SimpleVarDctCodestreamProfile& profile,
                         VarDctEncoderFrame* frame) {
  FrameGeometry geometry;
  Status status = FrameGeometry::Create({r.width, r.height}, &geometry);
  if (!status.ok()) return status;
  AcStrategyGrid grid;
  status = AcStrategyGrid::CreateFromEncodedCells({r.bx, r.by}, r.cells, &grid);
  if (!status.ok()) return status;
  Quantizer quantizer;
  status = Quantizer::Create({.global_scale = r.global_scale, .quant_dc = r.quant_dc},
                             &quantizer);
  if (!status.ok()) return status;
  std::vector<uint8_t> sharpness(r.bx * r.by);
  status = FillDefaultEpfSharpness({sharpness.data(), {r.bx, r.by}, r.bx});
  if (!status.ok()) return status;

  std::vector<int32_t> ac;
  ac.reserve(3 * r.pw * r.ph);
  std::vector<vardct_frame_internal::QuantizedAcTransformLayout> transforms;
  const size_t plane = r.pw * r.ph;
  status = grid.ForEachAnchor([&](size_t x, size_t y, AcStrategyType strategy) {
    const AcStrategyInfo* info = GetAcStrategyInfo(strategy);
    if (info == nullptr) return Status::InvalidArgument("unknown strategy in the grid");
    const size_t w = info->covered_blocks.width * 8, h = info->covered_blocks.height * 8;
    if ((x * 8 + w) > r.pw || (y * 8 + h) > r.ph) {
      return Status::InvalidArgument("transform footprint leaves the padded image");
    }
    vardct_frame_internal::QuantizedAcTransformLayout t;
    t.block_x = x;
    t.block_y = y;
    t.strategy = strategy;
    t.coefficient_count = w * h;
    for (size_t c = 0; c < 3; ++c) {
      t.coefficient_offsets[c] = ac.size();
      for (size_t row = 0; row < h; ++row) {
        const int32_t* src = r.quantized_ac.data() + c * plane + (y * 8 + row) * r.pw + x * 8;
        ac.insert(ac.end(), src, src + w);
      }
    }
    transforms.push_back(t);
    return Status::Ok();
  });
  if (!status.ok()) return status;

  ConstImage3I32View dc;
  for (size_t c = 0; c < 3; ++c) {
    dc.plane[c] = {r.quantized_dc.data() + c * r.bx * r.by, {r.bx, r.by}, r.bx};
  }
  status = vardct_frame_internal::AssembleVarDctEncoderFrame(
    vardct_frame_internal::QuantizedFrameAssemblyInput{
      .geometry = geometry,
      .strategies = &grid,
      .raw_quant_field = {r.raw_quant.data(), {r.bx, r.by}, r.bx},
      .quantizer = &quantizer,
      .y_to_x = {r.y_to_x.data(), {r.tx, r.ty}, r.tx},
      .y_to_b = {r.y_to_b.data(), {r.tx, r.ty}, r.tx},
      .epf_sharpness = {sharpness.data(), {r.bx, r.by}, r.bx},
      .profile = profile,
      .quantized_dc = dc,
      .quantized_ac = std::span<const int32_t>(ac.data(), ac.size()),
      .transforms = transforms,
      .reject_unwritten_coefficients = false,
    },
    frame);
  if (!status.ok()) return status;
  return ValidateSimpleCodestreamFrame(*frame);
}

// Scan order families of the simple codestream (coefficient_order.h) and the
// device tokenizer's order modes.
int OrderMode(VarDctCoefficientOrderBehavior behavior) {
  return behavior == VarDctCoefficientOrderBehavior::kEffort7Dct8Sampled ? 2 : 1;
}

// AC tokens of the session's frame computed on the device for the block
// context map and coefficient orders the serializer hands to Begin.
class B200AcTokenizer final : public codestream_internal::AcTokenizationProvider {
 public:
  B200AcTokenizer(const gjxl_b200_outputs& outputs, VarDctCoefficientOrderBehavior behavior)
      : o_(outputs), order_mode_(OrderMode(behavior)) {}

  ~B200AcTokenizer() override {
    if (tokens_ != nullptr) gjxl_b200_ac_tokens_destroy(tokens_);
    if (device_ != nullptr) cudaFree(device_);
  }

  // The serializer overlaps its DC tokenization with Begin..Finish.
  bool SupportsEarlyEntropy() const noexcept override { return false; }

  Status Begin(const vardct_frame_internal::VarDctFrameView& frame,
               const SimpleCoefficientOrders& orders,
               const codestream_internal::SimpleAcNaturalOrders& natural,
               const SimpleBlockContextMap& contexts, bool populations) override {
    (void)frame;
    (void)natural;
    if (contexts.num_contexts == 0 || contexts.num_contexts > 16 ||
        contexts.qf_thresholds.size() > 15 ||
        contexts.context_map.size() != 3 * 13 * (contexts.qf_thresholds.size() + 1)) {
      return Status::Unsupported("block-context map outside the device tokenizer's range");
    }
    std::memset(&map_, 0, sizeof(map_));
    map_.threshold_count = static_cast<uint32_t>(contexts.qf_thresholds.size());
    std::copy(contexts.qf_thresholds.begin(), contexts.qf_thresholds.end(), map_.qf_thresholds);
    map_.num_contexts = contexts.num_contexts;
    std::copy(contexts.context_map.begin(), contexts.context_map.end(), map_.context_map);
    context_count_ = contexts.ac_context_count();
    populations_ = populations;
    // Natural scans when the serializer chose no custom order.
    const int mode = orders.used_order_mask == 0 ? 0 : order_mode_;
    expected_used_mask_ = orders.used_order_mask;
    expected_orders_ = &orders;

    const size_t groups = o_.groups;
    capacity_ = gjxl_b200_ac_token_capacity(o_.blocks_x, o_.blocks_y);
    Status status = FromB200(gjxl_b200_ac_tokens_create(o_.blocks_x, o_.blocks_y, &tokens_),
                             "ac_tokens_create");
    if (!status.ok()) return status;
    const size_t histogram_words = context_count_ * 128;
    offsets_bytes_ = Align((groups + 1) * 4);
    const size_t bytes = capacity_ * 4 + Align(capacity_ * 2) + offsets_bytes_ +
                         histogram_words * 4 + 13 * 3 * 1024 * 4 + 16;
    status = FromCuda(cudaMalloc(&device_, Align(capacity_ * 4) + bytes), "token buffers");
    if (!status.ok()) return status;
    unsigned char* p = static_cast<unsigned char*>(device_);
    auto take = [&](size_t n) {
      unsigned char* r = p;
      p += Align(n);
      return r;
    };
    gjxl_b200_ac_token_outputs outs;
    std::memset(&outs, 0, sizeof(outs));
    outs.token_values = reinterpret_cast<uint32_t*>(take(capacity_ * 4));
    outs.token_contexts = reinterpret_cast<uint16_t*>(take(capacity_ * 2));
    outs.token_capacity = capacity_;
    outs.group_offsets = reinterpret_cast<uint32_t*>(take((groups + 1) * 4));
    outs.histogram = reinterpret_cast<uint32_t*>(take(histogram_words * 4));
    outs.orders = reinterpret_cast<uint32_t*>(take(13 * 3 * 1024 * 4));
    outs.used_order_mask = reinterpret_cast<uint32_t*>(take(4));
    outs.device_error = reinterpret_cast<uint32_t*>(take(4));
    outs_ = outs;
    status = FromCuda(cudaMemset(outs.device_error, 0, 4), "token error word");
    if (!status.ok()) return status;
    return FromB200(gjxl_b200_ac_tokenize(tokens_, o_.strategy_cells, o_.raw_quant_field,
                                          o_.quantized_ac, o_.padded_width,
                                          o_.padded_width * o_.padded_height, &map_, mode,
                                          &outs_, nullptr),
                    "ac_tokenize");
  }

  Status Finish(codestream_internal::Storage<EntropyTokenStreamView>* streams,
                codestream_internal::Storage<codestream_internal::PreparedFixedAnsCluster>*
                  populations) override {
    if (tokens_ == nullptr || streams == nullptr || populations == nullptr) {
      return Status::FailedPrecondition("Finish without a device tokenization");
    }
    Status status = FromB200(gjxl_b200_check_device_error(outs_.device_error, 1, nullptr),
                             "device tokenization");
    if (!status.ok()) return status;
    const size_t groups = o_.groups;
    std::vector<uint32_t> offsets(groups + 1);
    status = FromCuda(cudaMemcpy(offsets.data(), outs_.group_offsets, (groups + 1) * 4,
                                 cudaMemcpyDeviceToHost), "group offsets");
    if (!status.ok()) return status;
    const size_t total = offsets[groups];
    if (total > capacity_) return Status::Internal("device token count exceeds its capacity");
    values_.resize(total);
    contexts_.resize(total);
    status = FromCuda(cudaMemcpy(values_.data(), outs_.token_values, total * 4,
                                 cudaMemcpyDeviceToHost), "token values");
    if (status.ok()) {
      status = FromCuda(cudaMemcpy(contexts_.data(), outs_.token_contexts, total * 2,
                                   cudaMemcpyDeviceToHost), "token contexts");
    }
    if (!status.ok()) return status;
    // The device scans must be the serializer's (same counts, same sort).
    uint32_t used = 0;
    std::vector<uint32_t> scans(13 * 3 * 1024);
    status = FromCuda(cudaMemcpy(&used, outs_.used_order_mask, 4, cudaMemcpyDeviceToHost),
                      "used order mask");
    if (status.ok()) {
      status = FromCuda(cudaMemcpy(scans.data(), outs_.orders, scans.size() * 4,
                                   cudaMemcpyDeviceToHost), "scans");
    }
    if (!status.ok()) return status;
    if (used != expected_used_mask_) {
      return Status::Internal("device coefficient orders differ from the serializer's");
    }
    for (size_t family = 0; family < 13; ++family) {
      if (!(used & (1u << family))) continue;
      for (size_t c = 0; c < 3; ++c) {
        const auto& want = expected_orders_->orders[family][c];
        if (!std::equal(want.begin(), want.end(), scans.begin() + (family * 3 + c) * 1024)) {
          return Status::Internal("device coefficient scan differs from the serializer's");
        }
      }
    }
    codestream_internal::Storage<EntropyTokenStreamView> result;
    result.reserve(groups);
    for (size_t g = 0; g < groups; ++g) {
      const size_t begin = offsets[g], count = offsets[g + 1] - offsets[g];
      result.push_back(EntropyTokenStreamView::Split({values_.data() + begin, count},
                                                     {contexts_.data() + begin, count}));
    }
    codestream_internal::Storage<codestream_internal::PreparedFixedAnsCluster> reduced;
    if (populations_) {
      std::vector<uint32_t> histogram(context_count_ * 128);
      status = FromCuda(cudaMemcpy(histogram.data(), outs_.histogram, histogram.size() * 4,
                                   cudaMemcpyDeviceToHost), "token histogram");
      if (!status.ok()) return status;
      reduced.resize(context_count_);
      uint64_t counted = 0;
      for (size_t context = 0; context < context_count_; ++context) {
        auto& cluster = reduced[context];
        for (uint32_t symbol = 0; symbol < 128; ++symbol) {
          const uint64_t n = histogram[context * 128 + symbol];
          cluster.counts[symbol] = n;
          cluster.token_count += n;
          if (n != 0) cluster.maximum_symbol = symbol;
          // Hybrid-uint tokens from 16 up carry 2 + (token - 16) / 4 raw bits
          // (the default 4/2/0 split of the JPEG XL entropy coder).
          if (symbol >= 16) cluster.extra_bits += n * (2 + ((symbol - 16) >> 2));
        }
        counted += cluster.token_count;
      }
      if (counted != total) return Status::Internal("token populations differ from the count");
    }
    *streams = std::move(result);
    *populations = std::move(reduced);
    return Status::Ok();
  }

 private:
  static size_t Align(size_t n) { return (n + 255) / 256 * 256; }

  gjxl_b200_outputs o_;
  int order_mode_;
  gjxl_b200_block_context_map map_{};
  size_t context_count_ = 0;
  bool populations_ = false;
  uint16_t expected_used_mask_ = 0;
  const SimpleCoefficientOrders* expected_orders_ = nullptr;
  gjxl_b200_ac_tokens* tokens_ = nullptr;
  void* device_ = nullptr;
  size_t capacity_ = 0, offsets_bytes_ = 0;
  gjxl_b200_ac_token_outputs outs_{};
  std::vector<uint32_t> values_;
  std::vector<uint16_t> contexts_;
};

// One complete attempt on a prepared session: the analysis at the session's
// current target, the frame, and the unchanged serializer. Fills the summary
// fields a target-size search reads (rate_control.cpp:140-165).
Status EncodeWithSession(gjxl_b200_session* session, const uint8_t* pixels, size_t width,
                         size_t height, size_t row_stride, int channels, float target,
                         int effort, bool device_tokens, std::vector<uint8_t>* codestream,
                         VarDctEncodingSummary* summary) {
  VarDctEncodingOptions options;
  options.butteraugli_target = target;
  options.effort = effort;
  Status status = FromB200(gjxl_b200_session_set_butteraugli_target(session, target),
                           "session_set_butteraugli_target");
  if (!status.ok()) return status;
  status = FromB200(gjxl_b200_session_analyze_host(session, pixels, row_stride, channels,
                                                   nullptr),
                    "session_analyze_host");
  if (!status.ok()) return status;
  gjxl_b200_outputs o;
  status = FromB200(gjxl_b200_session_outputs(session, &o), "session_outputs");
  if (!status.ok()) return status;
  SessionResults results;
  status = ReadSession(o, width, height, &results);
  if (!status.ok()) return status;
  ResolvedEncode resolved;
  status = ResolveEncodeOptions(options, results.stats, &resolved);
  if (!status.ok()) return status;
  const auto& profile = resolved.pipeline.adaptive_quantization.profile;
  if (results.device_matrix_scales[0] != profile.x_qm_scale ||
      results.device_matrix_scales[1] != profile.b_qm_scale) {
    return Status::Internal("device quantization-matrix scales differ from the workflow's");
  }
  VarDctEncoderFrame frame;
  status = AssembleB200Frame(results, profile, &frame);
  if (!status.ok()) return status;
  std::unique_ptr<B200AcTokenizer> tokenizer;
  if (device_tokens) {
    tokenizer = std::make_unique<B200AcTokenizer>(o, resolved.codestream.coefficient_order_behavior);
  }
  codestream_internal::CodestreamBuffer buffer;
  {
    codestream_internal::AcTokenizationProviderScope scope(tokenizer.get());
    status = codestream_internal::EncodeVarDctCodestreamToBuffer(
      vardct_frame_internal::BorrowFrame(frame), resolved.codestream, &buffer);
  }
  if (!status.ok()) return status;
  codestream->assign(buffer.data(), buffer.data() + buffer.size());
  if (summary != nullptr) {
    *summary = VarDctEncodingSummary{};
    summary->extent = {width, height};
    summary->encoded_bytes = codestream->size();
    summary->rate_control_mode = VarDctRateControlMode::kButteraugliTarget;
    summary->selected_butteraugli_target = target;
    summary->score_history.assign(o.host_score_history,
                                  o.host_score_history + o.iterations + 1);
  }
  return Status::Ok();
}

// An EntropyCode's tables on the device (gjxl_b200_entropy_code): context
// map, HybridUint configurations and, per cluster, the prefix code (depths,
// bits, degenerate symbol) or the ANS histogram (frequencies, reverse-map
// offsets, reverse map) padded to 128 / 256 symbols and 4096 entries.
class DeviceEntropyCode {
 public:
  ~DeviceEntropyCode() {
    if (device_ != nullptr) cudaFree(device_);
  }

  Status Upload(const EntropyCode& code) {
    const bool ans = code.mode == EntropyCodingMode::kAns;
    const size_t clusters = ans ? code.ans_histograms.size() : code.prefix_codes.size();
    if (code.context_count == 0 || clusters == 0 || clusters > 256 ||
        code.uint_configs.size() != clusters || code.context_map.size() != code.context_count) {
      return Status::InvalidArgument("entropy code outside the device writer's range");
    }
    // One host image of all tables, 16-byte aligned pieces.
    const auto align = [](size_t n) { return (n + 15) / 16 * 16; };
    const size_t map_at = 0, config_at = align(code.context_count);
    const size_t a_at = config_at + align(3 * clusters);
    const size_t a_bytes = ans ? 256 * 2 * clusters : 128 * clusters;
    const size_t b_at = a_at + align(a_bytes);
    const size_t b_bytes = ans ? 256 * 2 * clusters : 128 * 2 * clusters;
    const size_t c_at = b_at + align(b_bytes);
    const size_t c_bytes = ans ? 4096 * 2 * clusters : 2 * clusters;
    const size_t total = c_at + align(c_bytes);
    std::vector<uint8_t> host(total, 0);
    std::copy(code.context_map.begin(), code.context_map.end(), host.begin() + map_at);
    for (size_t c = 0; c < clusters; ++c) {
      host[config_at + 3 * c] = code.uint_configs[c].split_exponent;
      host[config_at + 3 * c + 1] = code.uint_configs[c].msb_in_token;
      host[config_at + 3 * c + 2] = code.uint_configs[c].lsb_in_token;
    }
    auto* a16 = reinterpret_cast<uint16_t*>(host.data() + a_at);
    auto* b16 = reinterpret_cast<uint16_t*>(host.data() + b_at);
    auto* c16 = reinterpret_cast<uint16_t*>(host.data() + c_at);
    for (size_t c = 0; c < clusters; ++c) {
      if (ans) {
        const AnsHistogram& h = code.ans_histograms[c];
        if (h.frequencies.size() > 256 || h.reverse_map.size() > 4096) {
          return Status::InvalidArgument("ANS histogram outside the device writer's range");
        }
        std::copy(h.frequencies.begin(), h.frequencies.end(), a16 + 256 * c);
        std::copy(h.reverse_offsets.begin(), h.reverse_offsets.end(), b16 + 256 * c);
        std::copy(h.reverse_map.begin(), h.reverse_map.end(), c16 + 4096 * c);
      } else {
        const PrefixCode& pc = code.prefix_codes[c];
        std::copy(pc.depths.begin(), pc.depths.end(), host.begin() + a_at + 128 * c);
        std::copy(pc.bits.begin(), pc.bits.end(), b16 + 128 * c);
        c16[c] = pc.degenerate_symbol;
      }
    }
    Status status = FromCuda(cudaMalloc(&device_, total), "entropy tables");
    if (status.ok()) {
      status = FromCuda(cudaMemcpy(device_, host.data(), total, cudaMemcpyHostToDevice),
                        "entropy tables");
    }
    if (!status.ok()) return status;
    auto* d = static_cast<uint8_t*>(device_);
    std::memset(&view_, 0, sizeof(view_));
    view_.mode = ans ? GJXL_B200_ENTROPY_ANS : GJXL_B200_ENTROPY_PREFIX;
    view_.context_count = code.context_count;
    view_.cluster_count = static_cast<uint32_t>(clusters);
    view_.context_map = d + map_at;
    view_.uint_configs = d + config_at;
    if (ans) {
      view_.ans_frequencies = reinterpret_cast<const uint16_t*>(d + a_at);
      view_.ans_reverse_offsets = reinterpret_cast<const uint16_t*>(d + b_at);
      view_.ans_reverse_map = reinterpret_cast<const uint16_t*>(d + c_at);
    } else {
      view_.prefix_depths = d + a_at;
      view_.prefix_bits = reinterpret_cast<const uint16_t*>(d + b_at);
      view_.prefix_degenerate = reinterpret_cast<const uint16_t*>(d + c_at);
    }
    return Status::Ok();
  }

  const gjxl_b200_entropy_code* view() const { return &view_; }

 private:
  void* device_ = nullptr;
  gjxl_b200_entropy_code view_{};
};

// WriteAcSections' per-group writes (src/codestream/vardct/encoder.cpp:
// 756-775) on the device: section g of `streams` (device token streams,
// total_tokens in all) written with `code` into sections[g], the same bits
// WriteValidatedTokenStream(streams[g], code, &sections[g]) writes.
Status WriteAcSectionsOnDevice(const EntropyCode& code, const gjxl_b200_token_sections& streams,
                               size_t total_tokens, std::vector<BitWriter>* sections,
                               float* device_ms = nullptr) {
  DeviceEntropyCode tables;
  Status status = tables.Upload(code);
  if (!status.ok()) return status;
  const size_t count = streams.count;
  const size_t words = gjxl_b200_entropy_slot_words(tables.view()->mode, total_tokens, count);
  const size_t offsets_bytes = (count + 1) * 8, bits_bytes = count * 8;
  void* device = nullptr;
  const size_t bytes = words * 8 * 2 + offsets_bytes + bits_bytes + 256;
  status = FromCuda(cudaMalloc(&device, bytes), "section buffers");
  if (!status.ok()) return status;
  auto* slots = static_cast<uint64_t*>(device);
  auto* packed = reinterpret_cast<uint8_t*>(slots + words);
  auto* byte_offsets = reinterpret_cast<uint64_t*>(packed + words * 8);
  auto* bit_counts = byte_offsets + count + 1;
  auto* error = reinterpret_cast<uint32_t*>(bit_counts + count);
  cudaEvent_t begin = nullptr, end = nullptr;
  cudaEventCreate(&begin);
  cudaEventCreate(&end);
  status = FromCuda(cudaMemset(error, 0, 4), "section error word");
  if (status.ok()) {
    cudaEventRecord(begin, nullptr);
    status = FromB200(gjxl_b200_entropy_write_sections(tables.view(), &streams, slots, words,
                                                       bit_counts, packed, words * 8,
                                                       byte_offsets, error, nullptr),
                      "entropy_write_sections");
    cudaEventRecord(end, nullptr);
  }
  if (status.ok()) {
    status = FromB200(gjxl_b200_check_device_error(error, 1, nullptr), "device sections");
  }
  std::vector<uint64_t> bits(count), offsets(count + 1);
  std::vector<uint8_t> host;
  if (status.ok()) {
    status = FromCuda(cudaMemcpy(bits.data(), bit_counts, bits_bytes, cudaMemcpyDeviceToHost),
                      "section bits");
  }
  if (status.ok()) {
    status = FromCuda(cudaMemcpy(offsets.data(), byte_offsets, offsets_bytes,
                                 cudaMemcpyDeviceToHost), "section offsets");
  }
  if (status.ok()) {
    host.resize(offsets[count]);
    status = FromCuda(cudaMemcpy(host.data(), packed, host.size(), cudaMemcpyDeviceToHost),
                      "section bytes");
  }
  if (status.ok() && device_ms != nullptr) cudaEventElapsedTime(device_ms, begin, end);
  cudaEventDestroy(begin);
  cudaEventDestroy(end);
  cudaFree(device);
  if (!status.ok()) return status;
  // Each section's whole bytes, then its last partial byte's bits.
  std::vector<BitWriter> result(count);
  for (size_t g = 0; g < count; ++g) {
    const uint8_t* b = host.data() + offsets[g];
    const size_t whole = bits[g] / 8, rest = bits[g] % 8;
    for (size_t i = 0; i < whole; i += 7) {
      const size_t n = std::min<size_t>(7, whole - i);
      uint64_t v = 0;
      for (size_t k = 0; k < n; ++k) v |= static_cast<uint64_t>(b[i + k]) << (8 * k);
      status = result[g].WriteBits(8 * n, v);
      if (!status.ok()) return status;
    }
    if (rest != 0) {
      status = result[g].WriteBits(rest, b[whole] & ((1u << rest) - 1));
      if (!status.ok()) return status;
    }
  }
  *sections = std::move(result);
  return Status::Ok();
}

// Fixed-ANS populations of a [contexts][128] device histogram (the
// provider's Finish, above).
std::vector<codestream_internal::PreparedFixedAnsCluster> Populations(
  const std::vector<uint32_t>& histogram, size_t contexts) {
  std::vector<codestream_internal::PreparedFixedAnsCluster> out(contexts);
  for (size_t context = 0; context < contexts; ++context) {
    auto& cluster = out[context];
    for (uint32_t symbol = 0; symbol < 128; ++symbol) {
      const uint64_t n = histogram[context * 128 + symbol];
      cluster.counts[symbol] = n;
      cluster.token_count += n;
      if (n != 0) cluster.maximum_symbol = symbol;
      if (symbol >= 16) cluster.extra_bits += n * (2 + ((symbol - 16) >> 2));
    }
  }
  return out;
}

struct SessionOwner {
  gjxl_b200_session* session = nullptr;
  ~SessionOwner() {
    if (session != nullptr) gjxl_b200_session_destroy(session);
  }
};

Status CreateSession(size_t width, size_t height, float target, int effort, int precision,
                     SessionOwner* owner, const float* proposal_weights = nullptr,
                     int learned_iterations = 0, float proposal_confidence = 0.6f) {
  gjxl_b200_options session_options;
  gjxl_b200_default_options(&session_options);
  session_options.butteraugli_target = target;
  session_options.effort = effort;
  session_options.tokenize = 0;  // the serializer asks for its own map's tokens
  session_options.precision = precision;
  session_options.proposal_weights = proposal_weights;
  session_options.learned_iterations = learned_iterations;
  session_options.proposal_confidence = proposal_confidence;
  return FromB200(gjxl_b200_session_create(width, height, &session_options, &owner->session),
                  "session_create");
}

}  // namespace
}  // namespace gjxl::b200_integration

using namespace gjxl;
using namespace gjxl::b200_integration;

GJXL_INTEGRATION_API const char* gjxl_b200_integration_last_error(void) {
  return g_last_error.c_str();
}

// Encodes packed 8-bit sRGB (3 or 4 channels) at the given distance and
// effort: the analysis half on the B200 (one session on the current device,
// default stream, candidate costs at `precision`), the serializer on the
// CPU. device_tokens != 0 installs the device AC tokenizer. Writes the
// codestream (size in *size, -2 when it does not fit `capacity`) and the
// session's final Butteraugli score.
GJXL_INTEGRATION_API int gjxl_b200_encode_image(const uint8_t* pixels, size_t width,
                                                size_t height, size_t row_stride, int channels,
                                                float butteraugli_target, int effort,
                                                int precision, int device_tokens, uint8_t* out,
                                                size_t capacity, size_t* size, double* score) {
  g_last_error.clear();
  SessionOwner owner;
  Status status = CreateSession(width, height, butteraugli_target, effort, precision, &owner);
  if (!status.ok()) return Fail(status);
  std::vector<uint8_t> bytes;
  VarDctEncodingSummary summary;
  status = EncodeWithSession(owner.session, pixels, width, height, row_stride, channels,
                             butteraugli_target, effort, device_tokens != 0, &bytes, &summary);
  if (!status.ok()) return Fail(status);
  *size = bytes.size();
  if (score != nullptr) *score = summary.score_history.back();
  if (bytes.size() > capacity) {
    g_last_error = "codestream capacity exceeded";
    return -2;
  }
  std::memcpy(out, bytes.data(), bytes.size());
  return 0;
}

// The same with the learned analysis mode (gjxl_b200_options.proposal_weights:
// device pointer to the proposal network's parameters; NULL for the plain
// method). Also writes the final evaluation's FP64 Butteraugli 3-norm.
GJXL_INTEGRATION_API int gjxl_b200_encode_image_learned(
  const uint8_t* pixels, size_t width, size_t height, size_t row_stride, int channels,
  float butteraugli_target, int effort, int precision, const float* proposal_weights,
  int learned_iterations, float proposal_confidence, uint8_t* out, size_t capacity, size_t* size,
  double* score, double* pnorm) {
  g_last_error.clear();
  SessionOwner owner;
  Status status = CreateSession(width, height, butteraugli_target, effort, precision, &owner,
                                proposal_weights, learned_iterations, proposal_confidence);
  if (!status.ok()) return Fail(status);
  std::vector<uint8_t> bytes;
  VarDctEncodingSummary summary;
  status = EncodeWithSession(owner.session, pixels, width, height, row_stride, channels,
                             butteraugli_target, effort, false, &bytes, &summary);
  if (!status.ok()) return Fail(status);
  *size = bytes.size();
  if (score != nullptr) *score = summary.score_history.back();
  if (pnorm != nullptr) {
    gjxl_b200_outputs o;
    status = FromB200(gjxl_b200_session_outputs(owner.session, &o), "session_outputs");
    if (!status.ok()) return Fail(status);
    *pnorm = o.host_pnorm_history[o.iterations];
  }
  if (bytes.size() > capacity) {
    g_last_error = "codestream capacity exceeded";
    return -2;
  }
  std::memcpy(out, bytes.data(), bytes.size());
  return 0;
}

// Target-size rate control with the B200 analysis: the reference's own
// bounded search over complete encodes (codestream_internal::SearchTargetSize,
// src/codestream/rate_control.cpp:246-320, as the workflow runs it at
// workflow.cpp:1686-1740) with an evaluator that retargets one prepared
// session per attempt (no reallocation between attempts) and serializes with
// the unchanged writer. tolerance is the relative byte tolerance (the
// workflow's target_size_tolerance), selection kLargestAtOrBelow. Writes the
// selected codestream, its Butteraugli target, the attempt count and whether
// the size is within tolerance.
GJXL_INTEGRATION_API int gjxl_b200_encode_target_size(
  const uint8_t* pixels, size_t width, size_t height, size_t row_stride, int channels,
  int effort, int precision, size_t target_bytes, double tolerance, size_t maximum_attempts,
  uint8_t* out, size_t capacity, size_t* size, float* selected_target, size_t* attempts,
  int* target_met) {
  g_last_error.clear();
  if (target_bytes == 0 || !(tolerance >= 0.0 && tolerance <= 1.0) || maximum_attempts == 0 ||
      maximum_attempts > codestream_internal::kMaximumTargetSizeEncodeAttempts) {
    return Fail(Status::InvalidArgument("target-size options are invalid"));
  }
  SessionOwner owner;
  Status status = CreateSession(width, height, 1.0f, effort, precision, &owner);
  if (!status.ok()) return Fail(status);
  codestream_internal::TargetSizeSearchOptions options;
  options.target_bytes = target_bytes;
  options.tolerance_bytes = static_cast<size_t>(
    std::ceil(static_cast<long double>(target_bytes) * static_cast<long double>(tolerance)));
  options.maximum_attempts = maximum_attempts;
  options.selection = TargetSizeSelectionPolicy::kLargestAtOrBelow;
  codestream_internal::TargetSizeSearchResult result;
  status = codestream_internal::SearchTargetSize(
    options,
    [&](float target, std::vector<uint8_t>* codestream, VarDctEncodingSummary* summary) {
      return EncodeWithSession(owner.session, pixels, width, height, row_stride, channels,
                               target, effort, false, codestream, summary);
    },
    &result);
  if (!status.ok()) return Fail(status);
  *size = result.codestream.size();
  *selected_target = result.summary.selected_butteraugli_target;
  *attempts = result.attempt_count;
  *target_met = result.target_size_met ? 1 : 0;
  if (result.codestream.size() > capacity) {
    g_last_error = "codestream capacity exceeded";
    return -2;
  }
  std::memcpy(out, result.codestream.data(), result.codestream.size());
  return 0;
}

// The AC sections of one analysis written twice with the same entropy code:
// by the reference's WriteValidatedTokenStream on host copies of the
// session's token streams (as WriteAcSections does) and on the device by
// WriteAcSectionsOnDevice from the session's device streams. The code is the
// one the serializer builds from the device populations: direct ANS
// (OptimizeDirectAnsEntropyCodeWithFixedPopulations, balanced) or, with
// prefix != 0, the fast prefix code. Reports the section count, the bytes,
// whether every section is identical, and both writers' times.
GJXL_INTEGRATION_API int gjxl_b200_compare_ac_sections(
  const uint8_t* pixels, size_t width, size_t height, size_t row_stride, int channels,
  float butteraugli_target, int effort, int prefix, size_t* sections, size_t* bytes,
  int* identical, double* device_ms, double* host_ms) {
  g_last_error.clear();
  gjxl_b200_options session_options;
  gjxl_b200_default_options(&session_options);
  session_options.butteraugli_target = butteraugli_target;
  session_options.effort = effort;
  session_options.tokenize = 1;
  SessionOwner owner;
  Status status = FromB200(gjxl_b200_session_create(width, height, &session_options,
                                                    &owner.session), "session_create");
  if (status.ok()) {
    status = FromB200(gjxl_b200_session_analyze_host(owner.session, pixels, row_stride, channels,
                                                     nullptr),
                      "session_analyze_host");
  }
  if (status.ok()) status = FromCuda(cudaDeviceSynchronize(), "analysis");
  gjxl_b200_outputs o;
  if (status.ok()) {
    status = FromB200(gjxl_b200_session_outputs(owner.session, &o), "session_outputs");
  }
  if (!status.ok()) return Fail(status);
  const size_t groups = o.groups, total = o.host_token_count;
  const size_t contexts = 4 * 495;
  std::vector<uint32_t> histogram(contexts * 128);
  status = FromCuda(cudaMemcpy(histogram.data(), o.token_histogram, histogram.size() * 4,
                               cudaMemcpyDeviceToHost), "token histogram");
  if (!status.ok()) return Fail(status);
  std::vector<EntropyTokenStreamView> views;
  for (size_t g = 0; g < groups; ++g) {
    const size_t begin = o.host_group_offsets[g], n = o.host_group_offsets[g + 1] - begin;
    views.push_back(EntropyTokenStreamView::Split({o.host_token_values + begin, n},
                                                  {o.host_token_contexts + begin, n}));
  }
  EntropyCodeOptions options;
  options.context_count = static_cast<uint32_t>(contexts);
  options.maximum_ans_clusters =
    codestream_internal::AcAnsClusterLimit(Extent2D{width, height});
  EntropyCode code;
  if (prefix != 0) {
    status = codestream_internal::OptimizeFastPrefixEntropyCode(views, options, &code);
  } else {
    const auto populations = Populations(histogram, contexts);
    status = codestream_internal::OptimizeDirectAnsEntropyCodeWithFixedPopulations(
      views, options, populations, &code);
  }
  if (!status.ok()) return Fail(status);
  // The reference's writer, one group after another on this thread.
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<BitWriter> want(groups);
  for (size_t g = 0; g < groups && status.ok(); ++g) {
    status = codestream_internal::WriteValidatedTokenStream(views[g], code, &want[g]);
  }
  const auto t1 = std::chrono::steady_clock::now();
  if (!status.ok()) return Fail(status);
  gjxl_b200_token_sections streams{};
  streams.values = o.token_values;
  streams.contexts = o.token_contexts;
  streams.offsets = o.group_offsets;
  streams.count = static_cast<uint32_t>(groups);
  streams.capacity = static_cast<uint32_t>(total);
  std::vector<BitWriter> got;
  float ms = 0.0f;
  status = WriteAcSectionsOnDevice(code, streams, total, &got, &ms);
  if (!status.ok()) return Fail(status);
  bool same = got.size() == want.size();
  size_t written = 0;
  for (size_t g = 0; same && g < groups; ++g) {
    const auto a = got[g].padded_bytes(), b = want[g].padded_bytes();
    same = got[g].bits_written() == want[g].bits_written() &&
           std::equal(a.begin(), a.end(), b.begin(), b.end());
    written += b.size();
  }
  *sections = groups;
  *bytes = written;
  *identical = same ? 1 : 0;
  *device_ms = ms;
  *host_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  return 0;
}
