// Analysis session: buffers + stage orchestration on one stream.
//
// Stage order follows the reference's CPU pipeline for an ordinary
// Butteraugli-target encode (src/codestream/workflow.cpp:700-730 and
// :885-945, src/codec/quantization_pipeline.cpp:155-213 and :429-560,
// src/codec/adaptive_quantization.cpp:1430-1730):
//   packed sRGB -> linear RGB + padded XYB -> quantization-matrix statistics
//   -> initial quant field (pre-Gaborish XYB) -> inverse Gaborish -> initial
//   CfL -> AC-strategy costs -> greedy merge -> forward coefficients of the
//   selected transforms -> adjusted field + policy bounds -> for each of the
//   iterations + 1 evaluations: quantizer, final CfL, coefficient coding, DC
//   quantization, EPF sigma, DC smoothing, reconstruction, Gaborish + EPF,
//   XYB -> linear, Butteraugli, per-transform reduction, field update.
// Nothing returns to the host between stages.

#include "session.h"

#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "aq.h"
#include "cnn.h"
#include "dc_tokens.cuh"
#include "host_util.h"

namespace gjxl_b200 {
namespace {

enum Stage : int {
  kStagePrepare = 0,
  kStageStats,
  kStageInitialQuant,
  kStageGaborishInverse,
  kStageInitialCfl,
  kStageProposals,
  kStageAcCosts,
  kStageAcMerge,
  kStageTransforms,
  kStageAqLoop,
  kStageTokenize,
  kStageCount,
};

const char* const kStageNames[kStageCount] = {
  "prepare_input",   "matrix_scale_stats", "initial_quant_field", "gaborish_inverse",
  "initial_cfl",     "proposals",          "ac_strategy_costs",  "ac_strategy_merge",   "forward_transforms",
  "adaptive_quantization", "ac_tokenize",
};

size_t Align(size_t v, size_t a) { return (v + a - 1) / a * a; }

int AqIterations(int effort) {
  // AdaptiveQuantizationIterations (src/codestream/workflow_internal.h:69-82).
  if (effort <= 5) return 0;
  if (effort == 6) return 1;
  if (effort == 7) return 2;
  if (effort == 8) return 3;
  return 4;
}

std::once_flag g_tables_once[64];

// The reference's initial block-context map (src/codestream/simple_ac_context.h:
// 27-31; DefaultSimpleBlockContextMap, block_context_map.cpp:245-252): no
// raw-quant thresholds, four contexts.
gjxl_b200_block_context_map DefaultBlockContextMap() {
  gjxl_b200_block_context_map m;
  std::memset(&m, 0, sizeof(m));
  const uint8_t rows[3][13] = {{0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1},
                               {2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 3},
                               {2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 3}};
  std::memcpy(m.context_map, rows, sizeof(rows));
  m.num_contexts = 4;
  return m;
}

// ResolveCoefficientOrderBehavior (src/codestream/workflow.cpp:2064-2072) for
// the default density and compression modes.
int OrderMode(const gjxl_b200_options& o) {
  if (o.order_mode >= 0) return o.order_mode;
  return o.effort == 7 ? 2 : 1;
}

}  // namespace

struct Session {
  size_t width = 0, height = 0, pw = 0, ph = 0, bx = 0, by = 0, tx = 0, ty = 0;
  int iterations = 2;
  gjxl_b200_options options{};
  void* arena = nullptr;
  size_t arena_bytes = 0;
  bool external_arena = false;  // device memory lent by the caller (not freed)
  bool host_mirrors = false;    // pinned mirrors allocated (first analyze_host)
  uint8_t* pixels = nullptr;
  size_t pixel_capacity = 0;
  float* linear = nullptr;
  size_t lin_stride = 0, lin_pitch = 0;
  float* opsin = nullptr;
  float* pre = nullptr;
  size_t pitch = 0;
  float* quant = nullptr;
  float* strategy_mask = nullptr;
  float* pixel_mask = nullptr;
  float* iq_scratch = nullptr;
  int8_t* y_to_x = nullptr;
  int8_t* y_to_b = nullptr;
  float* costs = nullptr;
  uint8_t* cells = nullptr;
  float* stats = nullptr;
  uint32_t* error = nullptr;
  // Adaptive quantization.
  int2* anchors = nullptr;
  uint32_t* anchor_counts = nullptr;
  float* coef = nullptr;       // forward coefficients, footprint layout
  float* field = nullptr;      // current quant field
  float* adjusted = nullptr;   // adjusted initial field
  float* range = nullptr;
  AqPolicy* policy = nullptr;
  AqQuantizer* quantizer = nullptr;
  void* select_state = nullptr;
  int32_t* raw = nullptr;
  int8_t* final_y_to_x = nullptr;
  int8_t* final_y_to_b = nullptr;
  int32_t* qac = nullptr;      // quantized AC, footprint layout
  float* dc = nullptr;         // extracted DC (3 x blocks)
  int32_t* qdc = nullptr;
  // Learned mode (proposal_weights set): the network's workspace over all
  // tiles, per-block proposals, top-3 mass and log field scale, per-tile
  // family masks.
  void* cnn_workspace = nullptr;
  uint8_t* proposals = nullptr;
  float* proposal_mass = nullptr;
  float* log_scale = nullptr;
  uint8_t* tile_masks = nullptr;
  uint32_t* kept_tiles = nullptr;   // per family, the tiles whose candidates are scored
  uint32_t* kept_counts = nullptr;
  bool learned = false;
  // DC-group token streams (tokenize != 0).
  uint2* dc_tokens = nullptr;
  uint2* meta_tokens = nullptr;
  uint32_t* dc_group_info = nullptr;
  uint32_t* dc_histogram = nullptr;
  void* dc_token_scratch = nullptr;
  size_t dc_groups = 0, meta_capacity = 0;
  uint32_t* host_dc_tokens = nullptr;
  uint32_t* host_meta_tokens = nullptr;
  uint32_t* host_dc_group_info = nullptr;
  uint32_t* host_dc_histogram = nullptr;
  size_t host_meta_count = 0;
  float* dc_rec = nullptr;
  float* dc_smooth = nullptr;
  float* inverse_sigma = nullptr;
  float* recon = nullptr;      // padded reconstructed XYB
  float* filter_a = nullptr;   // 3 x width x height
  float* filter_b = nullptr;
  float* filtered = nullptr;
  float* rec_linear = nullptr;
  float* distance_map = nullptr;
  float* block_distance = nullptr;
  double* scores = nullptr;
  double* pnorms = nullptr;       // FP64 p-norm (p = 3) of each evaluation's map
  double* pnorm_scratch = nullptr;
  float* matrix_multipliers = nullptr;
  int* matrix_scales = nullptr;
  ButteraugliState* butteraugli = nullptr;
  // AC tokens.
  gjxl_b200_ac_tokens* tokens = nullptr;
  size_t token_capacity = 0, groups = 0;
  uint32_t* tok_values = nullptr;
  uint16_t* tok_contexts = nullptr;
  uint32_t* group_offsets = nullptr;
  uint32_t* histogram = nullptr;
  uint32_t* scans = nullptr;
  uint32_t* order_masks = nullptr;
  uint32_t* host_tok_values = nullptr;
  uint16_t* host_tok_contexts = nullptr;
  uint32_t* host_group_offsets = nullptr;
  size_t host_token_count = 0;
  // Pinned host mirrors of the outputs.
  unsigned char* host_block = nullptr;
  uint8_t* host_cells = nullptr;
  float* host_quant = nullptr;
  int8_t* host_cfl = nullptr;
  float* host_stats = nullptr;
  uint32_t* host_error = nullptr;
  float* host_final_quant = nullptr;
  int32_t* host_raw = nullptr;
  int32_t* host_qdc = nullptr;
  double* host_scores = nullptr;
  double* host_pnorms = nullptr;
  AqQuantizer* host_quantizer = nullptr;
  int32_t* host_qac = nullptr;
  cudaEvent_t events[kStageCount + 1] = {};
  bool events_created = false;
  // The analysis as one CUDA graph, captured on the first analyze() call for
  // a channel count and replayed afterwards. The graph reads the session's
  // own input buffer (`pixels`, rows of width * channels bytes), so callers
  // may pass a new input pointer per image without a recapture.
  cudaStream_t capture_stream = nullptr;
  // Side streams: the fan for the per-family stages, and one stream for the
  // Butteraugli reference preparation, which only needs the input and runs
  // beside the whole front half.
  cudaStream_t fan_side[StreamFan::kSide] = {};
  cudaEvent_t fan_fork = nullptr, fan_join[StreamFan::kSide] = {};
  cudaStream_t prepare_stream = nullptr;
  cudaEvent_t prepare_fork = nullptr, prepare_join = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_channels = 0;
  bool graph_disabled = false;

  ~Session() {
    if (graph) cudaGraphExecDestroy(graph);
    if (capture_stream) cudaStreamDestroy(capture_stream);
    for (auto& side : fan_side) {
      if (side) cudaStreamDestroy(side);
    }
    for (auto& e : fan_join) {
      if (e) cudaEventDestroy(e);
    }
    if (fan_fork) cudaEventDestroy(fan_fork);
    if (prepare_stream) cudaStreamDestroy(prepare_stream);
    if (prepare_fork) cudaEventDestroy(prepare_fork);
    if (prepare_join) cudaEventDestroy(prepare_join);
    if (arena && !external_arena) cudaFree(arena);
    if (host_block) cudaFreeHost(host_block);
    if (butteraugli) ButteraugliDestroy(butteraugli);
    if (tokens) gjxl_b200_ac_tokens_destroy(tokens);
    if (host_tok_values) cudaFreeHost(host_tok_values);
    if (host_dc_tokens) cudaFreeHost(host_dc_tokens);
    if (events_created) {
      for (auto& e : events) cudaEventDestroy(e);
    }
  }
};

namespace {

// Device layout of a session: its own arena, then the Butteraugli planes.
// With `external`, both are carved from caller memory of at least
// DeviceBytes(); else allocated here.
int Allocate(Session* s, void* external, size_t external_bytes, size_t* device_bytes) {
  const size_t plane = s->pw * s->ph;
  const size_t image = s->width * s->height;
  s->lin_stride = Align(s->width, 4);
  s->lin_pitch = s->lin_stride * s->height;
  s->pitch = plane;
  const size_t blocks = s->bx * s->by;
  const size_t tiles = s->tx * s->ty;
  s->pixel_capacity = Align(s->width * 4, 16) * s->height;
  struct Item {
    void** ptr;
    size_t bytes;
  };
  const Item items[] = {
    {reinterpret_cast<void**>(&s->pixels), s->pixel_capacity},
    {reinterpret_cast<void**>(&s->linear), 3 * s->lin_pitch * sizeof(float)},
    {reinterpret_cast<void**>(&s->opsin), 3 * plane * sizeof(float)},
    {reinterpret_cast<void**>(&s->pre), 3 * plane * sizeof(float)},
    {reinterpret_cast<void**>(&s->quant), blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->strategy_mask), blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->pixel_mask), plane * sizeof(float)},
    {reinterpret_cast<void**>(&s->iq_scratch), InitialQuantScratchFloats(s->pw, s->ph) * 4},
    {reinterpret_cast<void**>(&s->y_to_x), tiles},
    {reinterpret_cast<void**>(&s->y_to_b), tiles},
    {reinterpret_cast<void**>(&s->costs), AcStrategyCostFloats(s->bx, s->by) * sizeof(float)},
    {reinterpret_cast<void**>(&s->cells), blocks},
    {reinterpret_cast<void**>(&s->stats), 4 * sizeof(float)},
    {reinterpret_cast<void**>(&s->error), 4 * sizeof(uint32_t)},
    {reinterpret_cast<void**>(&s->anchors), 7 * blocks * sizeof(int2)},
    {reinterpret_cast<void**>(&s->anchor_counts), 8 * sizeof(uint32_t)},
    {reinterpret_cast<void**>(&s->coef), 3 * plane * sizeof(float)},
    {reinterpret_cast<void**>(&s->field), blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->adjusted), blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->range), 4 * sizeof(float)},
    {reinterpret_cast<void**>(&s->policy), sizeof(AqPolicy)},
    {reinterpret_cast<void**>(&s->quantizer), sizeof(AqQuantizer)},
    {reinterpret_cast<void**>(&s->select_state), AqSelectStateBytes()},
    {reinterpret_cast<void**>(&s->raw), blocks * sizeof(int32_t)},
    {reinterpret_cast<void**>(&s->final_y_to_x), tiles},
    {reinterpret_cast<void**>(&s->final_y_to_b), tiles},
    {reinterpret_cast<void**>(&s->qac), 3 * plane * sizeof(int32_t)},
    {reinterpret_cast<void**>(&s->dc), 3 * blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->qdc), 3 * blocks * sizeof(int32_t)},
    {reinterpret_cast<void**>(&s->dc_rec), 3 * blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->dc_smooth), 3 * blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->inverse_sigma), blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->recon), 3 * plane * sizeof(float)},
    {reinterpret_cast<void**>(&s->filter_a), 3 * image * sizeof(float)},
    {reinterpret_cast<void**>(&s->filter_b), 3 * image * sizeof(float)},
    {reinterpret_cast<void**>(&s->filtered), 3 * image * sizeof(float)},
    {reinterpret_cast<void**>(&s->rec_linear), 3 * image * sizeof(float)},
    {reinterpret_cast<void**>(&s->distance_map), image * sizeof(float)},
    {reinterpret_cast<void**>(&s->block_distance), blocks * sizeof(float)},
    {reinterpret_cast<void**>(&s->scores), 8 * sizeof(double)},
    {reinterpret_cast<void**>(&s->pnorms), 8 * sizeof(double)},
    {reinterpret_cast<void**>(&s->pnorm_scratch), PnormScratchBytes()},
    {reinterpret_cast<void**>(&s->matrix_multipliers), 4 * sizeof(float)},
    {reinterpret_cast<void**>(&s->matrix_scales), 4 * sizeof(int)},
    {reinterpret_cast<void**>(&s->tok_values), s->token_capacity * sizeof(uint32_t)},
    {reinterpret_cast<void**>(&s->tok_contexts), s->token_capacity * sizeof(uint16_t)},
    {reinterpret_cast<void**>(&s->group_offsets), (s->groups + 1) * sizeof(uint32_t)},
    {reinterpret_cast<void**>(&s->histogram), (s->token_capacity ? 4 * 495 * 128 : 0) * 4},
    {reinterpret_cast<void**>(&s->scans), 13 * 3 * 1024 * sizeof(uint32_t)},
    {reinterpret_cast<void**>(&s->order_masks), 4 * sizeof(uint32_t)},
    {reinterpret_cast<void**>(&s->cnn_workspace),
     s->learned ? CnnWorkspaceBytes(static_cast<int>(tiles)) : 0},
    {reinterpret_cast<void**>(&s->proposals), s->learned ? 3 * blocks : 0},
    {reinterpret_cast<void**>(&s->proposal_mass), s->learned ? blocks * sizeof(float) : 0},
    {reinterpret_cast<void**>(&s->log_scale), s->learned ? blocks * sizeof(float) : 0},
    {reinterpret_cast<void**>(&s->tile_masks), s->learned ? tiles : 0},
    {reinterpret_cast<void**>(&s->kept_tiles), s->learned ? 7 * tiles * sizeof(uint32_t) : 0},
    {reinterpret_cast<void**>(&s->kept_counts), s->learned ? 8 * sizeof(uint32_t) : 0},
    {reinterpret_cast<void**>(&s->dc_tokens), s->options.tokenize ? 3 * blocks * 8 : 0},
    {reinterpret_cast<void**>(&s->meta_tokens), s->meta_capacity * 8},
    {reinterpret_cast<void**>(&s->dc_group_info), s->dc_groups * 5 * sizeof(uint32_t)},
    {reinterpret_cast<void**>(&s->dc_histogram),
     s->options.tokenize ? kDcContextCount * kHybridSymbols * sizeof(uint32_t) : 0},
    {reinterpret_cast<void**>(&s->dc_token_scratch),
     s->options.tokenize ? DcTokenScratchBytes(s->bx, s->by) : 0},
  };
  size_t total = 0;
  for (const Item& item : items) total = Align(total, 256) + item.bytes;
  const size_t butteraugli_offset = Align(total, 256);
  const size_t needed = butteraugli_offset + ButteraugliArenaBytes(s->width, s->height);
  if (device_bytes != nullptr) {
    *device_bytes = needed;
    return GJXL_B200_OK;
  }
  int status;
  if (external != nullptr) {
    if (external_bytes < needed || reinterpret_cast<uintptr_t>(external) % 256) {
      return SetError(GJXL_B200_INVALID_ARGUMENT, "session: device memory too small or unaligned");
    }
    s->arena = external;
    s->external_arena = true;
  } else {
    status = CheckCuda(DeviceMalloc(&s->arena, total), "session: cudaMalloc");
    if (status != GJXL_B200_OK) return status;
  }
  s->arena_bytes = external != nullptr ? needed : total;
  size_t offset = 0;
  for (const Item& item : items) {
    offset = Align(offset, 256);
    *item.ptr = static_cast<unsigned char*>(s->arena) + offset;
    offset += item.bytes;
  }
  status = ButteraugliCreate(s->width, s->height, 80.0f,
                             external != nullptr
                               ? static_cast<unsigned char*>(external) + butteraugli_offset
                               : nullptr,
                             &s->butteraugli);
  if (status != GJXL_B200_OK) return status;
  if (s->options.tokenize) {
    status = gjxl_b200_ac_tokens_create(s->bx, s->by, &s->tokens);
    if (status != GJXL_B200_OK) return status;
  }
  return GJXL_B200_OK;
}

// Pinned host mirrors of the results, allocated by the first host-input
// analysis (device-resident callers never need them).
int AllocateHostMirrors(Session* s) {
  if (s->host_mirrors) return GJXL_B200_OK;
  const size_t plane = s->pw * s->ph;
  const size_t blocks = s->bx * s->by;
  const size_t tiles = s->tx * s->ty;
  int status;
  const size_t host_bytes = Align(blocks, 16) + Align(blocks * 4, 16) + Align(2 * tiles, 16) +
                            16 + 16 + Align(blocks * 4, 16) + Align(blocks * 4, 16) +
                            Align(3 * blocks * 4, 16) + 64 + 64 +
                            Align(sizeof(AqQuantizer), 16) + Align(3 * plane * 4, 16);
  void* host = nullptr;
  status = CheckCuda(HostMalloc(&host, host_bytes), "session: cudaMallocHost");
  if (status != GJXL_B200_OK) return status;
  s->host_block = static_cast<unsigned char*>(host);
  unsigned char* h = s->host_block;
  auto take = [&](size_t bytes) {
    unsigned char* r = h;
    h += Align(bytes, 16);
    return r;
  };
  s->host_cells = take(blocks);
  s->host_quant = reinterpret_cast<float*>(take(blocks * 4));
  s->host_cfl = reinterpret_cast<int8_t*>(take(2 * tiles));
  s->host_stats = reinterpret_cast<float*>(take(16));
  s->host_error = reinterpret_cast<uint32_t*>(take(16));
  s->host_final_quant = reinterpret_cast<float*>(take(blocks * 4));
  s->host_raw = reinterpret_cast<int32_t*>(take(blocks * 4));
  s->host_qdc = reinterpret_cast<int32_t*>(take(3 * blocks * 4));
  s->host_scores = reinterpret_cast<double*>(take(64));
  s->host_pnorms = reinterpret_cast<double*>(take(64));
  s->host_quantizer = reinterpret_cast<AqQuantizer*>(take(sizeof(AqQuantizer)));
  s->host_qac = reinterpret_cast<int32_t*>(take(3 * plane * 4));
  if (s->options.tokenize) {
    void* mirror = nullptr;
    status = CheckCuda(HostMalloc(&mirror, s->token_capacity * 6 + (s->groups + 1) * 4 + 64),
                       "session: token mirrors");
    if (status != GJXL_B200_OK) return status;
    s->host_tok_values = static_cast<uint32_t*>(mirror);
    s->host_tok_contexts = reinterpret_cast<uint16_t*>(s->host_tok_values + s->token_capacity);
    s->host_group_offsets = reinterpret_cast<uint32_t*>(
      reinterpret_cast<unsigned char*>(mirror) + Align(s->token_capacity * 6, 16));
    const size_t dc_bytes = 3 * blocks * 8 + s->meta_capacity * 8 + s->dc_groups * 5 * 4 +
                            kDcContextCount * kHybridSymbols * 4 + 64;
    void* dc_mirror = nullptr;
    status = CheckCuda(HostMalloc(&dc_mirror, dc_bytes), "session: DC token mirrors");
    if (status != GJXL_B200_OK) return status;
    s->host_dc_tokens = static_cast<uint32_t*>(dc_mirror);
    s->host_meta_tokens = s->host_dc_tokens + 6 * blocks;
    s->host_dc_group_info = s->host_meta_tokens + 2 * s->meta_capacity;
    s->host_dc_histogram = s->host_dc_group_info + 5 * s->dc_groups;
  }
  s->host_mirrors = true;
  return GJXL_B200_OK;
}

int CreateStreams(Session* s) {
  int status;
  for (auto& side : s->fan_side) {
    status = CheckCuda(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking),
                       "session: side stream");
    if (status != GJXL_B200_OK) return status;
  }
  for (cudaEvent_t* e : {&s->fan_fork, &s->fan_join[0], &s->fan_join[1], &s->fan_join[2],
                         &s->prepare_fork, &s->prepare_join}) {
    status = CheckCuda(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "session: event");
    if (status != GJXL_B200_OK) return status;
  }
  status = CheckCuda(cudaStreamCreateWithFlags(&s->prepare_stream, cudaStreamNonBlocking),
                     "session: prepare stream");
  if (status != GJXL_B200_OK) return status;
  if (s->options.profile_stages) {
    for (auto& e : s->events) {
      status = CheckCuda(cudaEventCreate(&e), "session: cudaEventCreate");
      if (status != GJXL_B200_OK) return status;
    }
    s->events_created = true;
  }
  return GJXL_B200_OK;
}

void Mark(Session* s, int stage, cudaStream_t stream) {
  if (s->events_created) cudaEventRecord(s->events[stage], stream);
}

#define GJXL_TRY(expr)                         \
  do {                                         \
    const int gjxl_status_ = (expr);           \
    if (gjxl_status_ != GJXL_B200_OK) return gjxl_status_; \
  } while (0)

StreamFan MakeFan(const Session* s, cudaStream_t stream) {
  StreamFan fan;
  fan.main = stream;
  for (int i = 0; i < StreamFan::kSide; ++i) {
    fan.side[i] = s->fan_side[i];
    fan.join[i] = s->fan_join[i];
  }
  fan.fork = s->fan_fork;
  return fan;
}

int RunAq(Session* s, cudaStream_t stream) {
  const float target = s->options.butteraugli_target;
  const size_t blocks = s->bx * s->by;
  GJXL_TRY(AqBuildAnchors(s->cells, s->bx, s->by, s->anchors, s->anchor_counts, stream));
  const StreamFan fan = MakeFan(s, stream);
  GJXL_TRY(AqForwardCoefficients(s->pre, s->pw, s->pitch, s->bx, s->by, s->anchors,
                                 s->anchor_counts, s->coef, stream, &fan));
  GJXL_TRY(AqAdjustField(s->cells, s->bx, s->by, s->quant, s->adjusted, target, stream));
  // Learned mode: the refinement starts from the predicted field.
  if (s->learned) GJXL_TRY(CnnScaleField(s->adjusted, s->log_scale, blocks, stream));
  GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->field, s->adjusted, blocks * sizeof(float),
                                     cudaMemcpyDeviceToDevice, stream), "session: field"));
  GJXL_TRY(AqPolicySetup(s->adjusted, blocks, target, s->range, s->policy, s->error, stream));
  // The reference preparation (queued on its own stream after the input)
  // must be done before the first comparison.
  GJXL_TRY(CheckCuda(cudaStreamWaitEvent(stream, s->prepare_join, 0), "session: prepare join"));
  Mark(s, kStageAqLoop, stream);
  for (int iteration = 0; iteration <= s->iterations; ++iteration) {
    GJXL_TRY(AqQuantizer_(s->field, blocks, s->policy, s->quantizer, s->raw, s->select_state,
                          s->error, stream));
    GJXL_TRY(AqFinalCfl(s->cells, s->bx, s->by, s->coef, s->pw, s->pitch, s->raw, s->quantizer,
                        s->final_y_to_x, s->final_y_to_b, stream));
    GJXL_TRY(AqCoding(s->anchors, s->anchor_counts, s->bx, s->by, s->coef, s->pw, s->pitch,
                      s->qac, s->dc, s->raw, s->quantizer, s->final_y_to_x, s->final_y_to_b,
                      s->matrix_multipliers, s->error, stream, &fan));
    GJXL_TRY(AqDcQuantize(s->dc, s->bx, s->by, s->quantizer, s->qdc, s->dc_rec, 1,
                          iteration == s->iterations && s->options.tokenize ? s->dc_tokens
                                                                            : nullptr,
                          s->error + 2,
                          stream));
    GJXL_TRY(AqInverseSigma(s->cells, s->bx, s->by, s->raw, s->quantizer, s->inverse_sigma,
                            stream));
    GJXL_TRY(AqSmoothDc(s->dc_rec, s->bx, s->by, s->quantizer, s->dc_smooth, stream));
    GJXL_TRY(AqReconstruct(s->anchors, s->anchor_counts, s->bx, s->by, s->qac, s->pw, s->pitch,
                           s->dc_smooth, s->raw, s->quantizer, s->final_y_to_x, s->final_y_to_b,
                           s->matrix_multipliers, s->recon, stream, &fan));
    // The last loop-filter pass writes the linear image Butteraugli compares.
    GJXL_TRY(AqLoopFilters(s->recon, s->pw, s->pitch, s->width, s->height, s->inverse_sigma,
                           s->bx, s->filter_a, s->filter_b, s->filtered, s->error, stream,
                           s->rec_linear, s->options.intensity_target));
    GJXL_TRY(ButteraugliCompare(s->butteraugli, s->rec_linear, s->width, s->width * s->height,
                                s->distance_map, s->width, s->scores + iteration, stream));
    GJXL_TRY(LaunchPnorm(s->distance_map, s->width, s->width, s->height, 3.0,
                         s->pnorm_scratch, s->pnorms + iteration, stream));
    GJXL_TRY(AqBlockReduce(s->cells, s->bx, s->by, s->distance_map, s->width, s->height,
                           s->block_distance, stream));
    if (iteration < s->iterations) {
      GJXL_TRY(AqPolicyUpdate(s->field, s->adjusted, s->block_distance, blocks, iteration, target,
                              s->policy, s->quantizer, s->error, stream));
    }
  }
  // Fold the Butteraugli error word into the session's.
  return GJXL_B200_OK;
}

int Run(Session* s, const uint8_t* pixels, size_t row_stride, int channels,
        cudaStream_t stream) {
  GJXL_TRY(CheckCuda(cudaMemsetAsync(s->error, 0, 4 * sizeof(uint32_t), stream),
                     "session: clear error"));
  const float target = s->options.butteraugli_target;
  Mark(s, kStagePrepare, stream);
  GJXL_TRY(gjxl_b200_prepare_input(pixels, s->width, s->height, row_stride, channels,
                                   s->options.intensity_target, s->linear, s->lin_stride,
                                   s->lin_pitch, s->opsin, s->pw, s->pitch, s->pw, s->ph,
                                   s->error, stream));
  // Butteraugli reference preparation beside the front half.
  GJXL_TRY(CheckCuda(cudaEventRecord(s->prepare_fork, stream), "session: prepare fork"));
  GJXL_TRY(CheckCuda(cudaStreamWaitEvent(s->prepare_stream, s->prepare_fork, 0),
                     "session: prepare fork"));
  GJXL_TRY(ButteraugliPrepare(s->butteraugli, s->linear, s->lin_stride, s->lin_pitch,
                              s->prepare_stream));
  GJXL_TRY(CheckCuda(cudaEventRecord(s->prepare_join, s->prepare_stream),
                     "session: prepare join"));
  Mark(s, kStageStats, stream);
  const bool stats = s->options.effort >= 7;  // ShouldComputeQuantizationMatrixScaleStats
  if (stats) {
    GJXL_TRY(gjxl_b200_matrix_scale_stats(s->opsin, s->pw, s->pitch, s->width, s->height,
                                          s->stats, stream));
  } else {
    GJXL_TRY(CheckCuda(cudaMemsetAsync(s->stats, 0, 4 * sizeof(float), stream),
                       "session: clear stats"));
  }
  GJXL_TRY(AqMatrixScales(s->stats, stats, target, s->matrix_multipliers, s->matrix_scales,
                          stream));
  Mark(s, kStageInitialQuant, stream);
  // Initial quantization samples the pre-Gaborish image at the full target
  // (Gaborish is on for efforts >= 5: quantization_pipeline.cpp:452-456).
  GJXL_TRY(LaunchInitialQuantField(s->opsin, s->pw, s->pitch, s->pw, s->ph, target, 1.0f,
                                   s->quant, s->strategy_mask, s->pixel_mask, s->pw,
                                   s->iq_scratch, s->error, stream));
  Mark(s, kStageGaborishInverse, stream);
  const float multipliers[3] = {1.0f, 1.0f, 1.0f};
  GJXL_TRY(LaunchGaborishInverse(s->opsin, s->pw, s->pitch, s->pre, s->pw, s->pitch, s->pw,
                                 s->ph, multipliers, s->error, stream));
  Mark(s, kStageInitialCfl, stream);
  GJXL_TRY(LaunchInitialCfl(s->pre, s->pw, s->pitch, s->pw, s->ph, s->y_to_x, s->y_to_b,
                            stream));
  Mark(s, kStageProposals, stream);
  if (s->learned) {
    const int tiles = static_cast<int>(s->tx * s->ty);
    const CnnActivations a = CnnLayout(s->cnn_workspace, tiles);
    GJXL_TRY(CnnGather(s->pre, s->pw, s->pitch, s->pw, s->ph, nullptr, tiles, target, a.act[0],
                       stream));
    GJXL_TRY(CnnForward(s->options.proposal_weights, a, tiles, stream, true, s->error));
    GJXL_TRY(CnnPropose(a.head, tiles, s->bx, s->by, s->proposals, s->proposal_mass,
                        s->log_scale, stream));
    GJXL_TRY(CnnTileMasks(s->proposals, s->proposal_mass, s->bx, s->by,
                          s->options.proposal_confidence, s->tile_masks, stream));
    GJXL_TRY(CnnKeptTiles(s->tile_masks, s->tx * s->ty, s->kept_tiles, s->kept_counts, stream));
  }
  Mark(s, kStageAcCosts, stream);
  const StreamFan fan = MakeFan(s, stream);
  const bool dense = s->options.effort >= 10;
  GJXL_TRY(LaunchAcStrategyCosts(s->pre, s->pw, s->pitch, s->pw, s->ph, s->quant, s->pixel_mask,
                                 s->pw, s->y_to_x, s->y_to_b, target, dense,
                                 s->options.precision, s->costs, s->error, stream, &fan,
                                 s->learned ? s->kept_tiles : nullptr,
                                 s->learned ? s->kept_counts : nullptr));
  if (s->learned) GJXL_TRY(CnnMaskCosts(s->costs, s->tile_masks, s->bx, s->by, stream));
  Mark(s, kStageAcMerge, stream);
  GJXL_TRY(LaunchAcStrategySearch(s->costs, s->pw, s->ph, target, dense, s->cells, s->error,
                                  stream));
  Mark(s, kStageTransforms, stream);
  GJXL_TRY(RunAq(s, stream));
  Mark(s, kStageTokenize, stream);
  if (s->tokens != nullptr) {
    const gjxl_b200_block_context_map map = DefaultBlockContextMap();
    gjxl_b200_ac_token_outputs outs;
    std::memset(&outs, 0, sizeof(outs));
    outs.token_values = s->tok_values;
    outs.token_contexts = s->tok_contexts;
    outs.token_capacity = s->token_capacity;
    outs.group_offsets = s->group_offsets;
    outs.histogram = s->histogram;
    outs.orders = s->scans;
    outs.present_mask = s->order_masks;
    outs.used_order_mask = s->order_masks + 1;
    outs.device_error = s->error + 2;
    GJXL_TRY(gjxl_b200_ac_tokenize(s->tokens, s->cells, s->raw, s->qac, s->pw, s->pitch, &map,
                                   OrderMode(s->options), &outs, stream));
  }
  if (s->options.tokenize) {
    // The DC tokens came with the last DC quantization; the AC metadata of
    // the final strategy, quant field and CfL maps (default EPF sharpness 4).
    GJXL_TRY(LaunchMetaTokens(s->cells, s->raw, nullptr, s->final_y_to_x, s->final_y_to_b, s->bx,
                              s->by, s->dc_tokens, s->meta_tokens, s->dc_group_info,
                              s->dc_histogram, s->dc_token_scratch, s->error + 2, stream));
  }
  Mark(s, kStageCount, stream);
  // Merge the Butteraugli error word into the session error word.
  GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->error + 1, ButteraugliErrorWord(s->butteraugli),
                                     sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream),
                     "session: error word"));
  return GJXL_B200_OK;
}

// Runs the analysis as a replay of its captured graph: one launch instead of
// ~350, with the same kernels and arguments. The graph reads the session's
// input buffer; input elsewhere on the device is first copied there (one
// stream-ordered 2D copy, 37 MB at 12 MP), so a new input pointer per image
// costs that copy and never a recapture. Stage profiling, a caller stream
// that is itself being captured, or a failed capture run the stages directly
// on the caller's pointer.
int RunReplay(Session* s, const uint8_t* pixels, size_t row_stride, int channels,
              cudaStream_t stream) {
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  if (s->events_created || s->graph_disabled ||
      cudaStreamIsCapturing(stream, &capturing) != cudaSuccess ||
      capturing != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return Run(s, pixels, row_stride, channels, stream);
  }
  const size_t packed_row = s->width * static_cast<size_t>(channels);
  if (pixels != s->pixels) {
    GJXL_TRY(CheckCuda(cudaMemcpy2DAsync(s->pixels, packed_row, pixels, row_stride, packed_row,
                                         s->height, cudaMemcpyDeviceToDevice, stream),
                       "session: input copy"));
  } else if (row_stride != packed_row) {
    return SetError(GJXL_B200_INVALID_ARGUMENT,
                    "session_analyze: the session input buffer holds packed rows");
  }
  if (s->graph == nullptr || s->graph_channels != channels) {
    if (s->graph != nullptr) {
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
    }
    if (s->capture_stream == nullptr) {
      GJXL_TRY(CheckCuda(cudaStreamCreateWithFlags(&s->capture_stream, cudaStreamNonBlocking),
                         "session: capture stream"));
    }
    cudaGraph_t graph = nullptr;
    bool ok = cudaStreamBeginCapture(s->capture_stream, cudaStreamCaptureModeRelaxed) ==
              cudaSuccess;
    if (ok) {
      const int run_status = Run(s, s->pixels, packed_row, channels, s->capture_stream);
      ok = cudaStreamEndCapture(s->capture_stream, &graph) == cudaSuccess &&
           run_status == GJXL_B200_OK;
    }
    if (ok) ok = !InjectFailure(kInjectGraph) && cudaGraphInstantiate(&s->graph, graph, 0) ==
                                                 cudaSuccess;
    if (graph != nullptr) cudaGraphDestroy(graph);
    if (!ok) {
      cudaGetLastError();
      ClearLastError();
      s->graph = nullptr;
      s->graph_disabled = true;
      return Run(s, s->pixels, packed_row, channels, stream);
    }
    s->graph_channels = channels;
  }
  return CheckCuda(cudaGraphLaunch(s->graph, stream), "session: graph launch");
}

int CopyOutputs(Session* s, cudaStream_t stream) {
  const size_t blocks = s->bx * s->by, tiles = s->tx * s->ty, plane = s->pw * s->ph;
  const struct {
    void* dst;
    const void* src;
    size_t bytes;
  } copies[] = {
    {s->host_cells, s->cells, blocks},
    {s->host_quant, s->quant, blocks * sizeof(float)},
    {s->host_cfl, s->final_y_to_x, tiles},
    {s->host_cfl + tiles, s->final_y_to_b, tiles},
    {s->host_stats, s->stats, 3 * sizeof(float)},
    {s->host_error, s->error, 3 * sizeof(uint32_t)},
    {s->host_final_quant, s->field, blocks * sizeof(float)},
    {s->host_raw, s->raw, blocks * sizeof(int32_t)},
    {s->host_qdc, s->qdc, 3 * blocks * sizeof(int32_t)},
    {s->host_scores, s->scores, (s->iterations + 1) * sizeof(double)},
    {s->host_pnorms, s->pnorms, (s->iterations + 1) * sizeof(double)},
    {s->host_quantizer, s->quantizer, sizeof(AqQuantizer)},
    // Quantized AC returns to the host only without tokenization (the tokens
    // carry it otherwise).
    {s->host_qac, s->qac, s->tokens != nullptr ? 0 : 3 * plane * sizeof(int32_t)},
  };
  for (const auto& c : copies) {
    if (c.bytes == 0) continue;
    GJXL_TRY(CheckCuda(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, stream),
                       "session: output copy"));
  }
  return GJXL_B200_OK;
}

}  // namespace
}  // namespace gjxl_b200

using namespace gjxl_b200;

struct gjxl_b200_session : public Session {};

extern "C" void gjxl_b200_default_options(gjxl_b200_options* options) {
  if (options == nullptr) return;
  std::memset(options, 0, sizeof(*options));
  options->struct_size = sizeof(*options);
  options->butteraugli_target = 1.0f;
  options->effort = 7;
  options->intensity_target = 255.0f;
  options->profile_stages = 0;
  options->tokenize = 1;
  options->order_mode = -1;
  options->precision = GJXL_B200_PRECISION_EXACT;
  options->proposal_weights = nullptr;
  options->learned_iterations = 1;
  options->proposal_confidence = 0.6f;
}

namespace {

// Session creation proper. With `query`, only the device bytes the session
// needs (its arena and the Butteraugli planes) are computed; with
// `external`, those come from the caller's memory.
int CreateSession(size_t width, size_t height, const gjxl_b200_options* options, void* external,
                  size_t external_bytes, size_t* query, gjxl_b200_session** out) {
  if ((out == nullptr && query == nullptr) || width == 0 || height == 0 ||
      width > (1u << 20) || height > (1u << 20)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_create: invalid extent");
  }
  if (out != nullptr) *out = nullptr;
  gjxl_b200_options o;
  gjxl_b200_default_options(&o);
  if (options != nullptr) {
    if (options->struct_size != sizeof(gjxl_b200_options)) {
      return SetError(GJXL_B200_INVALID_ARGUMENT, "session_create: options struct_size");
    }
    o = *options;
  }
  if (!std::isfinite(o.butteraugli_target) || o.butteraugli_target <= 0.0f ||
      !std::isfinite(o.intensity_target) || o.intensity_target <= 0.0f) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_create: invalid options");
  }
  if (o.order_mode < -1 || o.order_mode > 2) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_create: order_mode is -1..2");
  }
  if (o.precision != GJXL_B200_PRECISION_EXACT && o.precision != GJXL_B200_PRECISION_FAST) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_create: precision is 0 or 1");
  }
  if (o.proposal_weights != nullptr &&
      (o.learned_iterations > 4 || !(o.proposal_confidence >= 0.0f && o.proposal_confidence <= 1.0f))) {
    return SetError(GJXL_B200_INVALID_ARGUMENT,
                    "session_create: learned_iterations <= 4, proposal_confidence in [0, 1]");
  }
  if (o.effort < 5 || o.effort > 10) {
    return SetError(GJXL_B200_UNSUPPORTED,
                    "session_create: efforts 5-10 (mixed-transform search) are supported");
  }
  int device = 0;
  int status = CheckCuda(cudaGetDevice(&device), "session_create: cudaGetDevice");
  if (status != GJXL_B200_OK) return status;
  if (device >= 0 && device < 64) {
    std::call_once(g_tables_once[device], [] {
      UploadDcTables();
      UploadDcReconTables();
    });
  }
  auto* s = new (std::nothrow) gjxl_b200_session();
  if (s == nullptr) return SetError(GJXL_B200_OUT_OF_MEMORY, "session_create: host allocation");
  s->width = width;
  s->height = height;
  s->pw = (width + 7) / 8 * 8;
  s->ph = (height + 7) / 8 * 8;
  s->bx = s->pw / 8;
  s->by = s->ph / 8;
  s->tx = (s->bx + 7) / 8;
  s->ty = (s->by + 7) / 8;
  s->options = o;
  s->learned = o.proposal_weights != nullptr;
  s->iterations = s->learned && o.learned_iterations >= 0 ? o.learned_iterations
                                                           : AqIterations(o.effort);
  s->groups = ((s->bx + 31) / 32) * ((s->by + 31) / 32);
  s->token_capacity = o.tokenize ? gjxl_b200_ac_token_capacity(s->bx, s->by) : 0;
  if (o.tokenize) {
    s->dc_groups = ((s->bx + 255) / 256) * ((s->by + 255) / 256);
    s->meta_capacity = MetaTokenCapacity(s->bx, s->by);
  }
  if (query != nullptr) {
    status = Allocate(s, nullptr, 0, query);
    delete s;
    return status;
  }
  status = Allocate(s, external, external_bytes, nullptr);
  if (status == GJXL_B200_OK) status = CreateStreams(s);
  if (status != GJXL_B200_OK) {
    delete s;
    return status;
  }
  *out = s;
  return GJXL_B200_OK;
}

}  // namespace

extern "C" int gjxl_b200_session_create(size_t width, size_t height,
                                        const gjxl_b200_options* options,
                                        gjxl_b200_session** out) {
  ClearLastError();
  return CreateSession(width, height, options, nullptr, 0, nullptr, out);
}

extern "C" int gjxl_b200_session_device_bytes(size_t width, size_t height,
                                              const gjxl_b200_options* options, size_t* bytes) {
  ClearLastError();
  if (bytes == nullptr) return SetError(GJXL_B200_INVALID_ARGUMENT, "session_device_bytes: null");
  return CreateSession(width, height, options, nullptr, 0, bytes, nullptr);
}

extern "C" int gjxl_b200_session_create_in(size_t width, size_t height,
                                           const gjxl_b200_options* options, void* device_memory,
                                           size_t device_bytes, gjxl_b200_session** out) {
  ClearLastError();
  if (device_memory == nullptr) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_create_in: null device memory");
  }
  return CreateSession(width, height, options, device_memory, device_bytes, nullptr, out);
}

extern "C" void gjxl_b200_session_destroy(gjxl_b200_session* session) { delete session; }

extern "C" int gjxl_b200_session_set_butteraugli_target(gjxl_b200_session* s, float target) {
  ClearLastError();
  if (s == nullptr || !std::isfinite(target) || target <= 0.0f) {
    return SetError(GJXL_B200_INVALID_ARGUMENT,
                    "session_set_butteraugli_target: invalid arguments");
  }
  if (s->options.butteraugli_target != target) {
    s->options.butteraugli_target = target;
    // The captured graph holds the old target's constants: capture again on
    // the next analysis. Every buffer is kept.
    if (s->graph != nullptr) {
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
    }
  }
  return GJXL_B200_OK;
}

extern "C" int gjxl_b200_session_analyze(gjxl_b200_session* s, const uint8_t* pixels,
                                         size_t row_stride, int channels, void* stream) {
  ClearLastError();
  if (s == nullptr || pixels == nullptr || (channels != 3 && channels != 4) ||
      row_stride < s->width * static_cast<size_t>(channels)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_analyze: invalid arguments");
  }
  if (InjectFailure(kInjectSubmission)) {
    return SetError(GJXL_B200_SUBMISSION_FAILED, "session_analyze: injected submission failure");
  }
  return RunReplay(s, pixels, row_stride, channels, static_cast<cudaStream_t>(stream));
}

extern "C" int gjxl_b200_session_analyze_host(gjxl_b200_session* s, const uint8_t* host_pixels,
                                              size_t row_stride, int channels, void* stream) {
  ClearLastError();
  if (s == nullptr || host_pixels == nullptr || (channels != 3 && channels != 4) ||
      row_stride < s->width * channels) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_analyze_host: invalid arguments");
  }
  if (InjectFailure(kInjectSubmission)) {
    return SetError(GJXL_B200_SUBMISSION_FAILED,
                    "session_analyze_host: injected submission failure");
  }
  GJXL_TRY(AllocateHostMirrors(s));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Packed rows in the session's input buffer (one contiguous copy when the
  // caller's rows are packed too).
  const size_t packed_row = s->width * static_cast<size_t>(channels);
  GJXL_TRY(CheckCuda(cudaMemcpy2DAsync(s->pixels, packed_row, host_pixels, row_stride,
                                       packed_row, s->height, cudaMemcpyHostToDevice, st),
                     "session: input upload"));
  GJXL_TRY(RunReplay(s, s->pixels, packed_row, channels, st));
  GJXL_TRY(CopyOutputs(s, st));
  s->host_token_count = 0;
  if (s->tokens != nullptr) {
    GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->host_group_offsets, s->group_offsets,
                                       (s->groups + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                       st),
                       "session: group offsets"));
    GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->host_dc_group_info, s->dc_group_info,
                                       s->dc_groups * 5 * sizeof(uint32_t),
                                       cudaMemcpyDeviceToHost, st),
                       "session: DC group table"));
    GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->host_dc_tokens, s->dc_tokens, 3 * s->bx * s->by * 8,
                                       cudaMemcpyDeviceToHost, st),
                       "session: DC tokens"));
    GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->host_dc_histogram, s->dc_histogram,
                                       kDcContextCount * kHybridSymbols * sizeof(uint32_t),
                                       cudaMemcpyDeviceToHost, st),
                       "session: DC histogram"));
    GJXL_TRY(CheckCuda(cudaStreamSynchronize(st), "session: analysis"));
    const size_t total = s->host_group_offsets[s->groups];
    if (total > s->token_capacity) {
      return SetError(GJXL_B200_INTERNAL, "session_analyze_host: token count exceeds capacity");
    }
    GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->host_tok_values, s->tok_values, total * 4,
                                       cudaMemcpyDeviceToHost, st),
                       "session: token values"));
    GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->host_tok_contexts, s->tok_contexts, total * 2,
                                       cudaMemcpyDeviceToHost, st),
                       "session: token contexts"));
    s->host_token_count = total;
    // DC-group streams: every DC token, the metadata tokens the group table
    // counts, and the histogram.
    const size_t meta = s->host_dc_group_info[5 * (s->dc_groups - 1) + 2] +
                        s->host_dc_group_info[5 * (s->dc_groups - 1) + 3];
    if (meta > s->meta_capacity) {
      return SetError(GJXL_B200_INTERNAL, "session_analyze_host: metadata token overflow");
    }
    GJXL_TRY(CheckCuda(cudaMemcpyAsync(s->host_meta_tokens, s->meta_tokens, meta * 8,
                                       cudaMemcpyDeviceToHost, st),
                       "session: metadata tokens"));
    s->host_meta_count = meta;
  }
  GJXL_TRY(CheckCuda(cudaStreamSynchronize(st), "session: analysis"));
  // A nonzero device error word fails the call, as the reference's
  // ReadAndCheckDeviceError does (src/gpu/cuda/cuda_aq_resident.cpp:3451).
  for (int i = 0; i < 3; ++i) {
    if (s->host_error[i] != 0) {
      return SetError(GJXL_B200_DEVICE_ERROR,
                      i == 0   ? "session_analyze_host: analysis device error word is set"
                      : i == 1 ? "session_analyze_host: Butteraugli device error word is set"
                               : "session_analyze_host: tokenization device error word is set");
    }
  }
  return GJXL_B200_OK;
}

extern "C" int gjxl_b200_session_outputs(const gjxl_b200_session* s, gjxl_b200_outputs* out) {
  ClearLastError();
  if (s == nullptr || out == nullptr) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_outputs: null argument");
  }
  std::memset(out, 0, sizeof(*out));
  out->padded_width = s->pw;
  out->padded_height = s->ph;
  out->blocks_x = s->bx;
  out->blocks_y = s->by;
  out->tiles_x = s->tx;
  out->tiles_y = s->ty;
  out->iterations = static_cast<size_t>(s->iterations);
  out->linear = s->linear;
  out->linear_stride = s->lin_stride;
  out->linear_plane_pitch = s->lin_pitch;
  out->opsin = s->opsin;
  out->preprocessed_opsin = s->pre;
  out->opsin_stride = s->pw;
  out->opsin_plane_pitch = s->pitch;
  out->initial_quant_field = s->quant;
  out->strategy_mask = s->strategy_mask;
  out->pixel_mask = s->pixel_mask;
  out->initial_y_to_x = s->y_to_x;
  out->initial_y_to_b = s->y_to_b;
  out->strategy_cells = s->cells;
  out->matrix_scale_stats = s->stats;
  out->matrix_scales = s->matrix_scales;
  out->quant_field = s->field;
  out->adjusted_quant_field = s->adjusted;
  if (s->learned) {
    out->proposals = s->proposals;
    out->proposal_mass = s->proposal_mass;
    out->proposal_log_scale = s->log_scale;
    out->tile_family_masks = s->tile_masks;
  }
  out->raw_quant_field = s->raw;
  out->y_to_x = s->final_y_to_x;
  out->y_to_b = s->final_y_to_b;
  out->quantized_ac = s->qac;
  out->quantized_dc = s->qdc;
  out->dc = s->dc_rec;
  out->block_distance = s->block_distance;
  out->reconstructed_linear = s->rec_linear;
  out->distance_map = s->distance_map;
  out->score_history = s->scores;
  out->quantizer_params = reinterpret_cast<const uint32_t*>(s->quantizer);
  out->device_error = s->error;
  out->host_strategy_cells = s->host_cells;
  out->host_initial_quant_field = s->host_quant;
  out->host_y_to_x = s->host_cfl;
  out->host_y_to_b = s->host_cfl + s->tx * s->ty;
  out->host_matrix_scale_stats = s->host_stats;
  out->host_device_error = s->host_error;
  out->host_quant_field = s->host_final_quant;
  out->host_raw_quant_field = s->host_raw;
  out->host_quantized_dc = s->host_qdc;
  out->host_score_history = s->host_scores;
  out->host_quantizer_params = reinterpret_cast<const uint32_t*>(s->host_quantizer);
  out->host_quantized_ac = s->host_qac;
  out->groups = s->groups;
  if (s->tokens != nullptr) {
    out->token_values = s->tok_values;
    out->token_contexts = s->tok_contexts;
    out->group_offsets = s->group_offsets;
    out->token_histogram = s->histogram;
    out->scans = s->scans;
    out->order_masks = s->order_masks;
    out->host_token_values = s->host_tok_values;
    out->host_token_contexts = s->host_tok_contexts;
    out->host_group_offsets = s->host_group_offsets;
  }
  out->host_token_count = s->host_token_count;
  out->dc_groups = s->dc_groups;
  if (s->options.tokenize) {
    out->dc_tokens = reinterpret_cast<const uint32_t*>(s->dc_tokens);
    out->meta_tokens = reinterpret_cast<const uint32_t*>(s->meta_tokens);
    out->dc_group_info = s->dc_group_info;
    out->dc_histogram = s->dc_histogram;
    out->host_dc_tokens = s->host_dc_tokens;
    out->host_meta_tokens = s->host_meta_tokens;
    out->host_dc_group_info = s->host_dc_group_info;
    out->host_dc_histogram = s->host_dc_histogram;
  }
  out->host_meta_token_count = s->host_meta_count;
  out->device_bytes = s->arena_bytes;
  out->pnorm_history = s->pnorms;
  out->host_pnorm_history = s->host_pnorms;
  out->input_pixels = s->pixels;
  out->input_capacity = s->pixel_capacity;
  out->graph_replay = s->graph != nullptr ? 1 : 0;
  return GJXL_B200_OK;
}

extern "C" int gjxl_b200_session_stage_times(gjxl_b200_session* s, float* milliseconds,
                                             int capacity) {
  ClearLastError();
  if (s == nullptr || milliseconds == nullptr) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_stage_times: null argument");
  }
  if (!s->events_created) {
    return SetError(GJXL_B200_FAILED_PRECONDITION, "session_stage_times: profiling is off");
  }
  const int n = capacity < kStageCount ? capacity : kStageCount;
  for (int i = 0; i < n; ++i) {
    const int status =
      CheckCuda(cudaEventElapsedTime(&milliseconds[i], s->events[i], s->events[i + 1]),
                "session_stage_times");
    if (status != GJXL_B200_OK) return -status;
  }
  return n;
}

extern "C" const char* gjxl_b200_stage_name(int stage) {
  return stage >= 0 && stage < kStageCount ? kStageNames[stage] : nullptr;
}

extern "C" int gjxl_b200_session_kernel_count(gjxl_b200_session* s, const uint8_t* pixels,
                                              size_t row_stride, int channels,
                                              size_t* kernels) {
  ClearLastError();
  if (s == nullptr || pixels == nullptr || kernels == nullptr) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_kernel_count: null argument");
  }
  if (s->events_created) {
    return SetError(GJXL_B200_FAILED_PRECONDITION,
                    "session_kernel_count: needs a session without stage profiling");
  }
  // Capture one analysis into a graph (nothing executes) and count its
  // kernel nodes.
  cudaStream_t st = nullptr;
  GJXL_TRY(CheckCuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking),
                     "session_kernel_count: stream"));
  int status = CheckCuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed),
                         "session_kernel_count: begin capture");
  const int run_status = status == GJXL_B200_OK ? Run(s, pixels, row_stride, channels, st)
                                                : status;
  cudaGraph_t graph = nullptr;
  if (status == GJXL_B200_OK) {
    status = CheckCuda(cudaStreamEndCapture(st, &graph), "session_kernel_count: end capture");
  }
  if (status == GJXL_B200_OK) status = run_status;
  size_t count = 0;
  if (status == GJXL_B200_OK) {
    size_t nodes = 0;
    status = CheckCuda(cudaGraphGetNodes(graph, nullptr, &nodes), "session_kernel_count: nodes");
    std::vector<cudaGraphNode_t> list(nodes);
    if (status == GJXL_B200_OK && nodes > 0) {
      status = CheckCuda(cudaGraphGetNodes(graph, list.data(), &nodes),
                         "session_kernel_count: nodes");
    }
    for (size_t i = 0; status == GJXL_B200_OK && i < nodes; ++i) {
      cudaGraphNodeType type;
      status = CheckCuda(cudaGraphNodeGetType(list[i], &type), "session_kernel_count: type");
      if (status == GJXL_B200_OK && type == cudaGraphNodeTypeKernel) ++count;
    }
  }
  if (graph != nullptr) cudaGraphDestroy(graph);
  cudaStreamDestroy(st);
  if (status == GJXL_B200_OK) *kernels = count;
  return status;
}
