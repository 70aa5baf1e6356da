// Analysis session: buffers + stage orchestration on one stream.
//
// Stage order follows the reference's CPU pipeline
// (src/codestream/workflow.cpp:700-730 for input preparation,
// src/codec/quantization_pipeline.cpp:155-213 and :429-560 for the
// quantization pipeline): packed sRGB -> linear RGB + padded XYB ->
// quantization-matrix statistics -> initial quant field (on the pre-Gaborish
// XYB) -> inverse Gaborish -> initial CfL -> AC-strategy candidate costs ->
// greedy merge.

#include "session.h"

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "host_util.h"

namespace gjxl_b200 {
namespace {

enum Stage : int {
  kStagePrepare = 0,
  kStageStats,
  kStageInitialQuant,
  kStageGaborishInverse,
  kStageInitialCfl,
  kStageAcCosts,
  kStageAcMerge,
  kStageCount,
};

const char* const kStageNames[kStageCount] = {
  "prepare_input", "matrix_scale_stats", "initial_quant_field", "gaborish_inverse",
  "initial_cfl", "ac_strategy_costs", "ac_strategy_merge",
};

size_t Align(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace

struct Session {
  size_t width = 0, height = 0, pw = 0, ph = 0, bx = 0, by = 0, tx = 0, ty = 0;
  gjxl_b200_options options{};
  // Device arena and views into it.
  void* arena = nullptr;
  size_t arena_bytes = 0;
  uint8_t* pixels = nullptr;
  size_t pixel_capacity = 0;
  float* linear = nullptr;  // 3 planes, stride lin_stride, pitch lin_pitch
  size_t lin_stride = 0, lin_pitch = 0;
  float* opsin = nullptr;  // padded, stride pw
  float* pre = nullptr;    // Gaborish-inverted
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
  // Pinned host mirrors of the outputs.
  uint8_t* host_cells = nullptr;
  float* host_quant = nullptr;
  int8_t* host_cfl = nullptr;
  float* host_stats = nullptr;
  uint32_t* host_error = nullptr;
  cudaEvent_t events[kStageCount + 1] = {};
  bool events_created = false;

  ~Session() {
    if (arena) cudaFree(arena);
    if (host_cells) cudaFreeHost(host_cells);
    if (events_created) {
      for (auto& e : events) cudaEventDestroy(e);
    }
  }
};

namespace {

int Allocate(Session* s) {
  const size_t plane = s->pw * s->ph;
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
  };
  size_t total = 0;
  for (const Item& item : items) total = Align(total, 256) + item.bytes;
  int status = CheckCuda(cudaMalloc(&s->arena, total), "session: cudaMalloc");
  if (status != GJXL_B200_OK) return status;
  s->arena_bytes = total;
  size_t offset = 0;
  for (const Item& item : items) {
    offset = Align(offset, 256);
    *item.ptr = static_cast<unsigned char*>(s->arena) + offset;
    offset += item.bytes;
  }
  // Pinned host mirrors: cells, quant field, CfL maps, stats, error word.
  const size_t host_bytes = Align(blocks, 16) + Align(blocks * sizeof(float), 16) +
                            Align(2 * tiles, 16) + 16 + 16;
  void* host = nullptr;
  status = CheckCuda(cudaMallocHost(&host, host_bytes), "session: cudaMallocHost");
  if (status != GJXL_B200_OK) return status;
  auto* h = static_cast<unsigned char*>(host);
  s->host_cells = h;
  h += Align(blocks, 16);
  s->host_quant = reinterpret_cast<float*>(h);
  h += Align(blocks * sizeof(float), 16);
  s->host_cfl = reinterpret_cast<int8_t*>(h);
  h += Align(2 * tiles, 16);
  s->host_stats = reinterpret_cast<float*>(h);
  h += 16;
  s->host_error = reinterpret_cast<uint32_t*>(h);
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

int Run(Session* s, const uint8_t* pixels, size_t row_stride, int channels,
        cudaStream_t stream) {
  int status = CheckCuda(cudaMemsetAsync(s->error, 0, sizeof(uint32_t), stream),
                         "session: clear error");
  if (status != GJXL_B200_OK) return status;
  const float target = s->options.butteraugli_target;
  Mark(s, kStagePrepare, stream);
  status = gjxl_b200_prepare_input(pixels, s->width, s->height, row_stride, channels,
                                   s->options.intensity_target, s->linear, s->lin_stride,
                                   s->lin_pitch, s->opsin, s->pw, s->pitch, s->pw, s->ph,
                                   s->error, stream);
  if (status != GJXL_B200_OK) return status;
  Mark(s, kStageStats, stream);
  status = gjxl_b200_matrix_scale_stats(s->opsin, s->pw, s->pitch, s->width, s->height,
                                        s->stats, stream);
  if (status != GJXL_B200_OK) return status;
  Mark(s, kStageInitialQuant, stream);
  // Initial quantization samples the pre-Gaborish image at the full target
  // (Gaborish is on for efforts >= 5: quantization_pipeline.cpp:452-456).
  status = LaunchInitialQuantField(s->opsin, s->pw, s->pitch, s->pw, s->ph, target, 1.0f,
                                   s->quant, s->strategy_mask, s->pixel_mask, s->pw,
                                   s->iq_scratch, s->error, stream);
  if (status != GJXL_B200_OK) return status;
  Mark(s, kStageGaborishInverse, stream);
  const float multipliers[3] = {1.0f, 1.0f, 1.0f};
  status = LaunchGaborishInverse(s->opsin, s->pw, s->pitch, s->pre, s->pw, s->pitch, s->pw,
                                 s->ph, multipliers, s->error, stream);
  if (status != GJXL_B200_OK) return status;
  Mark(s, kStageInitialCfl, stream);
  status = LaunchInitialCfl(s->pre, s->pw, s->pitch, s->pw, s->ph, s->y_to_x, s->y_to_b, stream);
  if (status != GJXL_B200_OK) return status;
  Mark(s, kStageAcCosts, stream);
  const bool dense = s->options.effort >= 10;
  status = LaunchAcStrategyCosts(s->pre, s->pw, s->pitch, s->pw, s->ph, s->quant, s->pixel_mask,
                                 s->pw, s->y_to_x, s->y_to_b, target, dense, s->costs, s->error,
                                 stream);
  if (status != GJXL_B200_OK) return status;
  Mark(s, kStageAcMerge, stream);
  status = LaunchAcStrategySearch(s->costs, s->pw, s->ph, target, dense, s->cells, s->error,
                                  stream);
  if (status != GJXL_B200_OK) return status;
  Mark(s, kStageCount, stream);
  return GJXL_B200_OK;
}

int CopyOutputs(Session* s, cudaStream_t stream) {
  const size_t blocks = s->bx * s->by, tiles = s->tx * s->ty;
  const struct {
    void* dst;
    const void* src;
    size_t bytes;
  } copies[] = {
    {s->host_cells, s->cells, blocks},
    {s->host_quant, s->quant, blocks * sizeof(float)},
    {s->host_cfl, s->y_to_x, tiles},
    {s->host_cfl + tiles, s->y_to_b, tiles},
    {s->host_stats, s->stats, 3 * sizeof(float)},
    {s->host_error, s->error, sizeof(uint32_t)},
  };
  for (const auto& c : copies) {
    int status = CheckCuda(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, stream),
                           "session: output copy");
    if (status != GJXL_B200_OK) return status;
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
}

extern "C" int gjxl_b200_session_create(size_t width, size_t height,
                                        const gjxl_b200_options* options,
                                        gjxl_b200_session** out) {
  ClearLastError();
  if (out == nullptr || width == 0 || height == 0 || width > (1u << 20) || height > (1u << 20)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_create: invalid extent");
  }
  *out = nullptr;
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
  if (o.effort < 5 || o.effort > 10) {
    return SetError(GJXL_B200_UNSUPPORTED,
                    "session_create: efforts 5-10 (mixed-transform search) are supported");
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
  int status = Allocate(s);
  if (status != GJXL_B200_OK) {
    delete s;
    return status;
  }
  *out = s;
  return GJXL_B200_OK;
}

extern "C" void gjxl_b200_session_destroy(gjxl_b200_session* session) { delete session; }

extern "C" int gjxl_b200_session_analyze(gjxl_b200_session* s, const uint8_t* pixels,
                                         size_t row_stride, int channels, void* stream) {
  ClearLastError();
  if (s == nullptr || pixels == nullptr) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_analyze: null argument");
  }
  return Run(s, pixels, row_stride, channels, static_cast<cudaStream_t>(stream));
}

extern "C" int gjxl_b200_session_analyze_host(gjxl_b200_session* s, const uint8_t* host_pixels,
                                              size_t row_stride, int channels, void* stream) {
  ClearLastError();
  if (s == nullptr || host_pixels == nullptr || (channels != 3 && channels != 4) ||
      row_stride < s->width * channels) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_analyze_host: invalid arguments");
  }
  const size_t bytes = row_stride * (s->height - 1) + s->width * channels;
  if (bytes > s->pixel_capacity) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "session_analyze_host: row stride too large");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int status = CheckCuda(cudaMemcpyAsync(s->pixels, host_pixels, bytes, cudaMemcpyHostToDevice,
                                         st), "session: input upload");
  if (status != GJXL_B200_OK) return status;
  status = Run(s, s->pixels, row_stride, channels, st);
  if (status != GJXL_B200_OK) return status;
  return CopyOutputs(s, st);
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
  out->y_to_x = s->y_to_x;
  out->y_to_b = s->y_to_b;
  out->strategy_cells = s->cells;
  out->matrix_scale_stats = s->stats;
  out->device_error = s->error;
  out->host_strategy_cells = s->host_cells;
  out->host_initial_quant_field = s->host_quant;
  out->host_y_to_x = s->host_cfl;
  out->host_y_to_b = s->host_cfl + s->tx * s->ty;
  out->host_matrix_scale_stats = s->host_stats;
  out->host_device_error = s->host_error;
  out->device_bytes = s->arena_bytes;
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
    int status = CheckCuda(cudaEventElapsedTime(&milliseconds[i], s->events[i], s->events[i + 1]),
                           "session_stage_times");
    if (status != GJXL_B200_OK) return status;
  }
  return n;
}

extern "C" const char* gjxl_b200_stage_name(int stage) {
  return stage >= 0 && stage < kStageCount ? kStageNames[stage] : nullptr;
}
