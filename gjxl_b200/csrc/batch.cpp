// Row N3: batched analysis of many images of uneven sizes.
//
// Mirrors the reference's VarDctBatchEncoder (src/codestream/batch_workflow.h:
// 74-118): a persistent bounded-concurrency driver whose Encode call runs
// every request, preserves request order in the results, reports failures per
// image and times each image as queue / service / ready. As there, images do
// not share a launch: every image runs its own analysis session. The B200
// form differs in what runs concurrently. The reference distributes worker
// threads over two CUDA lanes; here each lane is a CUDA stream whose images'
// analyses are captured graphs, so one host thread enqueues the whole batch
// and the GPU's work distributor interleaves the lanes' kernels across the
// SMs (small images, which cannot fill the GPU alone, run beside large ones).
//
// Scheduling: requests in the given order or largest first, each placed on
// the lane with the fewest pixels so far (longest-processing-time rule). An
// autotuner runs the batch at several lane counts and orders and keeps the
// fastest.
//
// Memory: a lane runs one image at a time, so all of a lane's sessions carve
// their working buffers from one region sized for the lane's largest image
// (gjxl_b200_session_create_in); the device footprint is the sum over lanes
// of their largest images, not over all images. Sessions are pooled per
// (lane, extent) and reused by later calls, so a repeated batch replays
// captured graphs. A session's device views hold its image's results until
// the lane's next image; host-input results stay in each session's own
// pinned mirrors.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <thread>
#include <utility>
#include <vector>

#include "gjxl_b200.h"
#include "host_util.h"

namespace gjxl_b200 {
namespace {

constexpr int kMaxLanes = 16;

struct Lane {
  void* memory = nullptr;
  size_t bytes = 0;
  std::map<std::pair<size_t, size_t>, std::vector<gjxl_b200_session*>> pools;

  void Release() {
    for (auto& [extent, pool] : pools)
      for (gjxl_b200_session* s : pool) gjxl_b200_session_destroy(s);
    pools.clear();
    if (memory) cudaFree(memory);
    memory = nullptr;
    bytes = 0;
  }
};

}  // namespace
}  // namespace gjxl_b200

using namespace gjxl_b200;

struct gjxl_b200_batch {
  gjxl_b200_options options;
  int lanes = 2;
  int largest_first = 1;
  Lane lane[kMaxLanes];
  std::map<std::pair<size_t, size_t>, size_t> session_bytes;  // per extent
  cudaStream_t streams[kMaxLanes] = {};
  cudaStream_t main = nullptr;
  cudaEvent_t t0 = nullptr, lane_done[kMaxLanes] = {};
  std::vector<cudaEvent_t> begin, end;
  // Each image's error words, copied out right after its analysis (a lane's
  // sessions share memory, so the words do not survive the lane's next image).
  uint32_t* error_slots = nullptr;
  size_t error_capacity = 0;
  std::vector<uint32_t> host_errors;
  double last_ms = 0.0;

  ~gjxl_b200_batch() {
    for (Lane& l : lane) l.Release();
    for (cudaStream_t s : streams)
      if (s) cudaStreamDestroy(s);
    if (main) cudaStreamDestroy(main);
    if (t0) cudaEventDestroy(t0);
    for (cudaEvent_t e : lane_done)
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : begin) cudaEventDestroy(e);
    for (cudaEvent_t e : end) cudaEventDestroy(e);
    if (error_slots) cudaFree(error_slots);
  }
};

extern "C" int gjxl_b200_batch_schedule(size_t count, const size_t* pixels, int lanes,
                                        int largest_first, int* lane_of, size_t* order) {
  ClearLastError();
  if ((count > 0 && (pixels == nullptr || lane_of == nullptr || order == nullptr)) ||
      lanes < 1 || lanes > kMaxLanes) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "batch_schedule: invalid arguments");
  }
  for (size_t i = 0; i < count; ++i) order[i] = i;
  if (largest_first) {
    std::stable_sort(order, order + count,
                     [&](size_t a, size_t b) { return pixels[a] > pixels[b]; });
  }
  std::vector<size_t> load(static_cast<size_t>(lanes), 0);
  for (size_t k = 0; k < count; ++k) {
    const size_t i = order[k];
    const int lane = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
    lane_of[i] = lane;
    load[static_cast<size_t>(lane)] += pixels[i];
  }
  return GJXL_B200_OK;
}

extern "C" int gjxl_b200_batch_create(int max_in_flight, const gjxl_b200_options* options,
                                      gjxl_b200_batch** out) {
  ClearLastError();
  if (out == nullptr || max_in_flight < 0 || max_in_flight > kMaxLanes) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "batch_create: invalid arguments");
  }
  auto* b = new (std::nothrow) gjxl_b200_batch();
  if (b == nullptr) return SetError(GJXL_B200_OUT_OF_MEMORY, "batch_create: host allocation");
  if (options != nullptr) {
    b->options = *options;
  } else {
    gjxl_b200_default_options(&b->options);
  }
  b->options.profile_stages = 0;
  b->lanes = max_in_flight == 0 ? 2 : max_in_flight;
  int status = CheckCuda(cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking),
                         "batch_create: stream");
  for (int i = 0; i < kMaxLanes && status == GJXL_B200_OK; ++i) {
    status = CheckCuda(cudaStreamCreateWithFlags(&b->streams[i], cudaStreamNonBlocking),
                       "batch_create: lane stream");
    if (status == GJXL_B200_OK) {
      status = CheckCuda(cudaEventCreateWithFlags(&b->lane_done[i], cudaEventDisableTiming),
                         "batch_create: event");
    }
  }
  if (status == GJXL_B200_OK) status = CheckCuda(cudaEventCreate(&b->t0), "batch_create: event");
  if (status != GJXL_B200_OK) {
    delete b;
    return status;
  }
  *out = b;
  return GJXL_B200_OK;
}

extern "C" void gjxl_b200_batch_destroy(gjxl_b200_batch* batch) { delete batch; }

extern "C" int gjxl_b200_batch_set_schedule(gjxl_b200_batch* b, int lanes, int largest_first) {
  ClearLastError();
  if (b == nullptr || lanes < 1 || lanes > kMaxLanes) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "batch_set_schedule: invalid arguments");
  }
  b->lanes = lanes;
  b->largest_first = largest_first ? 1 : 0;
  return GJXL_B200_OK;
}

namespace {

int Run(gjxl_b200_batch* b, const gjxl_b200_batch_request* requests, size_t count,
        int host_input, gjxl_b200_batch_result* results) {
  std::vector<size_t> pixels(count), order(count);
  std::vector<int> lane_of(count);
  for (size_t i = 0; i < count; ++i) pixels[i] = requests[i].width * requests[i].height;
  int status = gjxl_b200_batch_schedule(count, pixels.data(), b->lanes, b->largest_first,
                                        lane_of.data(), order.data());
  if (status != GJXL_B200_OK) return status;
  std::vector<std::vector<size_t>> queues(static_cast<size_t>(b->lanes));
  for (size_t k = 0; k < count; ++k)
    queues[static_cast<size_t>(lane_of[order[k]])].push_back(order[k]);

  // Each lane's region covers its largest image; a lane that must grow
  // releases its sessions first (they point into the old region).
  for (int l = 0; l < b->lanes; ++l) {
    size_t need = 0;
    for (size_t i : queues[static_cast<size_t>(l)]) {
      const auto key = std::make_pair(requests[i].width, requests[i].height);
      auto it = b->session_bytes.find(key);
      if (it == b->session_bytes.end()) {
        size_t bytes = 0;
        status = gjxl_b200_session_device_bytes(key.first, key.second, &b->options, &bytes);
        if (status != GJXL_B200_OK) return status;
        it = b->session_bytes.emplace(key, bytes).first;
      }
      need = std::max(need, it->second);
    }
    Lane& lane = b->lane[l];
    if (need > lane.bytes) {
      lane.Release();
      status = CheckCuda(DeviceMalloc(&lane.memory, need), "batch: lane memory");
      if (status != GJXL_B200_OK) return status;
      lane.bytes = need;
    }
  }
  // Sessions: the k-th image of an extent on a lane takes the lane pool's
  // k-th session.
  std::vector<gjxl_b200_session*> sessions(count, nullptr);
  for (int l = 0; l < b->lanes; ++l) {
    Lane& lane = b->lane[l];
    std::map<std::pair<size_t, size_t>, size_t> taken;
    for (size_t i : queues[static_cast<size_t>(l)]) {
      const auto key = std::make_pair(requests[i].width, requests[i].height);
      std::vector<gjxl_b200_session*>& pool = lane.pools[key];
      const size_t k = taken[key]++;
      if (k == pool.size()) {
        gjxl_b200_options o = b->options;
        o.butteraugli_target = requests[i].butteraugli_target;
        gjxl_b200_session* s = nullptr;
        status = gjxl_b200_session_create_in(key.first, key.second, &o, lane.memory, lane.bytes,
                                             &s);
        if (status != GJXL_B200_OK) return status;
        pool.push_back(s);
      }
      sessions[i] = pool[k];
      status =
        gjxl_b200_session_set_butteraugli_target(sessions[i], requests[i].butteraugli_target);
      if (status != GJXL_B200_OK) return status;
    }
  }
  if (b->error_capacity < count) {
    if (b->error_slots) cudaFree(b->error_slots);
    b->error_slots = nullptr;
    b->error_capacity = 0;
    status = CheckCuda(DeviceMalloc(reinterpret_cast<void**>(&b->error_slots),
                                    count * 4 * sizeof(uint32_t)),
                       "batch: error slots");
    if (status != GJXL_B200_OK) return status;
    b->error_capacity = count;
  }
  b->host_errors.assign(4 * count, 0);
  while (b->begin.size() < count) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    status = CheckCuda(cudaEventCreate(&e0), "batch: event");
    if (status == GJXL_B200_OK) status = CheckCuda(cudaEventCreate(&e1), "batch: event");
    if (status != GJXL_B200_OK) return status;
    b->begin.push_back(e0);
    b->end.push_back(e1);
  }

  // Arrival: every lane starts from t0 on the batch stream.
  status = CheckCuda(cudaEventRecord(b->t0, b->main), "batch: t0");
  for (int l = 0; l < b->lanes && status == GJXL_B200_OK; ++l)
    status = CheckCuda(cudaStreamWaitEvent(b->streams[l], b->t0, 0), "batch: lane start");
  if (status != GJXL_B200_OK) return status;
  std::vector<int> image_status(count, GJXL_B200_OK);
  auto analyze = [&](size_t i, cudaStream_t st) {
    const gjxl_b200_batch_request& r = requests[i];
    cudaEventRecord(b->begin[i], st);
    image_status[i] =
      host_input ? gjxl_b200_session_analyze_host(sessions[i], r.pixels, r.row_stride,
                                                  r.channels, st)
                 : gjxl_b200_session_analyze(sessions[i], r.pixels, r.row_stride, r.channels, st);
    cudaEventRecord(b->end[i], st);
    if (!host_input && image_status[i] == GJXL_B200_OK) {
      gjxl_b200_outputs o;
      gjxl_b200_session_outputs(sessions[i], &o);
      cudaMemcpyAsync(b->error_slots + 4 * i, o.device_error, 3 * sizeof(uint32_t),
                      cudaMemcpyDeviceToDevice, st);
    }
  };
  if (host_input) {
    // analyze_host returns once its results are on the host: one thread per
    // lane keeps the lanes' copies and analyses overlapping.
    std::vector<std::thread> threads;
    for (int l = 0; l < b->lanes; ++l) {
      threads.emplace_back([&, l] {
        for (size_t i : queues[static_cast<size_t>(l)]) analyze(i, b->streams[l]);
      });
    }
    for (auto& t : threads) t.join();
  } else {
    // Interleaved enqueue: every lane's first image, then every second ...
    for (size_t k = 0;; ++k) {
      bool any = false;
      for (int l = 0; l < b->lanes; ++l) {
        if (k < queues[static_cast<size_t>(l)].size()) {
          analyze(queues[static_cast<size_t>(l)][k], b->streams[l]);
          any = true;
        }
      }
      if (!any) break;
    }
  }
  for (int l = 0; l < b->lanes && status == GJXL_B200_OK; ++l) {
    status = CheckCuda(cudaEventRecord(b->lane_done[l], b->streams[l]), "batch: lane done");
    if (status == GJXL_B200_OK)
      status = CheckCuda(cudaStreamWaitEvent(b->main, b->lane_done[l], 0), "batch: join");
  }
  if (status == GJXL_B200_OK)
    status = CheckCuda(cudaStreamSynchronize(b->main), "batch: completion");
  if (status == GJXL_B200_OK && !host_input) {
    status = CheckCuda(cudaMemcpy(b->host_errors.data(), b->error_slots,
                                  4 * count * sizeof(uint32_t), cudaMemcpyDeviceToHost),
                       "batch: error words");
  }
  if (status != GJXL_B200_OK) return status;
  float total = 0.0f;
  for (size_t i = 0; i < count; ++i) {
    float queue = 0.0f, service = 0.0f, ready = 0.0f;
    cudaEventElapsedTime(&queue, b->t0, b->begin[i]);
    cudaEventElapsedTime(&service, b->begin[i], b->end[i]);
    cudaEventElapsedTime(&ready, b->t0, b->end[i]);
    total = std::max(total, ready);
    int st = image_status[i];
    if (st == GJXL_B200_OK && !host_input &&
        (b->host_errors[4 * i] | b->host_errors[4 * i + 1] | b->host_errors[4 * i + 2]) != 0) {
      st = GJXL_B200_DEVICE_ERROR;
    }
    if (results != nullptr) {
      results[i].status = st;
      results[i].session = sessions[i];
      results[i].lane = lane_of[i];
      results[i].queue_ms = queue;
      results[i].service_ms = service;
      results[i].ready_ms = ready;
    }
  }
  b->last_ms = total;
  return GJXL_B200_OK;
}

}  // namespace

extern "C" int gjxl_b200_batch_analyze(gjxl_b200_batch* b,
                                       const gjxl_b200_batch_request* requests, size_t count,
                                       int host_input, gjxl_b200_batch_result* results,
                                       double* batch_ms) {
  ClearLastError();
  if (b == nullptr || (count > 0 && requests == nullptr)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "batch_analyze: invalid arguments");
  }
  for (size_t i = 0; i < count; ++i) {
    const gjxl_b200_batch_request& r = requests[i];
    if (r.pixels == nullptr || r.width == 0 || r.height == 0 ||
        (r.channels != 3 && r.channels != 4) || r.row_stride < r.width * r.channels ||
        !(r.butteraugli_target > 0.0f)) {
      return SetError(GJXL_B200_INVALID_ARGUMENT, "batch_analyze: invalid request");
    }
  }
  const int status = Run(b, requests, count, host_input, results);
  if (status == GJXL_B200_OK && batch_ms != nullptr) *batch_ms = b->last_ms;
  return status;
}

extern "C" int gjxl_b200_batch_autotune(gjxl_b200_batch* b,
                                        const gjxl_b200_batch_request* requests, size_t count,
                                        const int* lane_counts, size_t lane_count_count,
                                        int* lanes_out, int* largest_first_out) {
  ClearLastError();
  if (b == nullptr || requests == nullptr || count == 0 || lane_counts == nullptr ||
      lane_count_count == 0) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "batch_autotune: invalid arguments");
  }
  double best = 0.0;
  int best_lanes = b->lanes, best_order = b->largest_first;
  for (size_t k = 0; k < lane_count_count; ++k) {
    for (int order = 0; order < 2; ++order) {
      int status = gjxl_b200_batch_set_schedule(b, lane_counts[k], order);
      if (status != GJXL_B200_OK) return status;
      // The first run plans (sessions, graphs); the second is timed.
      double ms = 0.0;
      for (int rep = 0; rep < 2 && status == GJXL_B200_OK; ++rep)
        status = gjxl_b200_batch_analyze(b, requests, count, 0, nullptr, &ms);
      if (status != GJXL_B200_OK) return status;
      if (best == 0.0 || ms < best) {
        best = ms;
        best_lanes = lane_counts[k];
        best_order = order;
      }
    }
  }
  b->lanes = best_lanes;
  b->largest_first = best_order;
  // Lanes past the chosen count give their memory back.
  for (int l = best_lanes; l < kMaxLanes; ++l) b->lane[l].Release();
  if (lanes_out != nullptr) *lanes_out = best_lanes;
  if (largest_first_out != nullptr) *largest_first_out = best_order;
  return GJXL_B200_OK;
}

extern "C" size_t gjxl_b200_batch_device_bytes(const gjxl_b200_batch* b) {
  if (b == nullptr) return 0;
  size_t bytes = 0;
  for (const Lane& l : b->lane) bytes += l.bytes;
  return bytes;
}
