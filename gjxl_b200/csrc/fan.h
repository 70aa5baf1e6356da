// Fork/join of independent launches (the per-family kernels of one stage)
// onto side streams of the session, so that their ramp-up and tail waves
// overlap. Inside a stream capture the fork and join events become graph
// dependencies; outside one they order plain stream work.
#pragma once

#include <cuda_runtime.h>

namespace gjxl_b200 {

struct StreamFan {
  static constexpr int kSide = 3;
  cudaStream_t main = nullptr;
  cudaStream_t side[kSide] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kSide] = {};
  bool enabled() const { return fork != nullptr; }
  // Stream of the i-th of a set of independent launches.
  cudaStream_t For(int i) const {
    const int slot = i % (kSide + 1);
    return !enabled() || slot == 0 ? main : side[slot - 1];
  }
};

// Side streams wait for the work queued on the main stream so far.
inline cudaError_t FanFork(const StreamFan* f) {
  if (f == nullptr || !f->enabled()) return cudaSuccess;
  cudaError_t e = cudaEventRecord(f->fork, f->main);
  for (int i = 0; i < StreamFan::kSide && e == cudaSuccess; ++i) {
    e = cudaStreamWaitEvent(f->side[i], f->fork, 0);
  }
  return e;
}

// The main stream waits for everything queued on the side streams.
inline cudaError_t FanJoin(const StreamFan* f) {
  if (f == nullptr || !f->enabled()) return cudaSuccess;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < StreamFan::kSide && e == cudaSuccess; ++i) {
    e = cudaEventRecord(f->join[i], f->side[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(f->main, f->join[i], 0);
  }
  return e;
}

}  // namespace gjxl_b200
