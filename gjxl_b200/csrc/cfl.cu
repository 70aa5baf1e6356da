// Row a5: initial chroma-from-luma map (y_to_x, y_to_b per 64x64 tile).
//
// Restates ComputeInitialColorCorrelationMap (src/codec/chroma_from_luma.cpp:
// 434-525), the CPU path's initial CfL: per tile, every 8x8 block's DCT8
// coefficients of the three channels (double-precision matrix DCT,
// src/codec/dct.cpp:135-180) with the LLF coefficient zeroed, scaled by the
// DCT8 inverse dequant weights of the X (resp. B) matrix
// (AppendStrategyCoefficients, :306-372); then the damped Newton solve of
// FindBestMultiplier (:98-151) with CflDerivatives (:22-79), whose four-lane
// float sums keep the reference's element order, and QuantizeMultiplier.
//
// One CTA of 256 threads per tile. Phase 1: each warp transforms (block,
// channel) pairs — lane l owns row-pass outputs l and l+32 and gathers the
// column inputs with double shuffles. Phase 2: per Newton iteration warps
// 1-7 evaluate the derivative terms of the next chunk while warp 0 adds the
// current one in order, twelve lanes per map, each owning one of the 3 sums
// x 4 lanes.

#include <cmath>
#include <cstring>

#include "common.cuh"
#include "host_util.h"
#include "tables.h"

namespace gjxl_b200 {
namespace {

constexpr int kTileValues = 64 * 64;  // up to 64 blocks of 64 coefficients
constexpr int kCflChunk = 128;        // elements per shared term chunk (divides kTileValues)

struct CflParams {
  const float* opsin;  // Gaborish-inverted padded XYB
  size_t stride, pitch;
  uint32_t blocks_x, blocks_y, tiles_x, tiles_y;
  const double* fwd;    // DCT8 forward basis [freq][sample]
  const float* inv_x;   // DCT8 inverse dequant, X channel
  const float* inv_b;   // DCT8 inverse dequant, B channel
  int iterations;       // Newton iteration limit (20)
  int8_t* y_to_x;
  int8_t* y_to_b;
};

__device__ __forceinline__ double ShflD(double v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

// QuantizeMultiplier (chroma_from_luma.cpp:81-96).
__device__ __forceinline__ int8_t QuantizeMultiplier(float x) {
  const float kTowardsZero = 2.6f;
  if (x >= kTowardsZero) {
    x -= kTowardsZero;
  } else if (x <= -kTowardsZero) {
    x += kTowardsZero;
  } else {
    x = 0.0f;
  }
  return static_cast<int8_t>(fminf(fmaxf(roundf(x), -128.0f), 127.0f));
}

__global__ void __launch_bounds__(256) InitialCflKernel(const __grid_constant__ CflParams p) {
  // [4][kTileValues]: per element a = luma / 84 and b = base * luma - chroma
  // for the y_to_x problem (base 0) and the y_to_b problem (base 1).
  extern __shared__ __align__(16) float values[];
  const int tile = blockIdx.x;
  const int tx = tile % p.tiles_x, ty = tile / p.tiles_x;
  const int bx0 = tx * 8, by0 = ty * 8;
  const int tw = min(8, static_cast<int>(p.blocks_x) - bx0);
  const int th = min(8, static_cast<int>(p.blocks_y) - by0);
  const int blocks = tw * th;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* luma_x = values;
  float* chroma_x = values + kTileValues;
  float* luma_b = values + 2 * kTileValues;
  float* chroma_b = values + 3 * kTileValues;
  __shared__ float y_coef[8][64];  // per warp: Y coefficients of the current block

  // Phase 1: DCT8 of every block, Y first so X/B can pair with it.
  for (int b = warp; b < blocks; b += 8) {
    const int bx = bx0 + b % tw, by = by0 + b / tw;
    for (int c = 1; c < 4; ++c) {
      const int ch = c == 1 ? 1 : c == 2 ? 2 : 0;  // order: Y, B, X
      const float* src = p.opsin + ch * p.pitch + static_cast<size_t>(by * 8) * p.stride + bx * 8;
      // Row pass: T[y][u] = sum_x pixel[y][x] * basis[u][x], outputs l, l+32.
      double t[2];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int o = lane + 32 * k, y = o >> 3, u = o & 7;
        const float* row = src + static_cast<size_t>(y) * p.stride;
        double sum = 0.0;
#pragma unroll
        for (int x = 0; x < 8; ++x) sum += static_cast<double>(row[x]) * __ldg(p.fwd + u * 8 + x);
        t[k] = sum;
      }
      // Column pass: coef[v][u] = sum_y basis[v][y] * T[y][u]; storage index
      // of a square transform is u * 8 + v.
      float coef[2];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int o = lane + 32 * k, v = o >> 3, u = o & 7;
        double sum = 0.0;
#pragma unroll
        for (int y = 0; y < 8; ++y) {
          const int src_index = y * 8 + u;  // T index
          const double lo = ShflD(t[0], src_index & 31);
          const double hi = ShflD(t[1], src_index & 31);
          const double value = src_index < 32 ? lo : hi;
          sum += __ldg(p.fwd + v * 8 + y) * value;
        }
        coef[k] = static_cast<float>(sum);
      }
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int o = lane + 32 * k, v = o >> 3, u = o & 7;
        const int index = u * 8 + v;
        float value = index == 0 ? 0.0f : coef[k];  // LLF zeroed
        const int at = b * 64 + index;
        if (ch == 1) {
          y_coef[warp][index] = value;
        } else if (ch == 2) {
          __syncwarp();
          const float luma = y_coef[warp][index] * __ldg(p.inv_b + index) * 1.0f;
          const float chroma = value * __ldg(p.inv_b + index) * 1.0f;
          luma_b[at] = luma / 84.0f;
          chroma_b[at] = 1.0f * luma - chroma;
        } else {
          const float luma = y_coef[warp][index] * __ldg(p.inv_x + index) * 1.0f;
          const float chroma = value * __ldg(p.inv_x + index) * 1.0f;
          luma_x[at] = luma / 84.0f;
          chroma_x[at] = 0.0f * luma - chroma;
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();

  // Phase 2: FindBestMultiplier (non-fast) for both maps. The element terms
  // of the three derivative sums (center, +eps, -eps) are computed a chunk of
  // kCflChunk elements at a time into one of two shared buffers while warp 0
  // adds the previous chunk in the reference's order: lanes 0..11 solve
  // y_to_x and 12..23 y_to_b, lane 4 * kind + slot of a group owning
  // derivative sum `kind` over the elements i = slot (mod 4), in increasing
  // i. One barrier per chunk. Elements skipped by the reference contribute
  // +0.0, which leaves the (never -0.0) sum unchanged.
  // Rows padded by 4 floats: the 24 summing lanes read 24 distinct banks.
  __shared__ float terms[2][2][3][kCflChunk + 4];
  __shared__ float solution[2];
  __shared__ int solved[2];
  const int count = blocks * 64;
  const int chunks = (count + kCflChunk - 1) / kCflChunk;
  const float kDistanceMultiplierAc = 1.0e-9f;
  const float kEpsilon = 100.0f;
  if (threadIdx.x < 2) {
    solution[threadIdx.x] = 0.0f;
    solved[threadIdx.x] = 0;
  }
  const int group = lane / 12;  // warp 0: 0 y_to_x, 1 y_to_b, 2 idle lanes
  const int member = lane % 12;
  const int kind = member / 4, slot = member % 4;
  __syncthreads();
  // Terms of chunk `chunk` into buffer `buffer`, by the threads first..255,
  // two adjacent elements per item (count is a multiple of 64, so pairs
  // never straddle its end).
  const auto produce = [&](int chunk, int buffer, int first, const float (&x_map)[2],
                           const int (&done_map)[2]) {
    for (int t = static_cast<int>(threadIdx.x) - first; t < kCflChunk;
         t += blockDim.x - first) {
      const int map = t / (kCflChunk / 2), e = 2 * (t % (kCflChunk / 2));
      const int i = chunk * kCflChunk + e;
      if (done_map[map] || i >= count) continue;
      const float* A = map == 0 ? luma_x : luma_b;       // a = luma / 84
      const float* Bv = map == 0 ? chroma_x : chroma_b;  // b = base * luma - chroma
      const float2 a2 = *reinterpret_cast<const float2*>(A + i);
      const float2 b2 = *reinterpret_cast<const float2*>(Bv + i);
      const float x = x_map[map], xp = x + kEpsilon, xm = x - kEpsilon;
      float* out = terms[buffer][map][0] + e;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const float a = q == 0 ? a2.x : a2.y, b = q == 0 ? b2.x : b2.y;
        const float center = fmaf(a, x, b);
        const bool skip = fabsf(center) >= 100.0f;
        const float scale = (2.0f / 3.0f) * a;
        const float r[3] = {center, fmaf(a, xp, b), fmaf(a, xm, b)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          float d = scale * (fabsf(r[k]) + 1.0f);
          d = r[k] < 0.0f ? -d : d;
          out[k * (kCflChunk + 4) + q] = skip ? 0.0f : d;
        }
      }
    }
  };
  for (int iteration = 0; iteration < p.iterations; ++iteration) {
    if (solved[0] && solved[1]) break;
    const float x_map[2] = {solution[0], solution[1]};
    const int done_map[2] = {solved[0], solved[1]};
    float lane_sum = 0.0f;
    produce(0, 0, 0, x_map, done_map);
    __syncthreads();
    for (int chunk = 0; chunk < chunks; ++chunk) {
      if (warp == 0) {
        if (group < 2 && !done_map[group]) {
          const float* t = terms[chunk & 1][group][kind];
          const int limit = min(kCflChunk, count - chunk * kCflChunk);
#pragma unroll 8
          for (int e = slot; e < limit; e += 4) lane_sum += t[e];
        }
      } else if (chunk + 1 < chunks) {
        produce(chunk + 1, (chunk + 1) & 1, 32, x_map, done_map);
      }
      __syncthreads();
    }
    if (warp == 0) {
      // Horizontal sums (l0 + l1) + (l2 + l3) for each kind of this group.
      const int group_base = 12 * (group < 2 ? group : 0);
      float sums[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float l0 = __shfl_sync(0xffffffffu, lane_sum, group_base + 4 * k + 0);
        const float l1 = __shfl_sync(0xffffffffu, lane_sum, group_base + 4 * k + 1);
        const float l2 = __shfl_sync(0xffffffffu, lane_sum, group_base + 4 * k + 2);
        const float l3 = __shfl_sync(0xffffffffu, lane_sum, group_base + 4 * k + 3);
        sums[k] = (l0 + l1) + (l2 + l3);
      }
      if (group < 2 && member == 0 && !done_map[group]) {
        const float x = x_map[group];
        const float n = static_cast<float>(count);
        const float center = 2.0f * kDistanceMultiplierAc * n * x + sums[0];
        const float plus = 2.0f * kDistanceMultiplierAc * n * (x + kEpsilon) + sums[1];
        const float minus = 2.0f * kDistanceMultiplierAc * n * (x - kEpsilon) + sums[2];
        const float second = (plus - minus) / (2.0f * kEpsilon);
        const float step = center / (second + 0.85f);
        solution[group] = x - fminf(fmaxf(step, -20.0f), 20.0f);
        if (fabsf(step) < 3.0e-3f) solved[group] = 1;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) p.y_to_x[tile] = QuantizeMultiplier(solution[0]);
  if (threadIdx.x == 1) p.y_to_b[tile] = QuantizeMultiplier(solution[1]);
}

}  // namespace

int LaunchInitialCfl(const float* opsin, size_t stride, size_t pitch, size_t pw, size_t ph,
                     int8_t* y_to_x, int8_t* y_to_b, cudaStream_t stream) {
  DeviceTables d;
  int status = GetDeviceTables(&d);
  if (status != GJXL_B200_OK) return status;
  const HostTables& h = GetHostTables();
  CflParams p;
  std::memset(&p, 0, sizeof(p));
  p.opsin = opsin;
  p.stride = stride;
  p.pitch = pitch;
  p.blocks_x = static_cast<uint32_t>(pw / 8);
  p.blocks_y = static_cast<uint32_t>(ph / 8);
  p.tiles_x = (p.blocks_x + 7) / 8;
  p.tiles_y = (p.blocks_y + 7) / 8;
  p.fwd = d.forward[0];
  const size_t n = h.layout.count[kTableDct8];
  p.inv_x = d.inverse_dequant + h.layout.offset[kTableDct8] + 0 * n;
  p.inv_b = d.inverse_dequant + h.layout.offset[kTableDct8] + 2 * n;
  p.iterations = 20;
  p.y_to_x = y_to_x;
  p.y_to_b = y_to_b;
  const size_t smem = 4 * kTileValues * sizeof(float);
  status = CheckCuda(cudaFuncSetAttribute(InitialCflKernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)),
                     "initial_cfl smem attribute");
  if (status != GJXL_B200_OK) return status;
  InitialCflKernel<<<p.tiles_x * p.tiles_y, 256, smem, stream>>>(p);
  return CheckLaunch("initial_cfl");
}

}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" int gjxl_b200_initial_cfl(const float* opsin, size_t opsin_stride,
                                     size_t opsin_plane_pitch, size_t padded_width,
                                     size_t padded_height, int8_t* y_to_x, int8_t* y_to_b,
                                     void* stream) {
  ClearLastError();
  if (opsin == nullptr || y_to_x == nullptr || y_to_b == nullptr || padded_width % 8 ||
      padded_height % 8 || padded_width == 0 || padded_height == 0 ||
      opsin_stride < padded_width || opsin_plane_pitch < opsin_stride * padded_height) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "initial_cfl: invalid arguments");
  }
  return LaunchInitialCfl(opsin, opsin_stride, opsin_plane_pitch, padded_width, padded_height,
                          y_to_x, y_to_b, static_cast<cudaStream_t>(stream));
}
