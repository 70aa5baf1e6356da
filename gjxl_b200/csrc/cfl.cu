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
// column inputs with double shuffles. Phase 2: warp 0 alone runs the Newton
// iterations, twelve lanes per map, each owning one of the 3 sums x 4 lanes
// and evaluating its terms as it adds them (no barriers); the other warps
// leave, so that the SM's other tiles take their issue slots.

#include <cmath>
#include <cstring>

#include "common.cuh"
#include "host_util.h"
#include "tables.h"

namespace gjxl_b200 {
namespace {

constexpr int kTileValues = 64 * 64;  // up to 64 blocks of 64 coefficients
constexpr int kMapPad = 4;            // pairs between the two maps' arrays

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
  // Per map (0: y_to_x, 1: y_to_b) and element the pair {a, b}:
  // a = luma / 84 and b = base * luma - chroma (base 0 for y_to_x, 1 for
  // y_to_b). Map 1 starts kMapPad pairs further on, so that the two maps'
  // elements of one index fall in different banks.
  extern __shared__ __align__(16) float2 pairs[];
  const int tile = blockIdx.x;
  const int tx = tile % p.tiles_x, ty = tile / p.tiles_x;
  const int bx0 = tx * 8, by0 = ty * 8;
  const int tw = min(8, static_cast<int>(p.blocks_x) - bx0);
  const int th = min(8, static_cast<int>(p.blocks_y) - by0);
  const int blocks = tw * th;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* pairs_x = pairs;
  float2* pairs_b = pairs + kTileValues + kMapPad;
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
          pairs_b[at] = make_float2(luma / 84.0f, 1.0f * luma - chroma);
        } else {
          const float luma = y_coef[warp][index] * __ldg(p.inv_x + index) * 1.0f;
          const float chroma = value * __ldg(p.inv_x + index) * 1.0f;
          pairs_x[at] = make_float2(luma / 84.0f, 0.0f * luma - chroma);
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (warp != 0) return;

  // Phase 2: FindBestMultiplier (non-fast) for both maps, by warp 0 alone.
  // Lanes 0..11 solve y_to_x and 12..23 y_to_b; lane 4 * kind + slot of a
  // map owns derivative sum `kind` (center, +eps, -eps) over the elements
  // i = slot (mod 4), in increasing i, the reference's four-lane order. Each
  // lane evaluates its terms as it adds them: the dependent adds of the 24
  // chains run back to back, with the term arithmetic between them. Elements
  // skipped by the reference contribute +0.0, which leaves the (never -0.0)
  // sum unchanged.
  const int count = blocks * 64;
  const float kDistanceMultiplierAc = 1.0e-9f;
  const float kEpsilon = 100.0f;
  const bool active = lane < 24;
  const int map = active ? lane / 12 : 0;
  const int member = lane % 12;
  const int kind = member / 4, slot = member % 4;
  const float2* ab = map == 0 ? pairs_x : pairs_b;
  float x = 0.0f;
  bool done = false;
  for (int iteration = 0; iteration < p.iterations; ++iteration) {
    const bool done_x = __shfl_sync(0xffffffffu, done, 0);
    const bool done_b = __shfl_sync(0xffffffffu, done, 12);
    if (done_x && done_b) break;
    const float xk = kind == 0 ? x : kind == 1 ? x + kEpsilon : x - kEpsilon;
    float lane_sum = 0.0f;
    if (active && !done) {
#pragma unroll 8
      for (int i = slot; i < count; i += 4) {
        const float2 v = ab[i];
        const float center = fmaf(v.x, x, v.y);
        const float r = fmaf(v.x, xk, v.y);
        float d = ((2.0f / 3.0f) * v.x) * (fabsf(r) + 1.0f);
        d = r < 0.0f ? -d : d;
        lane_sum += fabsf(center) >= 100.0f ? 0.0f : d;
      }
    }
    // Horizontal sums (l0 + l1) + (l2 + l3) for each kind of this map.
    const int map_base = 12 * map;
    float sums[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float l0 = __shfl_sync(0xffffffffu, lane_sum, map_base + 4 * k + 0);
      const float l1 = __shfl_sync(0xffffffffu, lane_sum, map_base + 4 * k + 1);
      const float l2 = __shfl_sync(0xffffffffu, lane_sum, map_base + 4 * k + 2);
      const float l3 = __shfl_sync(0xffffffffu, lane_sum, map_base + 4 * k + 3);
      sums[k] = (l0 + l1) + (l2 + l3);
    }
    if (active && !done) {
      const float n = static_cast<float>(count);
      const float center = 2.0f * kDistanceMultiplierAc * n * x + sums[0];
      const float plus = 2.0f * kDistanceMultiplierAc * n * (x + kEpsilon) + sums[1];
      const float minus = 2.0f * kDistanceMultiplierAc * n * (x - kEpsilon) + sums[2];
      const float second = (plus - minus) / (2.0f * kEpsilon);
      const float step = center / (second + 0.85f);
      x = x - fminf(fmaxf(step, -20.0f), 20.0f);
      if (fabsf(step) < 3.0e-3f) done = true;
    }
  }
  if (lane == 0) p.y_to_x[tile] = QuantizeMultiplier(x);
  if (lane == 12) p.y_to_b[tile] = QuantizeMultiplier(x);
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
  const size_t smem = (2 * kTileValues + kMapPad) * sizeof(float2);
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
