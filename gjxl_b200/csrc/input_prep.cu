// Row a1/a2: packed 8-bit sRGB -> linear RGB planes + padded XYB planes, and
// the quantization-matrix scale statistics.
//
// Follows the reference's arithmetic exactly:
//  - sRGB decode table: src/c_api/image_conversion.cpp:18-31 (computed on the
//    host in double precision, then rounded to float, as there);
//  - opsin transform: src/codec/color_transform.cpp:233-330 (scalar x86 path):
//    three fmaf per row of the opsin matrix, clamp at 0, CubeRootAndAdd,
//    then X = 0.5 (g0 - g1), Y = 0.5 (g0 + g1), B = g2;
//  - padding: transformed edge column/row replicated
//    (src/codec/color_transform.cpp:318-326, 381-390);
//  - statistics: src/codestream/workflow.cpp:1318-1432.
//
// HBM layout: planar float32, stride a multiple of 4 floats, so each thread
// writes one float4 per plane (4 pixels) — 128-bit coalesced stores.

#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "host_util.h"

namespace gjxl_b200 {
namespace {

struct PrepareParams {
  const uint8_t* pixels;
  size_t row_stride;
  uint32_t width, height;
  uint32_t padded_width, padded_height;
  uint32_t channels;
  float* linear;
  size_t linear_stride, linear_pitch;
  float* opsin;
  size_t opsin_stride, opsin_pitch;
  float matrix[3][3];  // scale * opsin matrix, rounded to float like the CPU
  float bias;
  float neg_bias_cuberoot;
  uint32_t* error;
  float table[256];
};

__device__ __forceinline__ void OpsinPixel(const PrepareParams& p, float r,
                                           float g, float b, float out[3]) {
  float gamma[3];
#pragma unroll
  for (int row = 0; row < 3; ++row) {
    float v = fmaf(p.matrix[row][2], b, p.bias);
    v = fmaf(p.matrix[row][1], g, v);
    v = fmaf(p.matrix[row][0], r, v);
    gamma[row] = CubeRootAndAdd(fmaxf(0.0f, v), p.neg_bias_cuberoot);
  }
  out[0] = 0.5f * (gamma[0] - gamma[1]);
  out[1] = 0.5f * (gamma[0] + gamma[1]);
  out[2] = gamma[2];
}

// One thread = 4 horizontally adjacent padded pixels of one row.
__global__ void __launch_bounds__(256)
PrepareInputKernel(const __grid_constant__ PrepareParams p) {
  __shared__ float table[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) table[i] = p.table[i];
  __syncthreads();

  const uint32_t quads_per_row = p.padded_width / 4;
  const uint64_t quad = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (quad >= static_cast<uint64_t>(quads_per_row) * p.padded_height) return;
  const uint32_t y = static_cast<uint32_t>(quad / quads_per_row);
  const uint32_t x0 = static_cast<uint32_t>(quad % quads_per_row) * 4;
  const uint32_t sy = min(y, p.height - 1);
  const uint8_t* row = p.pixels + sy * p.row_stride;

  float rgb[4][3];
  const bool fast = p.channels == 3 && x0 + 4 <= p.width &&
                    ((reinterpret_cast<uintptr_t>(row) + 3u * x0) & 3u) == 0;
  if (fast) {
    const uint32_t* words = reinterpret_cast<const uint32_t*>(row + 3u * x0);
    const uint32_t w0 = __ldg(words), w1 = __ldg(words + 1), w2 = __ldg(words + 2);
    const uint8_t bytes[12] = {
      uint8_t(w0), uint8_t(w0 >> 8), uint8_t(w0 >> 16), uint8_t(w0 >> 24),
      uint8_t(w1), uint8_t(w1 >> 8), uint8_t(w1 >> 16), uint8_t(w1 >> 24),
      uint8_t(w2), uint8_t(w2 >> 8), uint8_t(w2 >> 16), uint8_t(w2 >> 24)};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
      for (int c = 0; c < 3; ++c) rgb[i][c] = table[bytes[3 * i + c]];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t sx = min(x0 + i, p.width - 1);
      const uint8_t* px = row + static_cast<size_t>(sx) * p.channels;
#pragma unroll
      for (int c = 0; c < 3; ++c) rgb[i][c] = table[px[c]];
    }
  }

  float xyb[3][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float out[3];
    OpsinPixel(p, rgb[i][0], rgb[i][1], rgb[i][2], out);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (!IsFinite(out[c])) RaiseError(p.error, kErrorNonFiniteOutput);
      xyb[c][i] = out[c];
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float4* dst = reinterpret_cast<float4*>(p.opsin + c * p.opsin_pitch +
                                            static_cast<size_t>(y) * p.opsin_stride + x0);
    *dst = make_float4(xyb[c][0], xyb[c][1], xyb[c][2], xyb[c][3]);
  }

  if (y < p.height && x0 < p.width) {
    if (x0 + 4 <= p.width && (p.linear_stride & 3) == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float4* dst = reinterpret_cast<float4*>(
          p.linear + c * p.linear_pitch + static_cast<size_t>(y) * p.linear_stride + x0);
        *dst = make_float4(rgb[0][c], rgb[1][c], rgb[2][c], rgb[3][c]);
      }
    } else {
      for (int i = 0; i < 4 && x0 + i < p.width; ++i) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          p.linear[c * p.linear_pitch + static_cast<size_t>(y) * p.linear_stride + x0 + i] =
            rgb[i][c];
        }
      }
    }
  }
}

struct StatsParams {
  const float* opsin;
  size_t stride, pitch;
  uint32_t width, height;
  float* stats;
};

// Grid-stride over the pixels (x >= 1, y >= 1) of the unpadded region; each
// thread keeps running maxima, then warp shuffles and shared memory reduce
// them per CTA, and one atomicMax per CTA and statistic publishes the result
// (a max is order-independent, so the result is exact).
constexpr int kStatsThreads = 256;

__global__ void __launch_bounds__(kStatsThreads)
MatrixScaleStatsKernel(const __grid_constant__ StatsParams p) {
  __shared__ float partial[3][kStatsThreads / 32];
  const uint32_t w1 = p.width - 1;
  const uint64_t n = p.width > 1 && p.height > 1 ? static_cast<uint64_t>(w1) * (p.height - 1) : 0;
  float x_edge = 0.0f, b_edge = 0.0f, exposed = 0.0f;
  const float* X = p.opsin;
  const float* Y = p.opsin + p.pitch;
  const float* B = p.opsin + 2 * p.pitch;
  for (uint64_t index = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; index < n;
       index += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t y = 1 + static_cast<uint32_t>(index / w1);
    const uint32_t x = 1 + static_cast<uint32_t>(index % w1);
    const size_t at = static_cast<size_t>(y) * p.stride + x;
    const size_t left = at - 1, up = at - p.stride;
    const float cx = X[at];
    x_edge = fmaxf(x_edge, fmaxf(fabsf(cx - X[left]), fabsf(cx - X[up])));
    const float cy = Y[at], cb = B[at];
    const float diff = cb - cy;
    b_edge = fmaxf(b_edge,
                   fmaxf(fabsf(diff - (B[left] - Y[left])), fabsf(diff - (B[up] - Y[up]))));
    float e = cb - 1.2f * cy;
    if (e >= 0.0f) {
      e *= fabsf(cb - B[left]) + fabsf(cb - B[up]);
      exposed = fmaxf(exposed, e);
    }
  }
  x_edge = WarpMax(x_edge);
  b_edge = WarpMax(b_edge);
  exposed = WarpMax(exposed);
  const int warp = threadIdx.x / 32;
  if ((threadIdx.x & 31) == 0) {
    partial[0][warp] = x_edge;
    partial[1][warp] = b_edge;
    partial[2][warp] = exposed;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    float m = 0.0f;
    for (int w = 0; w < kStatsThreads / 32; ++w) m = fmaxf(m, partial[threadIdx.x][w]);
    AtomicMaxNonNegative(&p.stats[threadIdx.x], m);
  }
}

}  // namespace
}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" int gjxl_b200_prepare_input(
  const uint8_t* pixels, size_t width, size_t height, size_t row_stride_bytes,
  int channels, float intensity_target, float* linear, size_t linear_stride,
  size_t linear_plane_pitch, float* opsin, size_t opsin_stride,
  size_t opsin_plane_pitch, size_t padded_width, size_t padded_height,
  uint32_t* device_error, void* stream) {
  ClearLastError();
  if (pixels == nullptr || linear == nullptr || opsin == nullptr || width == 0 ||
      height == 0 || (channels != 3 && channels != 4) ||
      row_stride_bytes < width * channels || !std::isfinite(intensity_target) ||
      intensity_target <= 0.0f) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "prepare_input: invalid arguments");
  }
  if (padded_width % 8 != 0 || padded_height % 8 != 0 || padded_width < width ||
      padded_height < height || padded_width - width >= 8 || padded_height - height >= 8 ||
      opsin_stride < padded_width || opsin_stride % 4 != 0 || opsin_plane_pitch % 4 != 0 ||
      opsin_plane_pitch < opsin_stride * padded_height || linear_stride < width ||
      linear_plane_pitch < linear_stride * height || !Aligned16(opsin) ||
      (linear_stride % 4 == 0 && (!Aligned16(linear) || linear_plane_pitch % 4 != 0)) ||
      width > 0xffffffffu || height > 0xffffffffu) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "prepare_input: invalid geometry");
  }
  PrepareParams p;
  std::memset(&p, 0, sizeof(p));
  p.pixels = pixels;
  p.row_stride = row_stride_bytes;
  p.width = static_cast<uint32_t>(width);
  p.height = static_cast<uint32_t>(height);
  p.padded_width = static_cast<uint32_t>(padded_width);
  p.padded_height = static_cast<uint32_t>(padded_height);
  p.channels = static_cast<uint32_t>(channels);
  p.linear = linear;
  p.linear_stride = linear_stride;
  p.linear_pitch = linear_plane_pitch;
  p.opsin = opsin;
  p.opsin_stride = opsin_stride;
  p.opsin_pitch = opsin_plane_pitch;
  // Opsin absorbance matrix and bias (src/codec/color_transform.cpp:36-42).
  const float kMatrix[3][3] = {
    {0.30f, 0.622f, 0.078f},
    {0.23f, 0.692f, 0.078f},
    {0.24342268924547819f, 0.20476744424496821f, 0.55180986650955360f}};
  const float scale = intensity_target / 255.0f;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) p.matrix[r][c] = scale * kMatrix[r][c];
  p.bias = 0.0037930732552754493f;
  p.neg_bias_cuberoot = -HostCubeRootAndAdd(p.bias, 0.0f);
  p.error = device_error;
  for (int i = 0; i < 256; ++i) p.table[i] = SrgbToLinear(i);

  const uint64_t quads = static_cast<uint64_t>(padded_width / 4) * padded_height;
  const unsigned blocks = static_cast<unsigned>((quads + 255) / 256);
  PrepareInputKernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(p);
  return CheckLaunch("prepare_input");
}

extern "C" int gjxl_b200_matrix_scale_stats(const float* opsin, size_t opsin_stride,
                                            size_t opsin_plane_pitch, size_t width,
                                            size_t height, float* stats, void* stream) {
  ClearLastError();
  if (opsin == nullptr || stats == nullptr || width == 0 || height == 0 ||
      opsin_stride < width || opsin_plane_pitch < opsin_stride * height ||
      width > 0xffffffffu || height > 0xffffffffu) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "matrix_scale_stats: invalid arguments");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(stats, 0, 3 * sizeof(float), s) != cudaSuccess) {
    return CheckLaunch("matrix_scale_stats memset");
  }
  StatsParams p{opsin, opsin_stride, opsin_plane_pitch, static_cast<uint32_t>(width),
                static_cast<uint32_t>(height), stats};
  const uint64_t n = width > 1 && height > 1 ? (width - 1) * (height - 1) : 0;
  if (n == 0) return GJXL_B200_OK;
  // Eight CTAs per SM of a B200, fewer for small images.
  const unsigned blocks =
    static_cast<unsigned>(std::min<uint64_t>((n + kStatsThreads - 1) / kStatsThreads, 148 * 8));
  MatrixScaleStatsKernel<<<blocks, kStatsThreads, 0, s>>>(p);
  return CheckLaunch("matrix_scale_stats");
}
