// Rows a13, a15, a16: decoder-equivalent reconstruction, loop filters,
// XYB -> linear RGB, per-transform Butteraugli reduction and the AQ field
// update, on the device.
//
// Restates, with the reference's exact operation order:
//   SmoothDcCoefficients            src/codec/dc_smoothing.cpp:13-80
//   ReconstructQuantizedCoefficients src/codec/reconstruction.cpp:790-936
//   ConvertDcToLowFrequencies       src/codec/dc_conversion.cpp:238-299
//   DequantizeAcBlock               src/codec/quantization.cpp:822-862
//   ApplyLoopFilters / ApplyGaborish src/codec/loop_filter.cpp, src/codec/gaborish.cpp:101-185
//   ApplyEpf (two iterations: pass 1 then pass 2)  src/codec/epf.cpp:11-160, 297-410
//   OpsinToLinearRgb                src/codec/color_transform.cpp:433-469
//   ReduceButteraugliDistanceMap    src/codec/butteraugli.cpp:116-199
//   RunAdaptiveQuantizationPolicyImpl update  src/codec/adaptive_quantization.cpp:1684-1726

#include <cmath>
#include <cstring>

#include "aq.h"
#include "common.cuh"
#include "host_util.h"
#include "line_dct.cuh"
#include "tables.h"
#include "transform.cuh"

namespace gjxl_b200 {

struct DcTablesRecon {
  double forward[3][4][4];
  float upsample[3][4];
};
__constant__ DcTablesRecon c_dc_recon;

namespace {

constexpr int kThreads = 256;

unsigned Blocks(size_t n, unsigned threads = kThreads) {
  return static_cast<unsigned>((n + threads - 1) / threads);
}

__global__ void SmoothDcKernel(const float* dc, int w, int h, size_t pitch, const AqQuantizer* q,
                               float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w * h) return;
  const int x = i % w, y = i / w;
  if (x == 0 || y == 0 || x + 1 >= w || y + 1 >= h) {
    for (int c = 0; c < 3; ++c) out[c * pitch + i] = dc[c * pitch + i];
    return;
  }
  constexpr float side_weight = 0.20345139757231578f;
  constexpr float corner_weight = 0.0334829185968739f;
  constexpr float center_weight = 1.0f - 4.0f * (side_weight + corner_weight);
  float center[3], smoothed[3];
  float gap = 0.5f;
  for (int c = 0; c < 3; ++c) {
    const float* row = dc + c * pitch + static_cast<size_t>(y) * w;
    const float* top = row - w;
    const float* bottom = row + w;
    const float corners = (top[x - 1] + top[x + 1]) + (bottom[x - 1] + bottom[x + 1]);
    const float sides = (row[x - 1] + row[x + 1]) + (top[x] + bottom[x]);
    center[c] = row[x];
    smoothed[c] = fmaf(corners, corner_weight, fmaf(sides, side_weight, row[x] * center_weight));
    const float normalized_gap = fabsf((row[x] - smoothed[c]) / q->dc_steps[c]);
    gap = fmaxf(gap, normalized_gap);
  }
  const float factor = fmaxf(0.0f, fmaf(-4.0f, gap, 3.0f));
  for (int c = 0; c < 3; ++c) out[c * pitch + i] = fmaf(smoothed[c] - center[c], factor, center[c]);
}

__device__ __forceinline__ float QuantBiasR(int32_t quantized, int channel) {
  const float kBias[4] = {1.0f - 0.05465007330715401f, 1.0f - 0.07005449891748593f,
                          1.0f - 0.049935103337343655f, 0.145f};
  const float value = static_cast<float>(quantized);
  const float absolute = fabsf(value);
  if (absolute < 0.125f) return 0.0f;
  if (absolute < 1.125f) return copysignf(kBias[channel], value);
  return value - kBias[3] / value;
}

__device__ __forceinline__ int LenIdx(int len) { return len == 1 ? 0 : len == 2 ? 1 : 2; }

// ConvertDcToLowFrequencies for one channel of one transform.
template <int W, int H>
__device__ void DcToLowFrequencies(const float* dc_plane, int blocks_x, int ax, int ay,
                                   float* plane, int row_pitch) {
  using S = TransformShape<W, H>;
  constexpr int CW = S::CW, CH = S::CH;
  const int lh = LenIdx(CH), lw = LenIdx(CW);
  // LLF coefficient (v, u) lands at row v, column u of the natural plane.
  for (int v = 0; v < CH; ++v) {
    for (int u = 0; u < CW; ++u) {
      double value = 0.0;
      for (int y = 0; y < CH; ++y) {
        for (int x = 0; x < CW; ++x) {
          value += static_cast<double>(dc_plane[(ay + y) * blocks_x + ax + x]) *
                   c_dc_recon.forward[lh][v][y] * c_dc_recon.forward[lw][u][x];
        }
      }
      plane[v * row_pitch + u] =
        static_cast<float>(value * static_cast<double>(c_dc_recon.upsample[lh][v]) *
                           static_cast<double>(c_dc_recon.upsample[lw][u]));
    }
  }
}

struct ReconParams {
  const int2* anchors;
  const uint32_t* count;
  int blocks_x;
  size_t dc_pitch;
  const int32_t* qac;
  size_t stride, pitch;
  const float* dc;  // smoothed DC, 3 planes of blocks
  const int32_t* raw;
  const AqQuantizer* q;
  const int8_t* y_to_x;
  const int8_t* y_to_b;
  int tiles_x;
  const float* dequant;  // family table [3][N]
  const float* matrix_multiplier;  // device, X / Y / B
  float* recon;
  uint32_t capacity;  // entries of the family's anchor list
};

// K = 1024 / N transforms (3 channels each) per CTA of 384 threads; the
// inverse DCT gives every thread one 8-output chunk of one line per pass
// (line_dct.cuh). Coefficients sit at their natural (v, u) position of a
// padded plane.
constexpr int kReconThreads = 384;

template <int W, int H>
__global__ void __launch_bounds__(kReconThreads, 2) ReconstructKernel(const __grid_constant__ ReconParams p) {
  constexpr int N = W * H, K = 1024 / N, KC = 3 * K;
  using Batch = PlaneBatch<W, H, KC>;
  static_assert(Batch::Items == kReconThreads, "one chunk per thread and pass");
  extern __shared__ __align__(16) unsigned char smem[];
  double* tmp = reinterpret_cast<double*>(smem);                  // [KC] padded planes
  float* coef = reinterpret_cast<float*>(tmp + Batch::Elements);  // [KC] padded planes
  using S = TransformShape<W, H>;
  __shared__ int2 anchor[K];
  __shared__ float scales[K][3];
  __shared__ float factors[K][2];
  __shared__ float dc_values[K][3][S::CW * S::CH];  // the transforms' DC blocks
  const uint32_t first = blockIdx.x * K;
  // The anchor loads do not wait for the count: the list index is clamped to
  // the list, and anchors past the count are never used. Every later global
  // load depends only on the anchors, so the CTA waits for two round trips.
  constexpr int kPerThread = KC * N / kReconThreads;
  const auto anchor_at = [&](int k) {
    return p.anchors[min(first + static_cast<uint32_t>(k), p.capacity - 1)];
  };
  int2 item_anchor[kPerThread];
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    item_anchor[q] = anchor_at((threadIdx.x + q * kReconThreads) / (3 * N));
  }
  const int2 own_anchor = anchor_at(threadIdx.x < K ? threadIdx.x : 0);
  const int2 dc_anchor = anchor_at(threadIdx.x < 3 * K ? threadIdx.x / 3 : 0);
  const uint32_t n = *p.count;
  if (first >= n) return;
  const int active = min(K, static_cast<int>(n - first));
  // Dequantize coefficient j = coefficient_index(v, u) (footprint (j % W, j / W))
  // into (v, u). All of a thread's loads are issued before the first store.
  int32_t qv[kPerThread];
  float dq[kPerThread];
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const int i = threadIdx.x + q * kReconThreads;
    const int r = i % (3 * N), c = r / N, j = r % N;
    const bool live = i < active * 3 * N;
    const int2 a = item_anchor[q];
    qv[q] = live ? p.qac[c * p.pitch + static_cast<size_t>(a.y * 8 + j / W) * p.stride + a.x * 8 +
                         j % W]
                 : 0;
    dq[q] = p.dequant[c * N + j];
  }
  if (threadIdx.x < active) {
    const int k = threadIdx.x;
    const int2 a = own_anchor;
    anchor[k] = a;
    const int raw = p.raw[a.y * p.blocks_x + a.x];
    for (int c = 0; c < 3; ++c) {
      scales[k][c] = (p.q->inverse_global_scale / static_cast<float>(raw)) / p.matrix_multiplier[c];
    }
    const int tile = (a.y / 8) * p.tiles_x + (a.x / 8);
    factors[k][0] = static_cast<float>(p.y_to_x[tile]) / 84.0f;
    factors[k][1] = 1.0f + static_cast<float>(p.y_to_b[tile]) / 84.0f;
  }
  if (threadIdx.x < active * 3) {
    const int k = threadIdx.x / 3, c = threadIdx.x % 3;
    const int2 a = dc_anchor;
    for (int y = 0; y < S::CH; ++y) {
      for (int x = 0; x < S::CW; ++x) {
        dc_values[k][c][y * S::CW + x] =
          p.dc[c * p.dc_pitch + static_cast<size_t>(a.y + y) * p.blocks_x + a.x + x];
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const int i = threadIdx.x + q * kReconThreads;
    if (i >= active * 3 * N) break;
    const int k = i / (3 * N), r = i % (3 * N), c = r / N, j = r % N;
    const int v = H < W ? j / W : j % H, u = H < W ? j % W : j / H;
    coef[Batch::At(k * 3 + c, v, u)] = QuantBiasR(qv[q], c) * (dq[q] * scales[k][c]);
  }
  __syncthreads();
  // Restore the chroma from luma.
  for (int i = threadIdx.x; i < active * N; i += kReconThreads) {
    const int k = i / N, r = i % N, v = r / W, u = r % W;
    const float y = coef[Batch::At(k * 3 + 1, v, u)];
    coef[Batch::At(k * 3 + 0, v, u)] += factors[k][0] * y;
    coef[Batch::At(k * 3 + 2, v, u)] += factors[k][1] * y;
  }
  __syncthreads();
  // LLF from the (smoothed) DC, one thread per transform channel.
  if (threadIdx.x < active * 3) {
    const int k = threadIdx.x / 3, c = threadIdx.x % 3;
    DcToLowFrequencies<W, H>(dc_values[k][c], S::CW, 0, 0, coef + Batch::At(k * 3 + c, 0, 0),
                             Batch::RowPitch);
  }
  __syncthreads();
  const auto present = [&](int plane) { return plane < 3 * active; };
  BatchRowPass<W, H, KC, false>(coef, tmp, threadIdx.x, kReconThreads, present);
  __syncthreads();
  BatchColumnPass<W, H, KC, false>(tmp, coef, threadIdx.x, kReconThreads, present);
  __syncthreads();
  for (int i = threadIdx.x; i < active * 3 * N; i += kReconThreads) {
    const int k = i / (3 * N), r = i % (3 * N), c = r / N, yx = r % N;
    const int2 a = anchor[k];
    p.recon[c * p.pitch + static_cast<size_t>(a.y * 8 + yx / W) * p.stride + a.x * 8 + yx % W] =
      coef[Batch::At(k * 3 + c, yx / W, yx % W)];
  }
}

__device__ __forceinline__ int MirrorR(int c, int n) {
  if (c >= 0 && c < n) return c;
  const int period = 2 * n;
  int phase;
  if (c >= 0) {
    phase = c % period;
  } else {
    const int r = (-c) % period;
    phase = r == 0 ? 0 : period - r;
  }
  return phase < n ? phase : period - 1 - phase;
}

// Loop filters on a shared-memory tile: each CTA of kTileW x kTileRows
// threads computes a kTileW x kTileH output tile (each thread kTileH /
// kTileRows rows) and first stages its input window (tile + halo, every
// coordinate mirrored at the image border as the reference's filters read
// it) for all three planes, so the filter taps read shared memory only.
constexpr int kTileW = 32, kTileH = 32, kTileRows = 8;
constexpr int kRowsPerThread = kTileH / kTileRows;

// The window is loaded with a 2D thread mapping (no index division), all of
// a thread's loads issued before its first store; windows that lie inside
// the image skip the mirroring.
template <int Halo>
__device__ __forceinline__ void StageWindow(const float* in, size_t stride, size_t pitch, int w,
                                            int h, int x0, int y0,
                                            float (*tile)[kTileH + 2 * Halo][kTileW + 2 * Halo]) {
  constexpr int TW = kTileW + 2 * Halo, TH = kTileH + 2 * Halo;
  constexpr int kCols = (TW + kTileW - 1) / kTileW, kRows = (TH + kTileRows - 1) / kTileRows;
  const bool interior = x0 >= Halo && y0 >= Halo && x0 + kTileW + Halo <= w &&
                        y0 + kTileH + Halo <= h;
  float v[3][kRows][kCols];
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
#pragma unroll
    for (int k = 0; k < kCols; ++k) {
      const int ty = threadIdx.y + r * kTileRows, tx = threadIdx.x + k * kTileW;
      if (ty < TH && tx < TW) {
        int gy = y0 + ty - Halo, gx = x0 + tx - Halo;
        if (!interior) {
          gy = MirrorR(gy, h);
          gx = MirrorR(gx, w);
        }
        const float* src = in + static_cast<size_t>(gy) * stride + gx;
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c][r][k] = src[c * pitch];
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
#pragma unroll
    for (int k = 0; k < kCols; ++k) {
      const int ty = threadIdx.y + r * kTileRows, tx = threadIdx.x + k * kTileW;
      if (ty < TH && tx < TW) {
#pragma unroll
        for (int c = 0; c < 3; ++c) tile[c][ty][tx] = v[c][r][k];
      }
    }
  }
}

struct GaborishParams {
  const float* in;
  size_t in_stride, in_pitch;
  float* out;  // dense width x height planes
  int w, h;
  float weights[3];  // center, axis, diagonal
  uint32_t* error;
};

__global__ void __launch_bounds__(kTileW * kTileRows)
GaborishForwardKernel(const __grid_constant__ GaborishParams p) {
  __shared__ float tile[3][kTileH + 2][kTileW + 2];
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH;
  StageWindow<1>(p.in, p.in_stride, p.in_pitch, p.w, p.h, x0, y0, tile);
  __syncthreads();
  const int x = x0 + threadIdx.x;
  if (x >= p.w) return;
  const int tx = threadIdx.x + 1;
  const size_t n = static_cast<size_t>(p.w) * p.h;
#pragma unroll
  for (int row = 0; row < kRowsPerThread; ++row) {
    const int oy = threadIdx.y + row * kTileRows, y = y0 + oy;
    if (y >= p.h) break;
    const int ty = oy + 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const auto& t = tile[c];
      const float axes = (t[ty][tx - 1] + t[ty][tx + 1]) + (t[ty - 1][tx] + t[ty + 1][tx]);
      const float diagonals =
        (t[ty - 1][tx - 1] + t[ty - 1][tx + 1]) + (t[ty + 1][tx - 1] + t[ty + 1][tx + 1]);
      const float value =
        p.weights[0] * t[ty][tx] + p.weights[1] * axes + p.weights[2] * diagonals;
      if (!IsFinite(value)) RaiseError(p.error, kErrorNonFiniteOutput);
      p.out[c * n + static_cast<size_t>(y) * p.w + x] = value;
    }
  }
}

struct LinearParams {
  const float* opsin;
  float* linear;
  size_t n;
  float bias_cuberoot;
  float scaled_matrix[3][3];  // scale * inverse opsin matrix
  uint32_t* error;
};

// OpsinToLinear (color_transform.cpp:433) of one pixel (x, y, b) into
// pixel i of the three linear planes.
__device__ __forceinline__ void OpsinToLinearPixel(const LinearParams& p, float x, float y,
                                                   float b, size_t i) {
  const float kOpsinBias = 0.0037930732552754493f;
  const float gamma[3] = {y + x + p.bias_cuberoot, y - x + p.bias_cuberoot, b + p.bias_cuberoot};
  float mixed[3];
  for (int c = 0; c < 3; ++c) mixed[c] = gamma[c] * gamma[c] * gamma[c] - kOpsinBias;
  for (int r = 0; r < 3; ++r) {
    float v = p.scaled_matrix[r][0] * mixed[0];
    v = fmaf(p.scaled_matrix[r][1], mixed[1], v);
    v = fmaf(p.scaled_matrix[r][2], mixed[2], v);
    if (!IsFinite(v)) RaiseError(p.error, kErrorNonFiniteOutput);
    p.linear[r * p.n + i] = v;
  }
}

struct EpfParams {
  const float* in;  // dense planes
  float* out;
  int w, h;
  const float* inverse_sigma;
  int blocks_x;
  float sigma_scale;
  // Pass 2 only: with to_linear, the filtered pixel goes through
  // OpsinToLinear into linear.linear instead of into `out`.
  int to_linear;
  LinearParams linear;
};

// One EPF iteration (epf.cpp:92-160). Pass 1 compares 5-pixel plus-shaped
// patches (halo 2); pass 2 compares single pixels (halo 1). For pass 1 the
// absolute differences of horizontal and vertical neighbours are taken once
// per window position: the patch distance for offset d at p adds
// |t[p + k] - t[p + d + k]| over the patch in the reference's order, and that
// term is the horizontal (vertical) difference at p + k for d = +1 and at
// p - 1 + k for d = -1 (|a - b| = |b - a| exactly).
template <int Pass>
__global__ void __launch_bounds__(kTileW * kTileRows) EpfKernel(const __grid_constant__ EpfParams p) {
  constexpr int Halo = Pass == 1 ? 2 : 1;
  constexpr int TW = kTileW + 2 * Halo, TH = kTileH + 2 * Halo;
  __shared__ float tile[3][TH][TW];
  // Pass 1: [0] horizontal |t[y][x] - t[y][x+1]|, [1] vertical |t[y][x] - t[y+1][x]|.
  __shared__ float diff[Pass == 1 ? 2 : 1][Pass == 1 ? 3 : 1][Pass == 1 ? TH : 1]
                       [Pass == 1 ? TW : 1];
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH;
  StageWindow<Halo>(p.in, p.w, static_cast<size_t>(p.w) * p.h, p.w, p.h, x0, y0, tile);
  __syncthreads();
  if constexpr (Pass == 1) {
    constexpr int kCols = (TW + kTileW - 1) / kTileW, kRows = (TH + kTileRows - 1) / kTileRows;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
#pragma unroll
      for (int k = 0; k < kCols; ++k) {
        const int ty = threadIdx.y + r * kTileRows, tx = threadIdx.x + k * kTileW;
        if (ty >= TH || tx >= TW) continue;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (tx + 1 < TW) diff[0][c][ty][tx] = fabsf(tile[c][ty][tx] - tile[c][ty][tx + 1]);
          if (ty + 1 < TH) diff[1][c][ty][tx] = fabsf(tile[c][ty][tx] - tile[c][ty + 1][tx]);
        }
      }
    }
    __syncthreads();
  }
  const int x = x0 + threadIdx.x;
  if (x >= p.w) return;
  const size_t n = static_cast<size_t>(p.w) * p.h;
  const int tx = threadIdx.x + Halo;
  const float kMinInverseSigma = -1.1715728752538099024f / 0.3f;
  const float channel_scale[3] = {40.0f, 5.0f, 3.5f};
  const int offsets[4][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}};
  const int plus[5][2] = {{0, 0}, {0, -1}, {-1, 0}, {0, 1}, {1, 0}};
#pragma unroll 1
  for (int row = 0; row < kRowsPerThread; ++row) {
    const int oy = threadIdx.y + row * kTileRows, y = y0 + oy;
    if (y >= p.h) break;
    const size_t i = static_cast<size_t>(y) * p.w + x;
    const int ty = oy + Halo;
    const float block_inverse_sigma = p.inverse_sigma[(y / 8) * p.blocks_x + x / 8];
    if (block_inverse_sigma < kMinInverseSigma) {
      if (Pass == 2 && p.to_linear) {
        OpsinToLinearPixel(p.linear, tile[0][ty][tx], tile[1][ty][tx], tile[2][ty][tx], i);
      } else {
        for (int c = 0; c < 3; ++c) p.out[c * n + i] = tile[c][ty][tx];
      }
      continue;
    }
    const bool border = x % 8 == 0 || x % 8 == 7 || y % 8 == 0 || y % 8 == 7;
    const float scaled = block_inverse_sigma * p.sigma_scale * (border ? 2.0f / 3.0f : 1.0f);
    float sum[3] = {tile[0][ty][tx], tile[1][ty][tx], tile[2][ty][tx]};
    float weight_sum = 1.0f;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      const int dx = offsets[o][0], dy = offsets[o][1];
      float sad = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if constexpr (Pass == 1) {
          // Differences along the offset's axis, based at p (d = +1) or at
          // p + d (d = -1).
          const auto& d = diff[dy != 0 ? 1 : 0][c];
          const int bx = tx + (dx < 0 ? dx : 0), by = ty + (dy < 0 ? dy : 0);
          float channel_sad = 0.0f;
#pragma unroll
          for (int k = 0; k < 5; ++k) channel_sad += d[by + plus[k][1]][bx + plus[k][0]];
          sad = fmaf(channel_sad, channel_scale[c], sad);
        } else {
          const auto& t = tile[c];
          sad = fmaf(fabsf(t[ty][tx] - t[ty + dy][tx + dx]), channel_scale[c], sad);
        }
      }
      const float weight = fmaxf(0.0f, fmaf(sad, scaled, 1.0f));
      weight_sum += weight;
#pragma unroll
      for (int c = 0; c < 3; ++c) sum[c] = fmaf(weight, tile[c][ty + dy][tx + dx], sum[c]);
    }
    if (Pass == 2 && p.to_linear) {
      OpsinToLinearPixel(p.linear, sum[0] / weight_sum, sum[1] / weight_sum,
                         sum[2] / weight_sum, i);
    } else {
      for (int c = 0; c < 3; ++c) p.out[c * n + i] = sum[c] / weight_sum;
    }
  }
}

__global__ void OpsinToLinearKernel(const __grid_constant__ LinearParams p) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i >= p.n) return;
  OpsinToLinearPixel(p, p.opsin[i], p.opsin[p.n + i], p.opsin[2 * p.n + i], i);
}

__global__ void BlockReduceKernel(const uint8_t* cells, int blocks_x, int blocks_y,
                                  const float* map, int w, int h, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= blocks_x * blocks_y) return;
  const uint8_t cell = cells[i];
  if (!(cell & 1)) return;
  const int f = StrategyFamily(cell >> 1);
  const int cw = FamilyCoveredW(f), ch = FamilyCoveredH(f);
  const int bx = i % blocks_x, by = i / blocks_x;
  const int x0 = bx * 8, y0 = by * 8;
  const int x1 = min(w, x0 + cw * 8), y1 = min(h, y0 + ch * 8);
  float norm = 0.0f;
  int count = 0;
  for (int y = y0; y < y1; ++y) {
    for (int x = x0; x < x1; ++x) {
      float v = map[static_cast<size_t>(y) * w + x];
      v *= v;
      v *= v;
      v *= v;
      v *= v;
      norm += v;
      ++count;
    }
  }
  // std::pow(float, 1/16): evaluated in double and rounded to float.
  const float mean = norm / static_cast<float>(count);
  const float d = 1.2f * static_cast<float>(pow(static_cast<double>(mean), 0.0625));
  for (int dy = 0; dy < ch; ++dy)
    for (int dx = 0; dx < cw; ++dx) out[(by + dy) * blocks_x + bx + dx] = d;
}

__global__ void PolicyUpdateKernel(float* field, const float* adjusted_initial,
                                   const float* block_distance, int n, int iteration,
                                   float target, const AqPolicy* policy, const AqQuantizer* q,
                                   uint32_t* error) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float lo = policy->lower_bound, hi = policy->upper_bound;
  float value = field[i];
  if (iteration == 1) {
    const float clamp = 0.4f * value + 0.6f * adjusted_initial[i];
    if (value < clamp) value = fminf(fmaxf(clamp, lo), hi);
  }
  const float difference = block_distance[i] / target;
  if (!(IsFinite(difference) && difference >= 0.0f)) RaiseError(error, kErrorInternal);
  if (difference <= 1.0f) {
    if (iteration < 2) value *= static_cast<float>(pow(static_cast<double>(difference), 0.2));
  } else {
    const float old = value;
    value *= difference;
    const long old_raw = lroundf(old * q->inverse_global_scale);
    const long new_raw = lroundf(value * q->inverse_global_scale);
    if (old_raw == new_raw) value = old + q->scale;
  }
  field[i] = fminf(fmaxf(value, lo), hi);
}

}  // namespace

void UploadDcReconTables() {
  DcTablesRecon t;
  std::memset(&t, 0, sizeof(t));
  const double sqrt2 = 1.41421356237309504880, pi = 3.14159265358979323846;
  const int lengths[3] = {1, 2, 4};
  for (int li = 0; li < 3; ++li) {
    const int len = lengths[li];
    for (int f = 0; f < len; ++f) {
      const double alpha = f == 0 ? sqrt2 / 2.0 : 1.0;
      for (int s = 0; s < len; ++s) {
        const double angle = (static_cast<double>(s) + 0.5) * static_cast<double>(f) * pi /
                             static_cast<double>(len);
        t.forward[li][f][s] = sqrt2 * alpha * std::cos(angle) / static_cast<double>(len);
      }
    }
  }
  const float up[3][4] = {{1.0f, 0, 0, 0},
                          {1.0f, 1.108937353592731823f, 0, 0},
                          {1.0f, 1.025760096781116015f, 1.108937353592731823f,
                           1.270559368765487251f}};
  std::memcpy(t.upsample, up, sizeof(up));
  cudaMemcpyToSymbol(c_dc_recon, &t, sizeof(t));
}

int AqSmoothDc(const float* dc, size_t bx, size_t by, const AqQuantizer* q, float* out,
               cudaStream_t stream) {
  SmoothDcKernel<<<Blocks(bx * by), kThreads, 0, stream>>>(dc, static_cast<int>(bx),
                                                           static_cast<int>(by), bx * by, q, out);
  return CheckLaunch("aq smooth dc");
}

template <int W, int H>
int LaunchReconstruct(ReconParams p, const DeviceTables& d, int family, size_t max_count,
                      cudaStream_t stream) {
  constexpr int N = W * H, K = 1024 / N;
  const HostTables& h = GetHostTables();
  const int table = StrategyTableFamily(FamilyStrategy(family));
  p.dequant = d.dequant + h.layout.offset[table];
  const size_t smem = static_cast<size_t>(PlaneBatch<W, H, 3 * K>::Elements) * 12;
  int status = CheckCuda(cudaFuncSetAttribute(ReconstructKernel<W, H>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(smem)),
                         "aq reconstruct attribute");
  if (status != GJXL_B200_OK) return status;
  const unsigned grid = static_cast<unsigned>((max_count + K - 1) / K);
  if (grid == 0) return GJXL_B200_OK;
  p.capacity = static_cast<uint32_t>(max_count);
  ReconstructKernel<W, H><<<grid, kReconThreads, smem, stream>>>(p);
  return CheckLaunch("aq reconstruct");
}

int AqReconstruct(const int2* lists, const uint32_t* counts, size_t bx, size_t by,
                  const int32_t* qac, size_t stride, size_t pitch, const float* dc,
                  const int32_t* raw, const AqQuantizer* q, const int8_t* y_to_x,
                  const int8_t* y_to_b, const float* matrix_multiplier, float* recon,
                  cudaStream_t stream, const StreamFan* fan) {
  DeviceTables d;
  int status = GetDeviceTables(&d);
  if (status != GJXL_B200_OK) return status;
  const size_t blocks = bx * by;
  ReconParams p;
  std::memset(&p, 0, sizeof(p));
  p.blocks_x = static_cast<int>(bx);
  p.dc_pitch = blocks;
  p.qac = qac;
  p.stride = stride;
  p.pitch = pitch;
  p.dc = dc;
  p.raw = raw;
  p.q = q;
  p.y_to_x = y_to_x;
  p.y_to_b = y_to_b;
  p.tiles_x = static_cast<int>((bx + 7) / 8);
  p.matrix_multiplier = matrix_multiplier;
  p.recon = recon;
  // The families are independent: with a fan they run side by side.
  if (status == GJXL_B200_OK) status = CheckCuda(FanFork(fan), "fork");
  for (int f = 0; f < kFamilyCountT && status == GJXL_B200_OK; ++f) {
    const cudaStream_t fs = fan != nullptr ? fan->For(f) : stream;
    p.anchors = lists + f * blocks;
    p.count = counts + f;
    const size_t max_count = blocks / (FamilyCoveredW(f) * FamilyCoveredH(f));
    switch (f) {
      case 0: status = LaunchReconstruct<8, 8>(p, d, f, max_count, fs); break;
      case 1: status = LaunchReconstruct<8, 16>(p, d, f, max_count, fs); break;
      case 2: status = LaunchReconstruct<16, 8>(p, d, f, max_count, fs); break;
      case 3: status = LaunchReconstruct<16, 16>(p, d, f, max_count, fs); break;
      case 4: status = LaunchReconstruct<16, 32>(p, d, f, max_count, fs); break;
      case 5: status = LaunchReconstruct<32, 16>(p, d, f, max_count, fs); break;
      case 6: status = LaunchReconstruct<32, 32>(p, d, f, max_count, fs); break;
    }
  }
  const cudaError_t joined = FanJoin(fan);
  if (status == GJXL_B200_OK) status = CheckCuda(joined, "join");
  return status;
}

LinearParams MakeLinearParams(const float* opsin, size_t width, size_t height,
                              float intensity_target, float* linear, uint32_t* error) {
  LinearParams p;
  p.opsin = opsin;
  p.linear = linear;
  p.n = width * height;
  p.bias_cuberoot = std::cbrt(0.0037930732552754493f);
  const float kInverse[3][3] = {
    {11.031566901960783f, -9.866943921568629f, -0.16462299647058826f},
    {-3.254147380392157f, 4.418770392156863f, -0.16462299647058826f},
    {-3.6588512862745097f, 2.7129230470588235f, 1.9459282392156863f}};
  const float scale = 255.0f / intensity_target;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) p.scaled_matrix[r][c] = scale * kInverse[r][c];
  p.error = error;
  return p;
}

int AqLoopFilters(const float* recon, size_t recon_stride, size_t recon_pitch, size_t width,
                  size_t height, const float* inverse_sigma, size_t bx, float* scratch_a,
                  float* scratch_b, float* filtered, uint32_t* error, cudaStream_t stream,
                  float* linear, float intensity_target) {
  GaborishParams g;
  g.in = recon;
  g.in_stride = recon_stride;
  g.in_pitch = recon_pitch;
  g.out = scratch_a;
  g.w = static_cast<int>(width);
  g.h = static_cast<int>(height);
  // ApplyGaborish weights (gaborish.cpp:118-138).
  const float w1 = 1.1f * 0.104699568f, w2 = 1.1f * 0.055680538f;
  const float divisor = 1.0f + 4.0f * (w1 + w2);
  g.weights[0] = 1.0f / divisor;
  g.weights[1] = w1 / divisor;
  g.weights[2] = w2 / divisor;
  g.error = error;
  const dim3 tiles(static_cast<unsigned>((width + kTileW - 1) / kTileW),
                   static_cast<unsigned>((height + kTileH - 1) / kTileH));
  const dim3 threads(kTileW, kTileRows);
  GaborishForwardKernel<<<tiles, threads, 0, stream>>>(g);
  EpfParams e;
  e.w = static_cast<int>(width);
  e.h = static_cast<int>(height);
  e.inverse_sigma = inverse_sigma;
  e.blocks_x = static_cast<int>(bx);
  e.in = scratch_a;
  e.out = scratch_b;
  e.sigma_scale = 1.65f * 1.0f;
  e.to_linear = 0;
  e.linear = MakeLinearParams(nullptr, width, height, intensity_target, linear, error);
  EpfKernel<1><<<tiles, threads, 0, stream>>>(e);
  e.in = scratch_b;
  e.out = filtered;
  e.to_linear = linear != nullptr ? 1 : 0;
  e.sigma_scale = 1.65f * 6.5f;
  EpfKernel<2><<<tiles, threads, 0, stream>>>(e);
  return CheckLaunch("aq loop filters");
}

int AqOpsinToLinear(const float* opsin, size_t width, size_t height, float intensity_target,
                    float* linear, uint32_t* error, cudaStream_t stream) {
  const LinearParams p = MakeLinearParams(opsin, width, height, intensity_target, linear, error);
  OpsinToLinearKernel<<<Blocks(p.n), kThreads, 0, stream>>>(p);
  return CheckLaunch("aq opsin to linear");
}

int AqBlockReduce(const uint8_t* cells, size_t bx, size_t by, const float* distance_map,
                  size_t width, size_t height, float* block_distance, cudaStream_t stream) {
  BlockReduceKernel<<<Blocks(bx * by), kThreads, 0, stream>>>(
    cells, static_cast<int>(bx), static_cast<int>(by), distance_map, static_cast<int>(width),
    static_cast<int>(height), block_distance);
  return CheckLaunch("aq block reduce");
}

int AqPolicyUpdate(float* field, const float* adjusted_initial, const float* block_distance,
                   size_t blocks, int iteration, float target, const AqPolicy* policy,
                   const AqQuantizer* q, uint32_t* error, cudaStream_t stream) {
  PolicyUpdateKernel<<<Blocks(blocks), kThreads, 0, stream>>>(
    field, adjusted_initial, block_distance, static_cast<int>(blocks), iteration, target, policy,
    q, error);
  return CheckLaunch("aq policy update");
}

}  // namespace gjxl_b200
