// Row a3: initial quantization field, strategy mask and blurred pixel mask.
// Row a4: inverse Gaborish (5x5 symmetric convolution with mirrored borders).
//
// Restates src/codec/adaptive_quantization.cpp:115-303 (masking helpers),
// :343-488 (per-block modulations) and :582-729 (ComputeInitialQuantField),
// src/codec/convolution.cpp (ConvolveSymmetric5) and src/codec/gaborish.cpp:
// 11-35 (inverse weights). Every floating-point operation keeps the
// reference's order and rounding (--fmad=false, explicit fmaf), so results
// are bit-identical.
//
// Kernels (all HBM-bound stencils over planar float32):
//   PreErosionKernel       one thread per 4x4 pixel cell: per-pixel masking,
//                          raw pixel mask, 4x4 pre-erosion average.
//   ErosionModulationKernel one thread per 8x8 block: fuzzy erosion (2x2 of
//                          pre-erosion cells), strategy mask, gamma / HF /
//                          blue modulations, FastPow2.
//   Symmetric5Kernel       32x32 output tile from a mirrored halo tile in shared memory.

#include <cmath>
#include <cstring>

#include "common.cuh"
#include "host_util.h"
#include "log1p.cuh"

namespace gjxl_b200 {
namespace {

constexpr float kInverseLog2E = 0.6931471805599453f;

// adaptive_quantization.cpp:121-145; Invert selects numerator / denominator.
template <bool Invert>
__device__ __forceinline__ float GammaDerivativeRatio(float value) {
  constexpr float kEpsilon = 1.0e-2f;
  constexpr float kSgMul = 226.77216153508914f;
  constexpr float kSgMul2 = 1.0f / 73.377132366608819f;
  constexpr float kSgReturnMul = kSgMul2 * 18.6580932135f * kInverseLog2E;
  constexpr float kSgOffset = 7.7825991679894591f;
  constexpr float kNumMul = kSgReturnMul * 3.0f * kSgMul;
  constexpr float kDenMul = kInverseLog2E * kSgMul;
  constexpr float kDenAdd = kSgOffset * kInverseLog2E + kEpsilon;
  value = fmaxf(value, 0.0f);
  const float squared = value * value;
  const float numerator = fmaf(kNumMul, squared, kEpsilon);
  const float denominator = fmaf(kDenMul * value, squared, kDenAdd);
  return Invert ? numerator / denominator : denominator / numerator;
}

// adaptive_quantization.cpp:147-165.
__device__ __forceinline__ float ComputeMask(float value) {
  constexpr float kBase = -0.7647f;
  constexpr float kMul4 = 9.4708735624378946f;
  constexpr float kMul2 = 17.35036561631863f;
  constexpr float kOffset2 = 302.59587815579727f;
  constexpr float kMul3 = 6.7943250517376494f;
  constexpr float kOffset3 = 3.7179635626140772f;
  constexpr float kOffset4 = 0.25f * kOffset3;
  constexpr float kMul0 = 0.80061762862741759f;
  const float v1 = fmaxf(value * kMul0, 1.0e-3f);
  const float v2 = 1.0f / (v1 + kOffset2);
  const float v3 = 1.0f / fmaf(v1, v1, kOffset3);
  const float v4 = 1.0f / fmaf(v1, v1, kOffset4);
  return kBase + fmaf(kMul4, v4, fmaf(kMul2, v2, kMul3 * v3));
}

struct PreErosionParams {
  const float* y_plane;  // opsin Y
  size_t stride;
  uint32_t width, height;  // padded extent (multiples of 8)
  float* raw_pixel_mask;   // width x height, stride `mask_stride`
  size_t mask_stride;
  float* pre_erosion;      // (width/4) x (height/4), dense
  float masking_inner_scale;  // sqrt(kMul * 1e8f), computed like the CPU
};

__global__ void __launch_bounds__(256)
PreErosionKernel(const __grid_constant__ PreErosionParams p) {
  const uint32_t cells_x = p.width / 4;
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= cells_x * (p.height / 4)) return;
  const uint32_t gx = cell % cells_x, gy = cell / cells_x;
  const uint32_t x0 = gx * 4;
  float column[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const uint32_t y = gy * 4 + r;
    const uint32_t top = y == 0 ? y : y - 1;
    const uint32_t bottom = y + 1 < p.height ? y + 1 : y;
    const float* row = p.y_plane + static_cast<size_t>(y) * p.stride;
    const float* top_row = p.y_plane + static_cast<size_t>(top) * p.stride;
    const float* bottom_row = p.y_plane + static_cast<size_t>(bottom) * p.stride;
    const float4 c4 = *reinterpret_cast<const float4*>(row + x0);
    const float4 t4 = *reinterpret_cast<const float4*>(top_row + x0);
    const float4 b4 = *reinterpret_cast<const float4*>(bottom_row + x0);
    const float cur[6] = {row[x0 == 0 ? 0 : x0 - 1], c4.x, c4.y, c4.z, c4.w,
                          row[x0 + 4 < p.width ? x0 + 4 : x0 + 3]};
    const float tops[4] = {t4.x, t4.y, t4.z, t4.w};
    const float bots[4] = {b4.x, b4.y, b4.z, b4.w};
    float mask_out[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float center = cur[i + 1];
      const float base = 0.25f * (((bots[i] + tops[i]) + cur[i]) + cur[i + 2]);
      const float gamma = GammaDerivativeRatio<false>(center + 0.019f);
      const float d = gamma * (center - base);
      const float pixel_difference = Log1pF(fabsf(d));
      mask_out[i] = 1.0f / (pixel_difference + 0.01f);
      float block_difference = d * d;
      block_difference = fminf(block_difference, 0.2f);
      // MaskingSqrt (adaptive_quantization.cpp:167-173).
      block_difference =
        0.25f * sqrtf(fmaf(block_difference, p.masking_inner_scale, 27.505837037000106f));
      if (r == 0) {
        column[i] = block_difference;
      } else {
        column[i] += block_difference;
      }
    }
    *reinterpret_cast<float4*>(p.raw_pixel_mask + static_cast<size_t>(y) * p.mask_stride + x0) =
      make_float4(mask_out[0], mask_out[1], mask_out[2], mask_out[3]);
  }
  p.pre_erosion[static_cast<size_t>(gy) * cells_x + gx] =
    (((column[0] + column[1]) + column[2]) + column[3]) * 0.25f;
}

struct ModulationParams {
  const float* opsin;  // padded XYB planes
  size_t stride, pitch;
  uint32_t blocks_x, blocks_y;
  const float* pre_erosion;  // (2*blocks_x) x (2*blocks_y)
  float weights[4];          // fuzzy-erosion weights, normalized on the host
  float multiplier, addend;  // PerBlockModulations scale/dampen terms
  float* quant_field;
  float* strategy_mask;
  uint32_t* error;
};

__device__ __forceinline__ void StoreMin4(float v, float& m0, float& m1, float& m2, float& m3) {
  if (v >= m3) return;
  if (v < m0) {
    m3 = m2; m2 = m1; m1 = m0; m0 = v;
  } else if (v < m1) {
    m3 = m2; m2 = m1; m1 = v;
  } else if (v < m2) {
    m3 = m2; m2 = v;
  } else {
    m3 = v;
  }
}

__device__ __forceinline__ void Swap(float& a, float& b) {
  const float t = a; a = b; b = t;
}

// adaptive_quantization.cpp:225-282 for one pre-erosion sample.
__device__ __forceinline__ float ErodedValue(const ModulationParams& p, int x, int y) {
  const int w = 2 * p.blocks_x, h = 2 * p.blocks_y;
  const int top = y == 0 ? y : y - 1, bottom = y + 1 < h ? y + 1 : y;
  const int left = x == 0 ? x : x - 1, right = x + 1 < w ? x + 1 : x;
  const float* s = p.pre_erosion;
  float m0 = s[y * w + x], m1 = s[y * w + left], m2 = s[y * w + right], m3 = s[top * w + left];
  if (m0 > m1) Swap(m0, m1);
  if (m0 > m2) Swap(m0, m2);
  if (m0 > m3) Swap(m0, m3);
  if (m1 > m2) Swap(m1, m2);
  if (m1 > m3) Swap(m1, m3);
  if (m2 > m3) Swap(m2, m3);
  StoreMin4(s[top * w + x], m0, m1, m2, m3);
  StoreMin4(s[top * w + right], m0, m1, m2, m3);
  StoreMin4(s[bottom * w + left], m0, m1, m2, m3);
  StoreMin4(s[bottom * w + x], m0, m1, m2, m3);
  StoreMin4(s[bottom * w + right], m0, m1, m2, m3);
  return ((p.weights[0] * m0 + p.weights[1] * m1) + p.weights[2] * m2) + p.weights[3] * m3;
}

__global__ void __launch_bounds__(128)
ErosionModulationKernel(const __grid_constant__ ModulationParams p) {
  const uint32_t block = blockIdx.x * blockDim.x + threadIdx.x;
  if (block >= p.blocks_x * p.blocks_y) return;
  const int bx = block % p.blocks_x, by = block / p.blocks_x;
  float q = ErodedValue(p, 2 * bx, 2 * by);
  q += ErodedValue(p, 2 * bx + 1, 2 * by);
  q += ErodedValue(p, 2 * bx, 2 * by + 1);
  q += ErodedValue(p, 2 * bx + 1, 2 * by + 1);
  const float strategy = 1.0f / (q + 0.001f);

  const float* X = p.opsin;
  const float* Y = p.opsin + p.pitch;
  const float* B = p.opsin + 2 * p.pitch;
  const size_t base = static_cast<size_t>(by) * 8 * p.stride + static_cast<size_t>(bx) * 8;

  // Gamma modulation (adaptive_quantization.cpp:343-374).
  float gamma_lanes[4] = {0, 0, 0, 0};
  // High-frequency modulation (:376-406).
  float hf_lanes[4] = {0, 0, 0, 0};
  // Blue modulation (:408-438).
  float blue_lanes[4] = {0, 0, 0, 0};
  constexpr float kHfLimit = 0.0206f;
  constexpr float kBlueLimit = 0.010474084867598155f;
  constexpr float kBlueOffset = 0.0031994768654636393f;
#pragma unroll 1
  for (int dy = 0; dy < 8; ++dy) {
    const float* xr = X + base + dy * p.stride;
    const float* yr = Y + base + dy * p.stride;
    const float* br = B + base + dy * p.stride;
    const float* yn = dy + 1 < 8 ? yr + p.stride : yr;
#pragma unroll
    for (int dx = 0; dx < 8; ++dx) {
      const float vx = xr[dx], vy = yr[dx], vb = br[dx];
      const float in_y = vy + 0.16f;
      gamma_lanes[dx & 3] += GammaDerivativeRatio<true>(in_y - vx);
      gamma_lanes[dx & 3] += GammaDerivativeRatio<true>(in_y + vx);
      if (dx + 1 < 8) hf_lanes[dx & 3] += fminf(kHfLimit, fabsf(vy - yr[dx + 1]));
      hf_lanes[dx & 3] += fminf(kHfLimit, fabsf(vy - yn[dx]));
      const float effective_y = vy + kBlueOffset + fabsf(vx);
      if (vb > effective_y) blue_lanes[dx & 3] += fminf(vb - effective_y, kBlueLimit);
    }
  }
  const float mask_value = ComputeMask(q);
  const float overall =
    ((gamma_lanes[0] + gamma_lanes[1]) + (gamma_lanes[2] + gamma_lanes[3])) * (0.5f / 64.0f);
  float gamma_value;
  if (!IsFinite(overall) || overall <= 0.0f) {
    gamma_value = __int_as_float(0x7fc00000);
  } else {
    gamma_value = fmaf(0.1005613337192697f, FastLog2(overall), mask_value);
  }
  const float hf_sum = (hf_lanes[0] + hf_lanes[1]) + (hf_lanes[2] + hf_lanes[3]);
  const float hf_value = gamma_value + (hf_sum * -0.38f + 0.42f);
  float blue_sum = (blue_lanes[0] + blue_lanes[1]) + (blue_lanes[2] + blue_lanes[3]);
  if (blue_sum >= 32.0f * kBlueLimit) blue_sum = 64.0f * kBlueLimit - blue_sum;
  blue_sum = fminf(blue_sum, 15.463398341612438f * kBlueLimit);
  const float blue_value = gamma_value + blue_sum * 0.90590804735610064f;
  const float exponent = fminf(hf_value, blue_value);
  const float result = FastPow2(exponent * 1.442695041f) * p.multiplier + p.addend;
  if (!(IsFinite(result) && result > 0.0f) || !(IsFinite(strategy) && strategy > 0.0f)) {
    RaiseError(p.error, kErrorNonFiniteOutput);
  }
  p.quant_field[block] = result;
  p.strategy_mask[block] = strategy;
}

// MirrorCoordinate (src/core/image_ops.h:20-49) for |offset| <= 2.
__device__ __forceinline__ int Mirror(int c, int n) {
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

struct Symmetric5Params {
  const float* input;
  float* output;
  size_t in_stride, in_pitch, out_stride, out_pitch;
  uint32_t width, height, planes;
  // distance0, distance1, distance2, distance4, distance8, distance5 per plane
  float w[3][6];
  uint32_t* error;
};


// One CTA of 32x8 threads per 32x32 output tile (four rows per thread): the
// tile with a mirrored 2-pixel halo is staged in shared memory with a 2D
// thread mapping, all of a thread's loads issued before its first store
// (tiles whose window lies inside the image skip the mirroring); then every
// output reads its 5x5 neighbourhood from there.
constexpr int kS5W = 32, kS5H = 32, kS5Rows = 8;

// WeightedRow (src/codec/convolution.cpp:14-30): far + (near + center), on a
// staged row (the halo is already mirrored).
__device__ __forceinline__ float WeightedTileRow(const float* row, float c, float n, float f) {
  const float far = f * (row[-2] + row[2]);
  const float near = n * (row[-1] + row[1]);
  const float center = c * row[0];
  return far + (near + center);
}

__global__ void __launch_bounds__(kS5W * kS5Rows)
Symmetric5Kernel(const __grid_constant__ Symmetric5Params p) {
  constexpr int TW = kS5W + 4, TH = kS5H + 4;
  constexpr int kCols = (TW + kS5W - 1) / kS5W, kRows = (TH + kS5Rows - 1) / kS5Rows;
  __shared__ float tile[TH][TW];
  const uint32_t plane = blockIdx.z;
  const int x0 = blockIdx.x * kS5W, y0 = blockIdx.y * kS5H;
  const int h = p.height, wd = p.width;
  const float* in = p.input + plane * p.in_pitch;
  const bool interior = x0 >= 2 && y0 >= 2 && x0 + kS5W + 2 <= wd && y0 + kS5H + 2 <= h;
  float staged[kRows][kCols];
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
#pragma unroll
    for (int k = 0; k < kCols; ++k) {
      const int ty = threadIdx.y + r * kS5Rows, tx = threadIdx.x + k * kS5W;
      if (ty < TH && tx < TW) {
        int gy = y0 + ty - 2, gx = x0 + tx - 2;
        if (!interior) {
          gy = Mirror(gy, h);
          gx = Mirror(gx, wd);
        }
        staged[r][k] = in[static_cast<size_t>(gy) * p.in_stride + gx];
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
#pragma unroll
    for (int k = 0; k < kCols; ++k) {
      const int ty = threadIdx.y + r * kS5Rows, tx = threadIdx.x + k * kS5W;
      if (ty < TH && tx < TW) tile[ty][tx] = staged[r][k];
    }
  }
  __syncthreads();
  const int x = x0 + threadIdx.x;
  if (x >= wd) return;
  const float* w = p.w[plane];
  const int cx = threadIdx.x + 2;
#pragma unroll
  for (int row = 0; row < kS5H / kS5Rows; ++row) {
    const int oy = threadIdx.y + row * kS5Rows, y = y0 + oy;
    if (y >= h) break;
    const int cy = oy + 2;
    float sum0 = WeightedTileRow(&tile[cy][cx], w[0], w[1], w[2]);
    sum0 += WeightedTileRow(&tile[cy - 2][cx], w[2], w[5], w[4]);
    float sum1 = WeightedTileRow(&tile[cy + 2][cx], w[2], w[5], w[4]);
    sum0 += WeightedTileRow(&tile[cy - 1][cx], w[1], w[3], w[5]);
    sum1 += WeightedTileRow(&tile[cy + 1][cx], w[1], w[3], w[5]);
    const float v = sum0 + sum1;
    if (!IsFinite(v)) RaiseError(p.error, kErrorNonFiniteOutput);
    p.output[plane * p.out_pitch + static_cast<size_t>(y) * p.out_stride + x] = v;
  }
}

// gaborish.cpp:11-35.
void GaborishInverseWeights(float multiplier, float out[6]) {
  const float k[5] = {-0.09495815671340026f, -0.041031725066768575f, 0.013710004822696948f,
                      0.006510206083837737f, -0.0014789063378272242f};
  double sum = 1.0 + static_cast<double>(multiplier) * 4.0 *
                       (k[0] + k[1] + k[2] + k[4] + 2.0 * k[3]);
  sum = std::max(sum, 1.0e-5);
  const float normalize = static_cast<float>(1.0 / sum);
  const float nm = multiplier * normalize;
  out[0] = normalize;
  out[1] = nm * k[0];
  out[2] = nm * k[2];
  out[3] = nm * k[1];
  out[4] = nm * k[4];
  out[5] = nm * k[3];
}

// adaptive_quantization.cpp:305-341 (BlurPixelMask weights).
void PixelMaskBlurWeights(float out[6]) {
  const float f[5] = {0.364911248f, 0.05f, 0.1688888021f, 0.221069183f, 0.306563504f};
  double weight_sum = 1.0 + 4.0 * (f[0] + f[1] + f[2] + f[4] + 2.0 * f[3]);
  weight_sum = std::max(weight_sum, 1.0e-5);
  const float normalize = static_cast<float>(1.0 / weight_sum);
  out[0] = normalize;
  out[1] = normalize * f[0];
  out[2] = normalize * f[2];
  out[3] = normalize * f[1];
  out[4] = normalize * f[4];
  out[5] = normalize * f[3];
}

int LaunchSymmetric5(const float* input, size_t in_stride, size_t in_pitch, float* output,
                     size_t out_stride, size_t out_pitch, size_t width, size_t height,
                     uint32_t planes, const float weights[][6], uint32_t* error,
                     cudaStream_t stream) {
  Symmetric5Params p;
  std::memset(&p, 0, sizeof(p));
  p.input = input;
  p.output = output;
  p.in_stride = in_stride;
  p.in_pitch = in_pitch;
  p.out_stride = out_stride;
  p.out_pitch = out_pitch;
  p.width = static_cast<uint32_t>(width);
  p.height = static_cast<uint32_t>(height);
  p.planes = planes;
  for (uint32_t c = 0; c < planes; ++c) std::memcpy(p.w[c], weights[c], sizeof(p.w[c]));
  p.error = error;
  if ((height + kS5H - 1) / kS5H > 65535) {
    return SetError(GJXL_B200_UNSUPPORTED, "symmetric5: image taller than 2,097,120 rows");
  }
  dim3 grid(static_cast<unsigned>((width + kS5W - 1) / kS5W),
            static_cast<unsigned>((height + kS5H - 1) / kS5H), planes);
  Symmetric5Kernel<<<grid, dim3(kS5W, kS5Rows), 0, stream>>>(p);
  return CheckLaunch("symmetric5");
}

}  // namespace

size_t InitialQuantScratchFloats(size_t padded_width, size_t padded_height) {
  // raw pixel mask + pre-erosion grid
  return padded_width * padded_height + (padded_width / 4) * (padded_height / 4);
}

int LaunchInitialQuantField(const float* opsin, size_t stride, size_t pitch, size_t pw,
                            size_t ph, float target, float rescale, float* quant_field,
                            float* strategy_mask, float* pixel_mask, size_t mask_stride,
                            float* scratch, uint32_t* error, cudaStream_t stream) {
  float* raw_mask = scratch;
  float* pre_erosion = scratch + pw * ph;

  PreErosionParams pe;
  pe.y_plane = opsin + pitch;
  pe.stride = stride;
  pe.width = static_cast<uint32_t>(pw);
  pe.height = static_cast<uint32_t>(ph);
  pe.raw_pixel_mask = raw_mask;
  pe.mask_stride = pw;
  pe.pre_erosion = pre_erosion;
  pe.masking_inner_scale = std::sqrt(211.66567973503678f * 1.0e8f);
  const uint64_t cells = static_cast<uint64_t>(pw / 4) * (ph / 4);
  PreErosionKernel<<<static_cast<unsigned>((cells + 255) / 256), 256, 0, stream>>>(pe);
  int status = CheckLaunch("initial_quant pre-erosion");
  if (status != GJXL_B200_OK) return status;

  ModulationParams mp;
  std::memset(&mp, 0, sizeof(mp));
  mp.opsin = opsin;
  mp.stride = stride;
  mp.pitch = pitch;
  mp.blocks_x = static_cast<uint32_t>(pw / 8);
  mp.blocks_y = static_cast<uint32_t>(ph / 8);
  mp.pre_erosion = pre_erosion;
  // FuzzyErosion weights (adaptive_quantization.cpp:199-223).
  const float mul_base[4] = {0.125f, 0.1f, 0.09f, 0.06f};
  const float mul_add[4] = {0.0f, -0.1f, -0.09f, -0.06f};
  const float total = 0.29959705784054957f;
  float target_mix = 0.0f;
  if (target < 2.0f) target_mix = (2.0f - target) * 0.5f;
  float weight_sum = 0.0f;
  for (int i = 0; i < 4; ++i) {
    mp.weights[i] = mul_base[i] + target_mix * mul_add[i];
    weight_sum += mp.weights[i];
  }
  for (int i = 0; i < 4; ++i) mp.weights[i] *= total / weight_sum;
  // PerBlockModulations scale terms (adaptive_quantization.cpp:446-458).
  const float scale = 0.765f / target * rescale;
  const float base_level = 0.48f * scale;
  float dampen = 1.0f;
  if (target >= 2.0f) {
    dampen = 1.0f - (target - 2.0f) / 12.0f;
    dampen = std::max(dampen, 0.0f);
  }
  mp.multiplier = scale * dampen;
  mp.addend = (1.0f - dampen) * base_level;
  mp.quant_field = quant_field;
  mp.strategy_mask = strategy_mask;
  mp.error = error;
  const uint64_t blocks = static_cast<uint64_t>(mp.blocks_x) * mp.blocks_y;
  ErosionModulationKernel<<<static_cast<unsigned>((blocks + 127) / 128), 128, 0, stream>>>(mp);
  status = CheckLaunch("initial_quant modulation");
  if (status != GJXL_B200_OK) return status;

  float blur[1][6];
  PixelMaskBlurWeights(blur[0]);
  return LaunchSymmetric5(raw_mask, pw, pw * ph, pixel_mask, mask_stride, mask_stride * ph, pw,
                          ph, 1, blur, error, stream);
}

int LaunchGaborishInverse(const float* input, size_t in_stride, size_t in_pitch, float* output,
                          size_t out_stride, size_t out_pitch, size_t width, size_t height,
                          const float multipliers[3], uint32_t* error, cudaStream_t stream) {
  float w[3][6];
  for (int c = 0; c < 3; ++c) GaborishInverseWeights(multipliers[c], w[c]);
  return LaunchSymmetric5(input, in_stride, in_pitch, output, out_stride, out_pitch, width,
                          height, 3, w, error, stream);
}

}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" size_t gjxl_b200_initial_quant_scratch_bytes(size_t padded_width,
                                                        size_t padded_height) {
  return InitialQuantScratchFloats(padded_width, padded_height) * sizeof(float);
}

extern "C" int gjxl_b200_initial_quant_field(
  const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch, size_t padded_width,
  size_t padded_height, float butteraugli_target, float rescale, float* quant_field,
  float* strategy_mask, float* pixel_mask, size_t pixel_mask_stride, void* scratch,
  size_t scratch_bytes, uint32_t* device_error, void* stream) {
  ClearLastError();
  if (opsin == nullptr || quant_field == nullptr || strategy_mask == nullptr ||
      pixel_mask == nullptr || scratch == nullptr || padded_width % 8 != 0 ||
      padded_height % 8 != 0 || padded_width == 0 || padded_height == 0 ||
      opsin_stride % 4 != 0 || opsin_plane_pitch % 4 != 0 || opsin_stride < padded_width ||
      !Aligned16(opsin) ||
      opsin_plane_pitch < opsin_stride * padded_height || pixel_mask_stride < padded_width ||
      !std::isfinite(butteraugli_target) || butteraugli_target <= 0.0f ||
      !std::isfinite(rescale) || rescale <= 0.0f || !Aligned16(scratch) ||
      scratch_bytes < gjxl_b200_initial_quant_scratch_bytes(padded_width, padded_height)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "initial_quant_field: invalid arguments");
  }
  return LaunchInitialQuantField(opsin, opsin_stride, opsin_plane_pitch, padded_width,
                                 padded_height, butteraugli_target, rescale, quant_field,
                                 strategy_mask, pixel_mask, pixel_mask_stride,
                                 static_cast<float*>(scratch), device_error,
                                 static_cast<cudaStream_t>(stream));
}

extern "C" int gjxl_b200_gaborish_inverse(const float* input, size_t input_stride,
                                          size_t input_plane_pitch, float* output,
                                          size_t output_stride, size_t output_plane_pitch,
                                          size_t width, size_t height,
                                          const float* multipliers, uint32_t* device_error,
                                          void* stream) {
  ClearLastError();
  if (input == nullptr || output == nullptr || input == output || width == 0 || height == 0 ||
      input_stride < width || output_stride < width || multipliers == nullptr ||
      width > 0x7fffffff || height > 0x7fffffff) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "gaborish_inverse: invalid arguments");
  }
  for (int c = 0; c < 3; ++c) {
    if (!std::isfinite(multipliers[c])) {
      return SetError(GJXL_B200_INVALID_ARGUMENT, "gaborish_inverse: non-finite multiplier");
    }
  }
  return LaunchGaborishInverse(input, input_stride, input_plane_pitch, output, output_stride,
                               output_plane_pitch, width, height, multipliers, device_error,
                               static_cast<cudaStream_t>(stream));
}
