// Rows a14/a15: Butteraugli distance map, its multiscale combination and
// global maximum, with a prepared (cached) reference image.
//
// Restates the reference's scalar Butteraugli (adapted there from libjxl):
//   src/codec/butteraugli_internal.cpp   Gaussian blurs (Separable5 :206-260,
//     ConvolutionWithTranspose :309-423, kernel :588-621), OpsinDynamicsImage
//     (:623-684), SeparateFrequencies (:728-856);
//   src/codec/butteraugli_distance_internal.cpp  Malta units (:156-281),
//     masking (:283-317, :561-628), L2 terms (:405-516), MaltaDiffMap
//     (:518-586), ComputeDifferenceStages (:657-851), multiscale driver
//     (:853-990), prepared reference (:992-1202).
// Every float operation keeps the reference's association and rounding:
// Highway's scalar MulAdd is an unfused multiply then add (--fmad=false), the
// mixed float/double steps of the Malta scaling and the masks are done in
// double exactly where the reference promotes, and the blur kernels come from
// the host C library's exp() exactly as in the reference.
//
// The reference blurs with two "convolve rows, write transposed" passes; here
// the second pass reads columns directly (same per-output arithmetic, no
// transposed copy). Planes are dense float32 (stride = width).

#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "host_util.h"

namespace gjxl_b200 {
namespace {

constexpr int kThreads = 256;

// --------------------------------------------------------------------------
// Blur kernels.

struct Kernel17 {
  float raw[33];     // unnormalized taps, index -r..r -> 0..2r
  float scaled[17];  // raw[i] * (1 / sum(raw)), i <= r
  float w5[3];       // Separable5 weights (center, +-1, +-2)
};

// Mirror (butteraugli_internal.cpp:196-204): reflect with the edge repeated.
__device__ __forceinline__ int MirrorB(int c, int size) {
  while (c < 0 || c >= size) c = c < 0 ? -c - 1 : 2 * size - 1 - c;
  return c;
}

// Separable5 (butteraugli_internal.cpp:222-260) runs on 32x32 output tiles
// of 32x8 threads (four output rows each): the mirrored input window (tile +
// 2 on each side) is staged in shared memory, all of a thread's loads issued
// before its first store; tiles whose window lies inside the image skip the
// mirroring. The horizontal 5-tap pass runs over the window's 36 rows, then
// the vertical pass, with the reference's operation order for every output
// (Blur5DynamicsKernel).
constexpr int kB5W = 32, kB5H = 32, kB5Rows = 8;

// ConvolveBorderColumn's renormalized sum at position x of a line of length
// n (samples at src[j * step]), with the taps unrolled: tap t reads sample
// x - R + t; taps outside the line add +0.0, which leaves both sums (never
// -0.0) unchanged, so the sums equal the reference's sums over the taps
// inside the line, in the same order. All samples are loaded first.
template <int R>
__device__ __forceinline__ float ConvolveBorder(const float* src, int step, int x, int n,
                                                const Kernel17& k) {
  float sample[2 * R + 1];
#pragma unroll
  for (int t = 0; t <= 2 * R; ++t) {
    const int j = x - R + t;
    sample[t] = j >= 0 && j < n ? src[static_cast<ptrdiff_t>(j) * step] : 0.0f;
  }
  float weight = 0.0f, sum = 0.0f;
#pragma unroll
  for (int t = 0; t <= 2 * R; ++t) {
    const int j = x - R + t;
    const bool inside = j >= 0 && j < n;
    weight += inside ? k.raw[t] : 0.0f;
    sum += inside ? sample[t] * k.raw[t] : 0.0f;
  }
  const float scale = 1.0f / weight;
  return sum * scale;
}

// One tap row of ConvolutionWithTranspose at position x of a line of length n
// (samples at src[j * step]). Interior: pair sums folded round-robin into four
// partial sums (ConvolveInterior7/13/15/33); border: renormalized direct sum
// (ConvolveBorderColumn).
template <int R>
__device__ __forceinline__ float ConvolveLine(const float* src, int step, int x, int n,
                                              const Kernel17& k) {
  if (x >= R && x < n - R) {
    const float* s = src + static_cast<ptrdiff_t>(x - R) * step;
    float sums[4];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const float term = (s[i * step] + s[(2 * R - i) * step]) * k.scaled[i];
      if (i < 4) {
        sums[i] = term;
      } else {
        sums[i & 3] += term;
      }
    }
    float out = s[R * step] * k.scaled[R];
#pragma unroll
    for (int i = 0; i < (R < 4 ? R : 4); ++i) out = out + sums[i];
    return out;
  }
  return ConvolveBorder<R>(src, step, x, n, k);
}

// Register-blocked blur along one axis: each thread computes kRun
// consecutive outputs of one line from a window of kRun + 2R samples held in
// registers (the interior pair-sum order of ConvolveLine for every output),
// and falls back to ConvolveLine for outputs within R of either end.
constexpr int kRun = 8;

template <int R>
__device__ __forceinline__ void ConvolveRun(const float* src, int step, int first, int n,
                                            const Kernel17& k, float* out, int out_step,
                                            int count) {
  if (first >= R && first + kRun - 1 < n - R) {
    float v[kRun + 2 * R];
    const float* s = src + static_cast<ptrdiff_t>(first - R) * step;
#pragma unroll
    for (int j = 0; j < kRun + 2 * R; ++j) v[j] = s[static_cast<ptrdiff_t>(j) * step];
#pragma unroll
    for (int o = 0; o < kRun; ++o) {
      float sums[4];
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const float term = (v[o + i] + v[o + 2 * R - i]) * k.scaled[i];
        if (i < 4) {
          sums[i] = term;
        } else {
          sums[i & 3] += term;
        }
      }
      float r = v[o + R] * k.scaled[R];
#pragma unroll
      for (int i = 0; i < (R < 4 ? R : 4); ++i) r = r + sums[i];
      out[static_cast<ptrdiff_t>(o) * out_step] = r;
    }
    return;
  }
  for (int o = 0; o < count; ++o) {
    out[static_cast<ptrdiff_t>(o) * out_step] = ConvolveLine<R>(src, step, first + o, n, k);
  }
}

// Interior outputs o = 0..kOut-1 of a register window v[kOut + 2R] (output o
// centred on v[o + R]), in ConvolveLine's pair-sum order.
template <int R, int kOut>
__device__ __forceinline__ void ConvolveWindow(const float (&v)[kOut + 2 * R], const Kernel17& k,
                                               float (&r)[kOut]) {
#pragma unroll
  for (int o = 0; o < kOut; ++o) {
    float sums[4];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const float term = (v[o + i] + v[o + 2 * R - i]) * k.scaled[i];
      if (i < 4) {
        sums[i] = term;
      } else {
        sums[i & 3] += term;
      }
    }
    float out = v[o + R] * k.scaled[R];
#pragma unroll
    for (int i = 0; i < (R < 4 ? R : 4); ++i) out = out + sums[i];
    r[o] = out;
  }
}

// Row blur: one CTA per 1024-sample segment of kBlurRows consecutive rows.
// The segments and their R-sample halos are loaded with coalesced loads, all
// rows' loads in flight at once (more bytes in flight per SM than one row per
// CTA gives), into shared rows whose pitch is a multiple of 4 floats. Each
// thread then reads the window of its 4 outputs with 128-bit (and, for odd
// R, one 64-bit) shared loads. Outputs within R of the row ends use
// ConvolveLine's renormalized border sum.
constexpr int kRowRun = 4;
constexpr int kRowSegment = kThreads * kRowRun;
constexpr int kBlurRows = 2;

template <int R>
__global__ void __launch_bounds__(kThreads)
BlurRowsKernel(const float* in, float* out, int w, int h, size_t in_pitch, size_t out_pitch,
               const __grid_constant__ Kernel17 k) {
  constexpr int kWindow = kRowRun + 2 * R;
  constexpr int kSpan = kRowSegment + 2 * R;
  constexpr int kLoads = (kSpan + kThreads - 1) / kThreads;
  constexpr int kPitch = (kSpan + 4 + 3) / 4 * 4;  // 16-byte aligned rows
  __shared__ __align__(16) float segment[kBlurRows][kPitch];
  const int plane = blockIdx.z;
  const int x0 = blockIdx.x * kRowSegment;
  const float* base = in + plane * in_pitch;
  // Rows beyond the grid's y extent (65535 row groups) are taken in further
  // rounds.
  for (int y0 = blockIdx.y * kBlurRows; y0 < h; y0 += gridDim.y * kBlurRows) {
    __syncthreads();
    // segment[r][j] holds sample x0 - R + j of row y0 + r.
    float staged[kBlurRows][kLoads];
#pragma unroll
    for (int r = 0; r < kBlurRows; ++r) {
      const float* row = base + static_cast<size_t>(min(y0 + r, h - 1)) * w;
#pragma unroll
      for (int q = 0; q < kLoads; ++q) {
        const int j = threadIdx.x + q * kThreads, x = x0 - R + j;
        staged[r][q] = j < kSpan && x >= 0 && x < w ? row[x] : 0.0f;
      }
    }
#pragma unroll
    for (int r = 0; r < kBlurRows; ++r) {
#pragma unroll
      for (int q = 0; q < kLoads; ++q) {
        const int j = threadIdx.x + q * kThreads;
        if (j < kSpan) segment[r][j] = staged[r][q];
      }
    }
    __syncthreads();
    const int first = x0 + threadIdx.x * kRowRun;
    if (first >= w) continue;
#pragma unroll 1
    for (int r = 0; r < kBlurRows && y0 + r < h; ++r) {
      const int y = y0 + r;
      float* dst = out + plane * out_pitch + static_cast<size_t>(y) * w + first;
      {
        float v[kWindow];
        const float* s = segment[r] + threadIdx.x * kRowRun;
#pragma unroll
        for (int j = 0; j + 4 <= kWindow; j += 4) {
          const float4 f = *reinterpret_cast<const float4*>(s + j);
          v[j] = f.x;
          v[j + 1] = f.y;
          v[j + 2] = f.z;
          v[j + 3] = f.w;
        }
        if constexpr (kWindow % 4 == 2) {
          const float2 f = *reinterpret_cast<const float2*>(s + kWindow - 2);
          v[kWindow - 2] = f.x;
          v[kWindow - 1] = f.y;
        }
        // Every thread computes its four outputs from the window; only the
        // interior ones are stored (the border CTA writes the others).
        float o4[kRowRun];
        ConvolveWindow<R, kRowRun>(v, k, o4);
#pragma unroll
        for (int o = 0; o < kRowRun; ++o) {
          if (first + o >= R && first + o < w - R) dst[o] = o4[o];
        }
      }
    }
  }
}

// The outputs within R of either row end (ConvolveLine's renormalized border
// sum), for the rows of the row-blur CTAs: one thread per row and border
// position, so that the row-blur CTAs run no divergent border code. The
// positions are x = 0..R-1 and x = w-2R+R..w-1, the latter kept only where
// x >= R (narrow rows).
template <int R>
__global__ void __launch_bounds__(kThreads)
BlurRowBordersKernel(const float* in, float* out, int w, int h, size_t in_pitch,
                     size_t out_pitch, const __grid_constant__ Kernel17 k) {
  constexpr int kPerRow = 2 * R;
  constexpr int kRowsPerCta = kThreads / kPerRow;
  const int plane = blockIdx.y;
  const int r = threadIdx.x / kPerRow, item = threadIdx.x % kPerRow;
  const int y = blockIdx.x * kRowsPerCta + r;
  if (r >= kRowsPerCta || y >= h) return;
  const int x = item < R ? item : w - kPerRow + item;
  if (item < R ? x >= w : (x < R || x >= w)) return;
  const float* row = in + plane * in_pitch + static_cast<size_t>(y) * w;
  out[plane * out_pitch + static_cast<size_t>(y) * w + x] = ConvolveBorder<R>(row, 1, x, w, k);
}

template <int R>
__global__ void __launch_bounds__(kThreads)
BlurColumnsKernel(const float* in, float* out, int w, int h, size_t in_pitch, size_t out_pitch,
                  const __grid_constant__ Kernel17 k) {
  const int plane = blockIdx.y;
  const int runs = (h + kRun - 1) / kRun;
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= w * runs) return;
  // Consecutive threads take consecutive columns of one run of rows, so the
  // window loads are coalesced across the warp.
  const int x = i % w, y = (i / w) * kRun;
  const float* column = in + plane * in_pitch + x;
  ConvolveRun<R>(column, w, y, h, k, out + plane * out_pitch + static_cast<size_t>(y) * w + x, w,
                 min(kRun, h - y));
}

// --------------------------------------------------------------------------
// Opsin dynamics and frequency separation.

__device__ __forceinline__ float ButteraugliFastLog2(float value) {
  const uint32_t bits = __float_as_uint(value);
  const int32_t e = static_cast<int32_t>(bits - 0x3f2aaaabu) >> 23;
  const float x = __uint_as_float(bits - (static_cast<uint32_t>(e) << 23)) - 1.0f;
  float num = 0.74245873327820566f * x + 1.4287160470083755f;
  num = num * x + -1.8503833400518310e-06f;
  float den = 0.17409343003366853f * x + 1.0096718572241148f;
  den = den * x + 0.99032814277590719f;
  return num / den + static_cast<float>(e);
}

__device__ __forceinline__ float GammaB(float value) {
  constexpr float kRetMul = 19.245013259874995f * 0.6931471805599453f;
  value = fmaxf(value, 0.0f);
  return kRetMul * ButteraugliFastLog2(value + 9.9710635769299145f) + -23.16046239805755f;
}

template <bool Clamp>
__device__ __forceinline__ void OpsinAbsorbance(float r, float g, float b, float& o0, float& o1,
                                                float& o2) {
  constexpr float k0 = 0.29956550340058319f, k1 = 0.63373087833825936f,
                  k2 = 0.077705617820981968f, k3 = 1.7557483643287353f,
                  k4 = 0.22158691104574774f, k5 = 0.69391388044116142f, k6 = 0.0987313588422f,
                  k7 = 1.7557483643287353f, k8 = 0.02f, k9 = 0.02f,
                  k10 = 0.20480129041026129f, k11 = 12.226454707163354f;
  o0 = k0 * r + (k1 * g + (k2 * b + k3));
  o1 = k4 * r + (k5 * g + (k6 * b + k7));
  o2 = k8 * r + (k9 * g + (k10 * b + k11));
  if (Clamp) {
    o0 = fmaxf(o0, k3);
    o1 = fmaxf(o1, k7);
    o2 = fmaxf(o2, k11);
  }
}

// OpsinDynamicsImage (butteraugli_internal.cpp:624-690) of one pixel: the
// blurred sample (b0, b1, b2) sets the sensitivity, the linear sample
// (r, g, b) is converted; writes XYB pixel i of the three planes.
__device__ __forceinline__ void OpsinDynamicsPixel(float b0, float b1, float b2, float r, float g,
                                                   float b, float* xyb, size_t i, size_t pitch,
                                                   float intensity, uint32_t* error) {
  float p0, p1, p2;
  OpsinAbsorbance<true>(b0 * intensity, b1 * intensity, b2 * intensity, p0, p1, p2);
  p0 = fmaxf(p0, 1.0e-4f);
  p1 = fmaxf(p1, 1.0e-4f);
  p2 = fmaxf(p2, 1.0e-4f);
  const float s0 = fmaxf(GammaB(p0) / p0, 1.0e-4f);
  const float s1 = fmaxf(GammaB(p1) / p1, 1.0e-4f);
  const float s2 = fmaxf(GammaB(p2) / p2, 1.0e-4f);
  // A non-finite input sample would be absorbed by the clamps below (fmaxf
  // returns the other operand for a NaN), so it is reported here.
  if (!(IsFinite(r) && IsFinite(g) && IsFinite(b))) RaiseError(error, kErrorNonFiniteInput);
  float c0, c1, c2;
  OpsinAbsorbance<false>(r * intensity, g * intensity, b * intensity, c0, c1, c2);
  c0 = fmaxf(c0 * s0, 1.7557483643287353f);
  c1 = fmaxf(c1 * s1, 1.7557483643287353f);
  c2 = fmaxf(c2 * s2, 12.226454707163354f);
  const float ox = c0 - c1, oy = c0 + c1;
  if (!IsFinite(ox) || !IsFinite(oy) || !IsFinite(c2)) RaiseError(error, kErrorNonFiniteOutput);
  xyb[i] = ox;
  xyb[pitch + i] = oy;
  xyb[2 * pitch + i] = c2;
}

// Separable5 of the three planes of a dense linear image with
// OpsinDynamicsPixel applied to each output
// pixel: the blurred planes stay in registers, the pixel's linear sample is
// the window's centre. Writes the three XYB planes.
__global__ void __launch_bounds__(kB5W * kB5Rows)
Blur5DynamicsKernel(const float* in, float* xyb, int w, int h, size_t pitch,
                    const __grid_constant__ Kernel17 k, float intensity, uint32_t* error) {
  constexpr int kSpanW = kB5W + 4, kSpanH = kB5H + 4, kSpan = kSpanW * kSpanH;
  constexpr int kThreadsB5 = kB5W * kB5Rows;
  constexpr int kLoads = (kSpan + kThreadsB5 - 1) / kThreadsB5;
  __shared__ float window[3][kSpanH][kSpanW];
  __shared__ float horizontal[3][kSpanH][kB5W];
  const int x0 = blockIdx.x * kB5W, y0 = blockIdx.y * kB5H;
  const int tid = threadIdx.y * kB5W + threadIdx.x;
  const bool interior = x0 >= 2 && y0 >= 2 && x0 + kSpanW - 2 <= w && y0 + kSpanH - 2 <= h;
#pragma unroll
  for (int plane = 0; plane < 3; ++plane) {
    const float* base = in + plane * pitch;
    float staged[kLoads];
#pragma unroll
    for (int q = 0; q < kLoads; ++q) {
      const int i = tid + q * kThreadsB5;
      if (i < kSpan) {
        const int ty = i / kSpanW, tx = i - ty * kSpanW;
        int gy = y0 + ty - 2, gx = x0 + tx - 2;
        if (!interior) {
          gy = MirrorB(gy, h);
          gx = MirrorB(gx, w);
        }
        staged[q] = base[static_cast<size_t>(gy) * w + gx];
      }
    }
#pragma unroll
    for (int q = 0; q < kLoads; ++q) {
      const int i = tid + q * kThreadsB5;
      if (i < kSpan) {
        const int ty = i / kSpanW, tx = i - ty * kSpanW;
        window[plane][ty][tx] = staged[q];
      }
    }
  }
  __syncthreads();
  const int tx = threadIdx.x;
#pragma unroll
  for (int plane = 0; plane < 3; ++plane) {
#pragma unroll
    for (int ty = threadIdx.y; ty < kSpanH; ty += kB5Rows) {
      const float* row = window[plane][ty] + tx + 2;
      float r = row[0] * k.w5[0];
      r = (row[-1] + row[1]) * k.w5[1] + r;
      r = (row[-2] + row[2]) * k.w5[2] + r;
      horizontal[plane][ty][tx] = r;
    }
  }
  __syncthreads();
  const int x = x0 + tx;
  if (x >= w) return;
#pragma unroll
  for (int q = 0; q < kB5H / kB5Rows; ++q) {
    const int oy = threadIdx.y + q * kB5Rows, y = y0 + oy;
    if (y >= h) break;
    const int ty = oy + 2;
    float blurred[3];
#pragma unroll
    for (int plane = 0; plane < 3; ++plane) {
      const auto& hz = horizontal[plane];
      float r = hz[ty][tx] * k.w5[0];
      r = (hz[ty - 1][tx] + hz[ty + 1][tx]) * k.w5[1] + r;
      r = (hz[ty - 2][tx] + hz[ty + 2][tx]) * k.w5[2] + r;
      blurred[plane] = r;
    }
    OpsinDynamicsPixel(blurred[0], blurred[1], blurred[2], window[0][ty][tx + 2],
                       window[1][ty][tx + 2], window[2][ty][tx + 2], xyb,
                       static_cast<size_t>(y) * w + x, pitch, intensity, error);
  }
}

// Psycho-image plane indices (OwnedPsychoImage): LF 0-2, MF 3-5, HF 6-7,
// UHF 8-9.
enum : int { kLF = 0, kMF = 3, kHF = 6, kUHF = 8, kPsychoPlanes = 10 };

__device__ __forceinline__ float RemoveRangeAroundZero(float v, float w) {
  return v > w ? v - w : v < -w ? v + w : 0.0f;
}
__device__ __forceinline__ float AmplifyRangeAroundZero(float v, float w) {
  return v > w ? v + w : v < -w ? v - w : v + v;
}
__device__ __forceinline__ float MaximumClamp(float v, float m) {
  constexpr float kMul = 0.724216145665f;
  if (v >= m) return (v - m) * kMul + m;
  if (v < -m) return (v + m) * kMul + -m;
  return v;
}

// Constants of one MaltaDiffMap stage: float casts of pre * norm (for
// differences above and below the reference) and of the norm.
struct MaltaScale {
  float norm2_gt, norm2_lt, norm;
};

// Scaled difference of MaltaDiffMap (butteraugli_distance_internal.cpp:544-575)
// of the samples v0 (reference side) and v1 at one position.
__device__ __forceinline__ float MaltaScaledValue(const MaltaScale& p, float v0, float v1) {
  const float absolute = 0.5f * (fabsf(v0) + fabsf(v1));
  const float difference = v0 - v1;
  const float scaler = p.norm2_gt / (p.norm + absolute);
  float scaled = scaler * difference;
  const float scaler2 = p.norm2_lt / (p.norm + absolute);
  const double magnitude = fabs(static_cast<double>(v0));
  const double too_small = 0.55 * magnitude;
  const double too_big = 1.05 * magnitude;
  const double s2 = static_cast<double>(scaler2);
  const double d1 = static_cast<double>(v1);
  if (v0 < 0.0f) {
    if (d1 > -too_small) {
      scaled = static_cast<float>(static_cast<double>(scaled) - s2 * (d1 + too_small));
    } else if (d1 < -too_big) {
      scaled = static_cast<float>(static_cast<double>(scaled) + s2 * (-d1 - too_big));
    }
  } else if (d1 < too_small) {
    scaled = static_cast<float>(static_cast<double>(scaled) + s2 * (too_small - d1));
  } else if (d1 > too_big) {
    scaled = static_cast<float>(static_cast<double>(scaled) - s2 * (d1 - too_big));
  }
  return scaled;
}

// After the 33-tap blur of all three XYB planes into psycho LF: MF = xyb - LF
// and the LF scaling (butteraugli_internal.cpp:750-776).
__global__ void __launch_bounds__(kThreads)
FrequencyLowKernel(const float* xyb, float* psycho, int n, size_t pitch, uint32_t* error) {
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  // All loads first: `psycho` is read and written, so loads after a store
  // could not be moved ahead of it.
  float lf[3], v[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    lf[c] = psycho[(kLF + c) * pitch + i];
    v[c] = xyb[c * pitch + i];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) psycho[(kMF + c) * pitch + i] = v[c] - lf[c];
  const float l2 = (-0.362267051518f * lf[1] + lf[2]) * 49.87984651440f;
  const float l0 = lf[0] * 33.832837186260f;
  const float l1 = lf[1] * 14.458268100570f;
  psycho[(kLF + 2) * pitch + i] = l2;
  psycho[(kLF + 0) * pitch + i] = l0;
  psycho[(kLF + 1) * pitch + i] = l1;
  if (!(IsFinite(l0) && IsFinite(l1) && IsFinite(l2))) RaiseError(error, kErrorNonFiniteOutput);
}

// After the 15-tap blur of MF into `blurred` (3 planes): HF = MF - blurred
// (X, Y), MF ranges, MF_B = blurred, then X suppression by Y
// (butteraugli_internal.cpp:778-810).
// The Malta stages' scaled differences of the distorted image against the
// reference, written beside the final planes they are taken from (plane k of
// `malta` for stage k: MF_Y, MF_X, HF_Y, HF_X, UHF_Y, UHF_X), so that each
// is computed once per pixel instead of once per Malta tile that reads it.
struct MaltaPlanes {
  const float* ref;  // reference psycho planes; null: the reference itself
  float* malta;      // 6 planes
  MaltaScale scale[6];
};

__global__ void __launch_bounds__(kThreads)
FrequencyHighKernel(const float* blurred, float* psycho, int n, size_t pitch, uint32_t* error,
                    const __grid_constant__ MaltaPlanes m) {
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const float mv0 = blurred[i], mv1 = blurred[pitch + i], mf_b = blurred[2 * pitch + i];
  float ref_mf0 = 0.0f, ref_mf1 = 0.0f;
  if (m.ref != nullptr) {
    ref_mf0 = m.ref[(kMF + 0) * pitch + i];
    ref_mf1 = m.ref[(kMF + 1) * pitch + i];
  }
  const float hf0 = psycho[(kMF + 0) * pitch + i] - mv0;
  const float hf1 = psycho[(kMF + 1) * pitch + i] - mv1;
  const float mf0 = RemoveRangeAroundZero(mv0, 0.29f);
  const float mf1 = AmplifyRangeAroundZero(mv1, 0.1f);
  psycho[(kMF + 0) * pitch + i] = mf0;
  psycho[(kMF + 1) * pitch + i] = mf1;
  psycho[(kMF + 2) * pitch + i] = mf_b;
  constexpr float kSuppress = 46.0f, kMinimumScale = 0.653020556257f;
  const float scaler =
    kSuppress / (hf1 * hf1 + kSuppress) * (1.0f - kMinimumScale) + kMinimumScale;
  psycho[(kHF + 0) * pitch + i] = scaler * hf0;
  psycho[(kHF + 1) * pitch + i] = hf1;
  if (m.ref != nullptr) {
    m.malta[0 * pitch + i] = MaltaScaledValue(m.scale[0], ref_mf1, mf1);
    m.malta[1 * pitch + i] = MaltaScaledValue(m.scale[1], ref_mf0, mf0);
  }
  // Finiteness of the final MF planes (the HF planes are rewritten, and
  // checked, by FrequencyUltraKernel).
  if (!(IsFinite(mf0) & IsFinite(mf1) & IsFinite(mf_b))) RaiseError(error, kErrorNonFiniteOutput);
}

// After the 7-tap blur of HF into `blurred` (2 planes): UHF and final HF
// (butteraugli_internal.cpp:812-849).
__global__ void __launch_bounds__(kThreads)
FrequencyUltraKernel(const float* blurred, float* psycho, int n, size_t pitch,
                     uint32_t* error, const __grid_constant__ MaltaPlanes m) {
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  float ref_hf0 = 0.0f, ref_hf1 = 0.0f, ref_uhf0 = 0.0f, ref_uhf1 = 0.0f;
  if (m.ref != nullptr) {
    ref_hf0 = m.ref[(kHF + 0) * pitch + i];
    ref_hf1 = m.ref[(kHF + 1) * pitch + i];
    ref_uhf0 = m.ref[(kUHF + 0) * pitch + i];
    ref_uhf1 = m.ref[(kUHF + 1) * pitch + i];
  }
  const float hv0 = blurred[i];
  const float ultra0 = psycho[(kHF + 0) * pitch + i];
  const float uhf0 = RemoveRangeAroundZero(ultra0 - hv0, 0.04f);
  const float hf0 = RemoveRangeAroundZero(hv0, 1.5f);
  const float hv1 = MaximumClamp(blurred[pitch + i], 28.4691806922f);
  const float ultra1 = psycho[(kHF + 1) * pitch + i];
  const float uv1 = MaximumClamp(ultra1 - hv1, 5.19175294647f);
  const float uhf1 = uv1 * 2.69313763794f;
  const float hf1 = AmplifyRangeAroundZero(hv1 * 2.155f, 0.132f);
  psycho[(kUHF + 0) * pitch + i] = uhf0;
  psycho[(kHF + 0) * pitch + i] = hf0;
  psycho[(kUHF + 1) * pitch + i] = uhf1;
  psycho[(kHF + 1) * pitch + i] = hf1;
  if (m.ref != nullptr) {
    m.malta[2 * pitch + i] = MaltaScaledValue(m.scale[2], ref_hf1, hf1);
    m.malta[3 * pitch + i] = MaltaScaledValue(m.scale[3], ref_hf0, hf0);
    m.malta[4 * pitch + i] = MaltaScaledValue(m.scale[4], ref_uhf1, uhf1);
    m.malta[5 * pitch + i] = MaltaScaledValue(m.scale[5], ref_uhf0, uhf0);
  }
  // Finiteness of the final HF and UHF planes; FrequencyLowKernel and
  // FrequencyHighKernel check the final LF and MF planes as they write them.
  if (!(IsFinite(uhf0) && IsFinite(hf0) && IsFinite(uhf1) && IsFinite(hf1))) {
    RaiseError(error, kErrorNonFiniteOutput);
  }
}

// --------------------------------------------------------------------------
// Difference stages.

struct MaltaParams {
  const float* scaled;  // the stage's scaled differences (MaltaPlanes)
  float* accumulate;    // block_diff_ac plane (+= stage value)
  int w, h;
  int tiles_x, tiles_y;  // output tiles of kMaltaTileW x kMaltaTileH
  int first;             // first stage of its channel: the plane starts at zero
  int tma;               // the window arrives by a tiled bulk tensor copy of `map`
  uint32_t* error;
};

__device__ __forceinline__ float Sum4(float a, float b, float c, float d) { return (a + b) + (c + d); }
__device__ __forceinline__ float Sum5(float a, float b, float c, float d, float e) {
  return Sum4(a, b, c, d + e);
}
__device__ __forceinline__ float Sum7(float a, float b, float c, float d, float e, float f,
                                      float g) {
  return Sum4(a, b, c, Sum4(d, e, f, g));
}
__device__ __forceinline__ float Sum9(float a, float b, float c, float d, float e, float f,
                                      float g, float h, float i) {
  return (Sum4(a, b, c, d) + Sum4(e, f, g, h)) + i;
}

// Output tile of one CTA: 64 x 16 pixels, each of the 256 threads computing
// kMaltaRun = 4 horizontally adjacent outputs. The scaled differences of the
// tile plus a 4-pixel halo (zero outside the image) are staged in shared
// memory from the stage's precomputed plane; every thread then copies the 9 x 12 window its four outputs read
// into registers with 128-bit loads, so each staged value is loaded once per
// thread instead of once per tap.
constexpr int kMaltaRun = 4;
constexpr int kMaltaTileW = 64, kMaltaTileH = 16;
constexpr int kMaltaHalo = 4;
constexpr int kMaltaSpanW = kMaltaTileW + 2 * kMaltaHalo;  // 72 (16-byte rows)
constexpr int kMaltaSpanH = kMaltaTileH + 2 * kMaltaHalo;  // 24
constexpr int kMaltaWindowW = kMaltaRun + 2 * kMaltaHalo;   // 12
constexpr int kMaltaThreads = (kMaltaTileW / kMaltaRun) * kMaltaTileH;

// MaltaUnitLf / MaltaUnitFull (butteraugli_distance_internal.cpp:156-281) at
// output k of the window: the 16 line sums with the reference's association.
template <bool kLowFrequency, int K>
__device__ __forceinline__ float MaltaUnit(const float (&v)[2 * kMaltaHalo + 1][kMaltaWindowW]) {
#define P(dx, dy) v[(dy) + kMaltaHalo][K + kMaltaHalo + (dx)]
  float r, s;
  if constexpr (kLowFrequency) {
    s = Sum5(P(-4, 0), P(-2, 0), P(0, 0), P(2, 0), P(4, 0));
    r = s * s;
    s = Sum5(P(0, -4), P(0, -2), P(0, 0), P(0, 2), P(0, 4)); r = s * s + r;
    s = Sum5(P(-3, -3), P(-2, -2), P(0, 0), P(2, 2), P(3, 3)); r = s * s + r;
    s = Sum5(P(3, -3), P(2, -2), P(0, 0), P(-2, 2), P(-3, 3)); r = s * s + r;
    s = Sum5(P(1, -4), P(1, -2), P(0, 0), P(-1, 2), P(-1, 4)); r = s * s + r;
    s = Sum5(P(-1, -4), P(-1, -2), P(0, 0), P(1, 2), P(1, 4)); r = s * s + r;
    s = Sum5(P(-4, -1), P(-2, -1), P(0, 0), P(2, 1), P(4, 1)); r = s * s + r;
    s = Sum5(P(-4, 1), P(-2, 1), P(0, 0), P(2, -1), P(4, -1)); r = s * s + r;
    s = Sum5(P(-2, -3), P(-1, -2), P(0, 0), P(1, 2), P(2, 3)); r = s * s + r;
    s = Sum5(P(2, -3), P(1, -2), P(0, 0), P(-1, 2), P(-2, 3)); r = s * s + r;
    s = Sum5(P(-3, -2), P(-2, -1), P(0, 0), P(2, 1), P(3, 2)); r = s * s + r;
    s = Sum5(P(3, -2), P(2, -1), P(0, 0), P(-2, 1), P(-3, 2)); r = s * s + r;
    s = Sum5(P(-4, 2), P(-2, 1), P(0, 0), P(2, -1), P(4, -2)); r = s * s + r;
    s = Sum5(P(-4, -2), P(-2, -1), P(0, 0), P(2, 1), P(4, 2)); r = s * s + r;
    s = Sum5(P(-2, -4), P(-1, -2), P(0, 0), P(1, 2), P(2, 4)); r = s * s + r;
    s = Sum5(P(2, -4), P(1, -2), P(0, 0), P(-1, 2), P(-2, 4)); r = s * s + r;
  } else {
    s = Sum9(P(-4, 0), P(-3, 0), P(-2, 0), P(-1, 0), P(0, 0), P(1, 0), P(2, 0), P(3, 0),
             P(4, 0));
    r = s * s;
    s = Sum9(P(0, -4), P(0, -3), P(0, -2), P(0, -1), P(0, 0), P(0, 1), P(0, 2), P(0, 3), P(0, 4));
    r = s * s + r;
    s = Sum7(P(-3, -3), P(-2, -2), P(-1, -1), P(0, 0), P(1, 1), P(2, 2), P(3, 3)); r = s * s + r;
    s = Sum7(P(3, -3), P(2, -2), P(1, -1), P(0, 0), P(-1, 1), P(-2, 2), P(-3, 3)); r = s * s + r;
    s = Sum9(P(1, -4), P(1, -3), P(1, -2), P(0, -1), P(0, 0), P(0, 1), P(-1, 2), P(-1, 3),
             P(-1, 4));
    r = s * s + r;
    s = Sum9(P(-1, -4), P(-1, -3), P(-1, -2), P(0, -1), P(0, 0), P(0, 1), P(1, 2), P(1, 3),
             P(1, 4));
    r = s * s + r;
    s = Sum9(P(-4, -1), P(-3, -1), P(-2, -1), P(-1, 0), P(0, 0), P(1, 0), P(2, 1), P(3, 1),
             P(4, 1));
    r = s * s + r;
    s = Sum9(P(-4, 1), P(-3, 1), P(-2, 1), P(-1, 0), P(0, 0), P(1, 0), P(2, -1), P(3, -1),
             P(4, -1));
    r = s * s + r;
    s = Sum7(P(-2, -3), P(-1, -2), P(-1, -1), P(0, 0), P(1, 1), P(1, 2), P(2, 3)); r = s * s + r;
    s = Sum7(P(2, -3), P(1, -2), P(1, -1), P(0, 0), P(-1, 1), P(-1, 2), P(-2, 3)); r = s * s + r;
    s = Sum7(P(-3, -2), P(-2, -1), P(-1, -1), P(0, 0), P(1, 1), P(2, 1), P(3, 2)); r = s * s + r;
    s = Sum7(P(3, -2), P(2, -1), P(1, -1), P(0, 0), P(-1, 1), P(-2, 1), P(-3, 2)); r = s * s + r;
    s = Sum9(P(-4, 1), P(-3, 1), P(-2, 1), P(-1, 0), P(0, 0), P(1, 0), P(2, -1), P(3, -1),
             P(4, -1));
    r = s * s + r;
    s = Sum9(P(-4, -1), P(-3, -1), P(-2, -1), P(-1, 0), P(0, 0), P(1, 0), P(2, 1), P(3, 1),
             P(4, 1));
    r = s * s + r;
    s = Sum9(P(-1, -4), P(-1, -3), P(-1, -2), P(0, -1), P(0, 0), P(0, 1), P(1, 2), P(1, 3),
             P(1, 4));
    r = s * s + r;
    s = Sum9(P(1, -4), P(1, -3), P(1, -2), P(0, -1), P(0, 0), P(0, 1), P(-1, 2), P(-1, 3),
             P(-1, 4));
    r = s * s + r;
  }
#undef P
  return r;
}

// Scaled differences of the tile in shared memory, then the Malta line sums
// of four outputs per thread, added onto the accumulator.
// Polls the mbarrier at shared address `bar` until the phase of parity
// `parity` has completed, at most 2^22 times; false when it gave up.
__device__ __forceinline__ bool WaitParity(uint32_t bar, uint32_t parity) {
  uint32_t done = 0;
  for (uint32_t poll = 0; poll < (1u << 22) && !done; ++poll) {
    asm volatile(
      "{\n.reg .pred q;\nmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n"
      "selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  }
  return done != 0;
}

template <bool kLowFrequency>
__global__ void __launch_bounds__(kMaltaThreads, 3)
MaltaKernel(const __grid_constant__ MaltaParams p, const __grid_constant__ CUtensorMap map) {
  // Two staging buffers: the CTA walks its tiles (tile index t, t + grid,
  // ...) and copies the next tile's window in while it computes the current
  // one. With `p.tma`, one thread asks the tensor-memory-access unit for the
  // whole 72 x 24 window of the plane (a 2D box at the tile's origin minus
  // the 4-pixel halo; samples outside the image arrive as zeros) and the
  // CTA waits on the buffer's mbarrier (bounded). The box's x start is a
  // multiple of 4 floats (16 bytes), as the copy requires.
  __shared__ __align__(128) float tile[2][kMaltaSpanH][kMaltaSpanW];
  __shared__ __align__(8) uint64_t full[2];
  // Otherwise, four samples per copy: x0 is a multiple of 4, so with the row
  // length a multiple of 4 every aligned group of 4 lies wholly inside or
  // wholly outside the image, and with a 16-byte aligned plane it is 16-byte
  // aligned (outside groups are zero-filled by the copy); other planes take
  // synchronous scalar loads (the half-scale planes follow the full-scale
  // ones in the arena, so their alignment depends on the image size).
  constexpr int kQuads = kMaltaSpanW / 4 * kMaltaSpanH;
  constexpr int kStage = (kQuads + kMaltaThreads - 1) / kMaltaThreads;
  constexpr uint32_t kBoxBytes = kMaltaSpanW * kMaltaSpanH * sizeof(float);
  static_assert(kMaltaSpanW % 4 == 0 && kMaltaHalo % 4 == 0, "aligned quads");
  const bool aligned = p.w % 4 == 0 && reinterpret_cast<uintptr_t>(p.scaled) % 16 == 0;
  const int tiles = p.tiles_x * p.tiles_y;
  if (p.tma) {
    if (threadIdx.x == 0) {
      for (int b = 0; b < 2; ++b) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(
          static_cast<uint32_t>(__cvta_generic_to_shared(&full[b]))));
      }
      asm volatile("fence.mbarrier_init.release.cluster;");
    }
    __syncthreads();
  }
  const auto stage = [&](int t, int buffer) {
    const int x0 = (t % p.tiles_x) * kMaltaTileW - kMaltaHalo;
    const int y0 = (t / p.tiles_x) * kMaltaTileH - kMaltaHalo;
    if (p.tma) {
      if (threadIdx.x == 0) {
        const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&full[buffer]));
        // The buffer was last read through the generic proxy.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(kBoxBytes));
        asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3}], [%4];"
          ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(&tile[buffer][0][0]))),
            "l"(reinterpret_cast<uint64_t>(&map)), "r"(x0), "r"(y0), "r"(bar)
          : "memory");
      }
      return;
    }
#pragma unroll
    for (int j = 0; j < kStage; ++j) {
      const int i = threadIdx.x + j * kMaltaThreads;
      if (i >= kQuads) break;
      const int ty = i / (kMaltaSpanW / 4), tx = (i % (kMaltaSpanW / 4)) * 4;
      const int x = x0 + tx, y = y0 + ty;
      float* dst = &tile[buffer][ty][tx];
      const bool row_inside = y >= 0 && y < p.h;
      if (aligned) {
        const bool inside = row_inside && x >= 0 && x < p.w;
        const float* src = inside ? p.scaled + static_cast<size_t>(y) * p.w + x : p.scaled;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(
                       static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                     "l"(src), "r"(inside ? 16 : 0));
      } else {
        const float* row = p.scaled + static_cast<size_t>(row_inside ? y : 0) * p.w;
        float4 v;
        v.x = row_inside && x >= 0 && x < p.w ? row[x] : 0.0f;
        v.y = row_inside && x + 1 >= 0 && x + 1 < p.w ? row[x + 1] : 0.0f;
        v.z = row_inside && x + 2 >= 0 && x + 2 < p.w ? row[x + 2] : 0.0f;
        v.w = row_inside && x + 3 >= 0 && x + 3 < p.w ? row[x + 3] : 0.0f;
        *reinterpret_cast<float4*>(dst) = v;
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  int buffer = 0;
  uint32_t phases = 0;  // bit b: parity of buffer b's next completion
  if (static_cast<int>(blockIdx.x) < tiles) stage(blockIdx.x, 0);
  for (int t = blockIdx.x; t < tiles; t += gridDim.x, buffer ^= 1) {
    // This tile's copies are done, and every thread is past the previous
    // tile's reads of the other buffer.
    if (p.tma) {
      const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&full[buffer]));
      const bool done = WaitParity(bar, (phases >> buffer) & 1u);
      if (!__syncthreads_and(done)) {
        // The copy did not arrive within the bound: record it, wait once
        // more (bounded) for it before the shared memory is released, stop.
        if (threadIdx.x == 0) {
          RaiseError(p.error, kErrorInternal);
          WaitParity(bar, (phases >> buffer) & 1u);
        }
        break;
      }
      phases ^= 1u << buffer;
    } else {
      asm volatile("cp.async.wait_all;\n" ::: "memory");
      __syncthreads();
    }
    if (t + static_cast<int>(gridDim.x) < tiles) stage(t + gridDim.x, buffer ^ 1);
    const int lx = (threadIdx.x % (kMaltaTileW / kMaltaRun)) * kMaltaRun;
    const int ly = threadIdx.x / (kMaltaTileW / kMaltaRun);
    float v[2 * kMaltaHalo + 1][kMaltaWindowW];
#pragma unroll
    for (int dy = 0; dy < 2 * kMaltaHalo + 1; ++dy) {
#pragma unroll
      for (int q = 0; q < kMaltaWindowW / 4; ++q) {
        const float4 f = *reinterpret_cast<const float4*>(&tile[buffer][ly + dy][lx + 4 * q]);
        v[dy][4 * q + 0] = f.x;
        v[dy][4 * q + 1] = f.y;
        v[dy][4 * q + 2] = f.z;
        v[dy][4 * q + 3] = f.w;
      }
    }
    const float r[kMaltaRun] = {MaltaUnit<kLowFrequency, 0>(v), MaltaUnit<kLowFrequency, 1>(v),
                                MaltaUnit<kLowFrequency, 2>(v), MaltaUnit<kLowFrequency, 3>(v)};
    const int x = (t % p.tiles_x) * kMaltaTileW + lx, y = (t / p.tiles_x) * kMaltaTileH + ly;
    if (y >= p.h) continue;
    float* out = p.accumulate + static_cast<size_t>(y) * p.w + x;
#pragma unroll
    for (int k = 0; k < kMaltaRun; ++k) {
      // The reference fills the stage with 0 and adds: 0 + r == r for r >= 0
      // (or NaN), so the first stage of a channel stores r, and later ones
      // add it to the plane.
      if (x + k < p.w) out[k] = p.first ? r[k] : out[k] + (0.0f + r[k]);
    }
  }
}

// One channel's three Malta stages in one pass: the first stage (full
// Malta) stores, the other two (low-frequency Malta) add, in the order of
// the per-stage launches (stage plane order {4, 2, 0} for Y, {5, 3, 1} for
// X): acc = r0; acc = acc + (0 + r1); acc = acc + (0 + r2), all in
// registers, one store. Each tile's three 72 x 24 windows arrive by three
// tiled bulk tensor copies on one mbarrier; needs planes that take tensor
// maps (the per-stage MaltaKernel covers the others).
struct MaltaChannelParams {
  float* accumulate;
  int w, h;
  int tiles_x, tiles_y;
  uint32_t* error;
};

__global__ void __launch_bounds__(kMaltaThreads, 2)
MaltaChannelKernel(const __grid_constant__ MaltaChannelParams p,
                   const __grid_constant__ CUtensorMap first,
                   const __grid_constant__ CUtensorMap second,
                   const __grid_constant__ CUtensorMap third) {
  __shared__ __align__(128) float tile[2][3][kMaltaSpanH][kMaltaSpanW];
  __shared__ __align__(8) uint64_t full[2];
  constexpr uint32_t kBoxBytes = kMaltaSpanW * kMaltaSpanH * sizeof(float);
  static_assert(kBoxBytes % 128 == 0, "each window starts on a 128-byte boundary");
  const int tiles = p.tiles_x * p.tiles_y;
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(
        static_cast<uint32_t>(__cvta_generic_to_shared(&full[b]))));
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  __syncthreads();
  const auto stage = [&](int t, int buffer) {
    if (threadIdx.x != 0) return;
    const int x0 = (t % p.tiles_x) * kMaltaTileW - kMaltaHalo;
    const int y0 = (t / p.tiles_x) * kMaltaTileH - kMaltaHalo;
    const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&full[buffer]));
    // The buffers were last read through the generic proxy.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                 "r"(3 * kBoxBytes));
    const auto copy = [&](const CUtensorMap& map, int k) {
      asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];"
        ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(&tile[buffer][k][0][0]))),
          "l"(reinterpret_cast<uint64_t>(&map)), "r"(x0), "r"(y0), "r"(bar)
        : "memory");
    };
    copy(first, 0);
    copy(second, 1);
    copy(third, 2);
  };
  int buffer = 0;
  uint32_t phases = 0;  // bit b: parity of buffer b's next completion
  if (static_cast<int>(blockIdx.x) < tiles) stage(blockIdx.x, 0);
  for (int t = blockIdx.x; t < tiles; t += gridDim.x, buffer ^= 1) {
    const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&full[buffer]));
    const bool done = WaitParity(bar, (phases >> buffer) & 1u);
    if (!__syncthreads_and(done)) {
      // The copies did not arrive within the bound: record it, wait once
      // more (bounded) for them before the shared memory is released, stop.
      if (threadIdx.x == 0) {
        RaiseError(p.error, kErrorInternal);
        WaitParity(bar, (phases >> buffer) & 1u);
      }
      break;
    }
    phases ^= 1u << buffer;
    if (t + static_cast<int>(gridDim.x) < tiles) stage(t + gridDim.x, buffer ^ 1);
    const int lx = (threadIdx.x % (kMaltaTileW / kMaltaRun)) * kMaltaRun;
    const int ly = threadIdx.x / (kMaltaTileW / kMaltaRun);
    float acc[kMaltaRun];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float v[2 * kMaltaHalo + 1][kMaltaWindowW];
#pragma unroll
      for (int dy = 0; dy < 2 * kMaltaHalo + 1; ++dy) {
#pragma unroll
        for (int q = 0; q < kMaltaWindowW / 4; ++q) {
          const float4 f =
            *reinterpret_cast<const float4*>(&tile[buffer][k][ly + dy][lx + 4 * q]);
          v[dy][4 * q + 0] = f.x;
          v[dy][4 * q + 1] = f.y;
          v[dy][4 * q + 2] = f.z;
          v[dy][4 * q + 3] = f.w;
        }
      }
      if (k == 0) {
        acc[0] = MaltaUnit<false, 0>(v);
        acc[1] = MaltaUnit<false, 1>(v);
        acc[2] = MaltaUnit<false, 2>(v);
        acc[3] = MaltaUnit<false, 3>(v);
      } else {
        const float r[kMaltaRun] = {MaltaUnit<true, 0>(v), MaltaUnit<true, 1>(v),
                                    MaltaUnit<true, 2>(v), MaltaUnit<true, 3>(v)};
#pragma unroll
        for (int j = 0; j < kMaltaRun; ++j) acc[j] = acc[j] + (0.0f + r[j]);
      }
    }
    const int x = (t % p.tiles_x) * kMaltaTileW + lx, y = (t / p.tiles_x) * kMaltaTileH + ly;
    if (y >= p.h) continue;
    float* out = p.accumulate + static_cast<size_t>(y) * p.w + x;
#pragma unroll
    for (int j = 0; j < kMaltaRun; ++j) {
      if (x + j < p.w) out[j] = acc[j];
    }
  }
}

struct L2Params {
  const float* ref;   // psycho planes of the reference
  const float* dist;  // psycho planes of the distorted image
  size_t pitch;
  int n;
  float* ac;  // 3 planes (X and Y already hold the Malta sums; B is 0)
  float* dc;  // 3 planes
  float* pre0;  // masking precompute of the reference (may be null)
  float* pre1;  // masking precompute of the distorted image
  float asym_gt[2], asym_lt[2];  // kL2Weights[c] * asym, / asym
  float mf_weight[3], lf_weight[3];
  float mask_multiplier, mask_bias, mask_sqrt_bias;
};

// CombineChannelsForMasking of one position from its HF and UHF values.
__device__ __forceinline__ float MaskActivity(float uhf0, float hf0, float uhf1, float hf1) {
  const float xdiff = (uhf0 + hf0) * 2.5f;
  const float ydiff = uhf1 * 0.4f + hf1 * 0.4f;
  return sqrtf(xdiff * xdiff + ydiff * ydiff);
}

// L2 terms (L2DiffAsymmetric, L2Diff, SetL2Diff) and the masking inputs
// (CombineChannelsForMasking + DiffPrecompute) in the reference's order. All
// of a thread's loads are issued before its first store (the output planes
// are written through other pointers, which the compiler cannot tell apart
// from the inputs).
__global__ void __launch_bounds__(kThreads) L2MaskKernel(const __grid_constant__ L2Params p) {
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= p.n) return;
  const size_t pitch = p.pitch;
  float ac_in[2], hf_ref[2], hf_dist[2], uhf_ref[2], uhf_dist[2];
  float mf_ref[3], mf_dist[3], lf_ref[3], lf_dist[3];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    ac_in[c] = p.ac[c * pitch + i];
    hf_ref[c] = p.ref[(kHF + c) * pitch + i];
    hf_dist[c] = p.dist[(kHF + c) * pitch + i];
    uhf_dist[c] = p.dist[(kUHF + c) * pitch + i];
    uhf_ref[c] = p.pre0 != nullptr ? p.ref[(kUHF + c) * pitch + i] : 0.0f;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    mf_ref[c] = p.ref[(kMF + c) * pitch + i];
    mf_dist[c] = p.dist[(kMF + c) * pitch + i];
    lf_ref[c] = p.ref[(kLF + c) * pitch + i];
    lf_dist[c] = p.dist[(kLF + c) * pitch + i];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float acc = c < 2 ? ac_in[c] : 0.0f;
    if (c < 2) {
      const float v0 = hf_ref[c], v1 = hf_dist[c];
      const float primary = p.asym_gt[c] * 0.8f;
      const float secondary_weight = p.asym_lt[c] * 0.8f;
      const float d = v0 - v1;
      const float total = (d * d) * primary + acc;
      const float magnitude = fabsf(v0);
      const float too_small = 0.4f * magnitude;
      float secondary = 0.0f;
      if (v0 < 0.0f) {
        if (v1 > -too_small) {
          secondary = v1 + too_small;
        } else if (v1 < -magnitude) {
          secondary = -v1 - magnitude;
        }
      } else if (v1 < too_small) {
        secondary = too_small - v1;
      } else if (v1 > magnitude) {
        secondary = v1 - magnitude;
      }
      acc = secondary_weight * (secondary * secondary) + total;
    }
    {
      const float d = mf_ref[c] - mf_dist[c];
      acc = (d * d) * p.mf_weight[c] + acc;
    }
    p.ac[c * pitch + i] = acc;
    const float d = lf_ref[c] - lf_dist[c];
    p.dc[c * pitch + i] = d * d * p.lf_weight[c];
  }
  const float m1 = MaskActivity(uhf_dist[0], hf_dist[0], uhf_dist[1], hf_dist[1]);
  p.pre1[i] = sqrtf(p.mask_multiplier * fabsf(m1) + p.mask_bias) - p.mask_sqrt_bias;
  if (p.pre0 != nullptr) {
    const float m0 = MaskActivity(uhf_ref[0], hf_ref[0], uhf_ref[1], hf_ref[1]);
    p.pre0[i] = sqrtf(p.mask_multiplier * fabsf(m0) + p.mask_bias) - p.mask_sqrt_bias;
  }
}

__device__ __forceinline__ void StoreMin3(float v, float& m0, float& m1, float& m2) {
  if (v < m2) {
    if (v < m0) {
      m2 = m1; m1 = m0; m0 = v;
    } else if (v < m1) {
      m2 = m1; m1 = v;
    } else {
      m2 = v;
    }
  }
}

// FuzzyErosion of the blurred reference mask (:588-628).
__global__ void __launch_bounds__(kThreads)
FuzzyErosionKernel(const float* in, float* out, int w, int h) {
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= w * h) return;
  const int x = i % w, y = i / w;
  constexpr int kStep = 3;
  auto at = [&](int xx, int yy) { return in[static_cast<size_t>(yy) * w + xx]; };
  float m0 = at(x, y);
  float m1 = 2.0f * m0;
  float m2 = m1;
  if (x >= kStep) {
    StoreMin3(at(x - kStep, y), m0, m1, m2);
    if (y >= kStep) StoreMin3(at(x - kStep, y - kStep), m0, m1, m2);
    if (y < h - kStep) StoreMin3(at(x - kStep, y + kStep), m0, m1, m2);
  }
  if (x < w - kStep) {
    StoreMin3(at(x + kStep, y), m0, m1, m2);
    if (y >= kStep) StoreMin3(at(x + kStep, y - kStep), m0, m1, m2);
    if (y < h - kStep) StoreMin3(at(x + kStep, y + kStep), m0, m1, m2);
  }
  if (y >= kStep) StoreMin3(at(x, y - kStep), m0, m1, m2);
  if (y < h - kStep) StoreMin3(at(x, y + kStep), m0, m1, m2);
  out[i] = 0.45f * m0 + 0.3f * m1 + 0.25f * m2;
}

__device__ __forceinline__ float MaskY(float delta) {
  const double kNorm = 0.79079917404;
  const double kGlobalScale = 1.0 / (17.83 * kNorm);
  const double v = kGlobalScale * (1.0 + 2.5485944793 / (0.451936922203 * delta + 0.829591754942));
  return static_cast<float>(v * v);
}

__device__ __forceinline__ float MaskDcY(float delta) {
  const double kNorm = 0.79079917404;
  const double kGlobalScale = 1.0 / (17.83 * kNorm);
  const double v = kGlobalScale * (1.0 + 0.505054525019 / (3.87449418804 * delta + 0.20025578522));
  return static_cast<float>(v * v);
}

// Masked Y AC term and the final composition (:805-851).
__global__ void __launch_bounds__(kThreads)
FinalCompositionKernel(const float* mask, const float* blurred0, const float* blurred1,
                       const float* ac, const float* dc, size_t pitch, int n, float x_multiplier,
                       float* final_map, uint32_t* error) {
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const float difference = blurred0[i] - blurred1[i];
  const float ac_y = ac[pitch + i] + 10.0f * difference * difference;
  const float m = mask[i];
  const float mask_value = MaskY(m);
  const float dc_mask_value = MaskDcY(m);
  const float diff_dc0 = dc[i] * x_multiplier;
  const float diff_ac0 = ac[i] * x_multiplier;
  const float masked_dc =
    diff_dc0 * dc_mask_value + dc[pitch + i] * dc_mask_value + dc[2 * pitch + i] * dc_mask_value;
  const float masked_ac = diff_ac0 * mask_value + ac_y * mask_value + ac[2 * pitch + i] * mask_value;
  const float v = sqrtf(masked_dc + masked_ac);
  if (!IsFinite(v)) RaiseError(error, kErrorNonFiniteOutput);
  final_map[i] = v;
}

// Subsample2x (:338-360) of three planes.
__global__ void __launch_bounds__(kThreads)
Subsample2xKernel(const float* in, size_t in_stride, size_t in_pitch, int w, int h, float* out,
                  int sw, int sh, size_t out_pitch) {
  const int plane = blockIdx.y;
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= sw * sh) return;
  const int x = i % sw, y = i / sw;
  const float* src = in + plane * in_pitch;
  float v = 0.0f;
  for (int dy = 0; dy < 2; ++dy) {
    const int yy = 2 * y + dy;
    if (yy >= h) continue;
    for (int dx = 0; dx < 2; ++dx) {
      const int xx = 2 * x + dx;
      if (xx >= w) continue;
      v += 0.25f * src[static_cast<size_t>(yy) * in_stride + xx];
    }
  }
  if ((w & 1) && x == sw - 1) v *= 2.0f;
  if ((h & 1) && y == sh - 1) v *= 2.0f;
  out[plane * out_pitch + i] = v;
}

// ExpandImage (:322-336) for images narrower or shorter than 8 pixels.
__global__ void __launch_bounds__(kThreads)
ExpandKernel(const float* in, size_t in_stride, size_t in_pitch, int w, int h, float* out,
             int ew, int eh, int xborder, int yborder, size_t out_pitch) {
  const int plane = blockIdx.y;
  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= ew * eh) return;
  const int x = i % ew, y = i / ew;
  const int sy = min(h - 1, y > yborder ? y - yborder : 0);
  const int sx = min(w - 1, x > xborder ? x - xborder : 0);
  out[plane * out_pitch + i] = in[plane * in_pitch + static_cast<size_t>(sy) * in_stride + sx];
}

// Main/sub combination (:956-963) or the cropped copy of an expanded map.
// Grid-stride over the pixels; the NaN-free maximum is reduced per CTA
// (warp shuffles, then shared memory) and published with one float atomicMax
// per CTA (a max is order-independent).
__global__ void __launch_bounds__(kThreads)
CombineKernel(const float* main_map, int main_w, const float* sub_map, int sub_w, int w, int h,
              int xborder, int yborder, float* out, size_t out_stride, float* maximum,
              uint32_t* error) {
  __shared__ float warp_max[kThreads / 32];
  float best = 0.0f;
  const size_t n = static_cast<size_t>(w) * h;
  for (size_t i = blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * kThreads) {
    const int x = static_cast<int>(i % w), y = static_cast<int>(i / w);
    const float m = main_map[static_cast<size_t>(y + yborder) * main_w + x + xborder];
    const float v =
      sub_map != nullptr ? m * 0.85f + 0.5f * sub_map[static_cast<size_t>(y / 2) * sub_w + x / 2]
                         : m;
    if (!(IsFinite(v) && v >= 0.0f)) RaiseError(error, kErrorNonFiniteOutput);
    out[static_cast<size_t>(y) * out_stride + x] = v;
    best = fmaxf(best, v);
  }
  best = WarpMax(best);
  if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x / 32] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kThreads / 32; ++k) best = fmaxf(best, warp_max[k]);
    AtomicMaxNonNegative(maximum, best);
  }
}

__global__ void ScoreKernel(const float* maximum, double* score) {
  *score = static_cast<double>(*maximum);
}

// --------------------------------------------------------------------------
// Host side.

Kernel17 MakeKernel(float sigma) {
  Kernel17 k;
  std::memset(&k, 0, sizeof(k));
  const float scaled_radius = 2.25f * std::abs(sigma);
  const int radius = std::max(1, static_cast<int>(scaled_radius));
  const double exponent_scale = -1.0 / (2.0 * sigma * sigma);
  for (int index = -radius; index <= radius; ++index) {
    k.raw[index + radius] = static_cast<float>(std::exp(exponent_scale * index * index));
  }
  float full = 0.0f;
  for (int i = 0; i < 2 * radius + 1; ++i) full += k.raw[i];
  const float scale = 1.0f / full;
  for (int i = 0; i <= radius && i < 17; ++i) k.scaled[i] = k.raw[i] * scale;
  if (radius == 2) {
    k.w5[0] = k.raw[2] * scale;
    k.w5[1] = k.raw[1] * scale;
    k.w5[2] = k.raw[0] * scale;
  }
  return k;
}

unsigned Blocks(size_t n) { return static_cast<unsigned>((n + kThreads - 1) / kThreads); }

// Butteraugli sigmas (butteraugli_internal.h).
constexpr float kOpsinSigma = 1.2f, kLowSigma = 7.15593339443f, kHighSigma = 3.22489901262f,
                kUltraSigma = 1.56416327805f, kMaskSigma = 2.7f;

struct Scale {
  int w = 0, h = 0;
  size_t n = 0;
  float* ref_psycho = nullptr;   // 10 planes
  float* dist_psycho = nullptr;  // 10 planes
  float* ref_mask = nullptr;     // FuzzyErosion(blur13(pre0))
  float* ref_blurred = nullptr;  // blur13(pre0)
  float* linear_tmp = nullptr;   // 3 planes: expanded/subsampled input
  float* blur3 = nullptr;        // 3 planes
  float* xyb = nullptr;          // 3 planes
  float* tmp = nullptr;          // 3 planes (row-pass outputs)
  float* ac = nullptr;           // 3 planes
  float* dc = nullptr;           // 3 planes
  float* pre0 = nullptr;
  float* pre1 = nullptr;
  float* blurred1 = nullptr;
  float* final_map = nullptr;
  float* malta = nullptr;        // 6 planes: Malta stage inputs (MaltaPlanes)
  // Tiled bulk-copy descriptors of the six Malta input planes (72 x 24
  // boxes), when the planes allow them (EncodeMaltaMaps).
  bool malta_tma = false;
  CUtensorMap malta_map[6];
};

size_t ScaleFloats(size_t n) {
  return n * (10 + 10 + 1 + 1 + 3 + 3 + 3 + 3 + 3 + 3 + 1 + 1 + 1 + 1 + 6);
}

void AssignScale(Scale& s, float* base) {
  float* p = base;
  auto take = [&](size_t planes) {
    float* r = p;
    p += planes * s.n;
    return r;
  };
  s.ref_psycho = take(10);
  s.dist_psycho = take(10);
  s.ref_mask = take(1);
  s.ref_blurred = take(1);
  s.linear_tmp = take(3);
  s.blur3 = take(3);
  s.xyb = take(3);
  s.tmp = take(3);
  s.ac = take(3);
  s.dc = take(3);
  s.pre0 = take(1);
  s.pre1 = take(1);
  s.blurred1 = take(1);
  s.final_map = take(1);
  s.malta = take(6);
}

}  // namespace

struct ButteraugliState {
  int width = 0, height = 0;
  float intensity_target = 80.0f;
  float hf_asymmetry = 1.0f, x_multiplier = 1.0f;
  bool expanded = false, has_sub = false;
  int xborder = 0, yborder = 0;
  Scale main, sub;
  float* arena = nullptr;
  float* maximum = nullptr;
  uint32_t* error = nullptr;
  bool prepared = false;
  bool reference_mask_ready = false;  // reference mask planes computed
  int sm_count = 0;                   // SMs of the device the state lives on
  Kernel17 k_opsin, k_low, k_high, k_ultra, k_mask;

  bool external_arena = false;  // planes lent by the owner (not freed)

  // The half-resolution scale runs on its own stream beside the full one
  // (fork / join events; inside a captured graph they become branches).
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;

  ~ButteraugliState() {
    if (arena && !external_arena) cudaFree(arena);
    if (side) cudaStreamDestroy(side);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
  }
};

namespace {

template <int R>
void BlurPlanes(const float* in, float* tmp, float* out, int w, int h, size_t pitch, int planes,
                const Kernel17& k, cudaStream_t stream) {
  const size_t column_runs = static_cast<size_t>(w) * ((h + kRun - 1) / kRun);
  const int row_groups = std::min((h + kBlurRows - 1) / kBlurRows, 65535);
  BlurRowsKernel<R><<<dim3((w + kRowSegment - 1) / kRowSegment, row_groups, planes), kThreads, 0,
                      stream>>>(in, tmp, w, h, pitch, pitch, k);
  constexpr int kBorderRows = kThreads / (2 * R);
  BlurRowBordersKernel<R><<<dim3((h + kBorderRows - 1) / kBorderRows, planes), kThreads, 0,
                            stream>>>(in, tmp, w, h, pitch, pitch, k);
  BlurColumnsKernel<R><<<dim3(Blocks(column_runs), planes), kThreads, 0, stream>>>(
    tmp, out, w, h, pitch, pitch, k);
}

// Constants of the six Malta stages (MaltaDiffMap calls of
// butteraugli_distance_internal.cpp:659-674): MF_Y, MF_X, HF_Y, HF_X, UHF_Y,
// UHF_X, with kMaltaWeights / kMaltaNorms (:24-31).
void MaltaStageScales(float hf_asymmetry, MaltaScale out[6]) {
  const float asym = hf_asymmetry;
  const float sqrt_asym = std::sqrt(asym);
  const double kMaltaWeights[6] = {37.0819870399, 8246.75321353, 18.7237414387,
                                   6923.99476109, 1.10039032555, 173.5};
  const double kMaltaNorms[6] = {130262059.556, 1009002.70582, 4498534.45232,
                                 8051.15833247, 71.7800275169, 5.0};
  const double up[6] = {kMaltaWeights[0], kMaltaWeights[1], kMaltaWeights[2] * sqrt_asym,
                        kMaltaWeights[3] * sqrt_asym, kMaltaWeights[4] * asym,
                        kMaltaWeights[5] * asym};
  const double down[6] = {kMaltaWeights[0], kMaltaWeights[1], kMaltaWeights[2] / sqrt_asym,
                          kMaltaWeights[3] / sqrt_asym, kMaltaWeights[4] / asym,
                          kMaltaWeights[5] / asym};
  for (int index = 0; index < 6; ++index) {
    const bool lf = index < 4;
    const double multiplier = lf ? 0.611612573796 : 0.39905817637;
    const double kLength = 3.75;
    const double pre_gt = multiplier * std::sqrt(0.5f * up[index]) / (kLength * 2.0 + 1.0);
    const double pre_lt = multiplier * std::sqrt(0.33f * down[index]) / (kLength * 2.0 + 1.0);
    out[index].norm2_gt = static_cast<float>(pre_gt * kMaltaNorms[index]);
    out[index].norm2_lt = static_cast<float>(pre_lt * kMaltaNorms[index]);
    out[index].norm = static_cast<float>(kMaltaNorms[index]);
  }
}

// Opsin dynamics + frequency separation of one image at one scale
// (OpsinDynamicsImage + SeparateFrequencies) into `psycho`.
// For the distorted image (`ref_psycho` set: the reference's final planes)
// the frequency kernels also write the Malta stage inputs into s.malta.
void Psycho(ButteraugliState& st, Scale& s, const float* linear, size_t stride, size_t pitch,
            float* psycho, const float* ref_psycho, cudaStream_t stream) {
  MaltaPlanes mp;
  mp.ref = ref_psycho;
  mp.malta = s.malta;
  MaltaStageScales(st.hf_asymmetry, mp.scale);
  const size_t n = s.n;
  // Dense copy of the input planes for the mirrored 5-tap blur.
  const float* dense = linear;
  if (stride != static_cast<size_t>(s.w) || pitch != n) {
    cudaMemcpy2DAsync(s.linear_tmp, s.w * sizeof(float), linear, stride * sizeof(float),
                      s.w * sizeof(float), s.h, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpy2DAsync(s.linear_tmp + n, s.w * sizeof(float), linear + pitch,
                      stride * sizeof(float), s.w * sizeof(float), s.h,
                      cudaMemcpyDeviceToDevice, stream);
    cudaMemcpy2DAsync(s.linear_tmp + 2 * n, s.w * sizeof(float), linear + 2 * pitch,
                      stride * sizeof(float), s.w * sizeof(float), s.h,
                      cudaMemcpyDeviceToDevice, stream);
    dense = s.linear_tmp;
  }
  // Opsin blur and dynamics in one pass (the blurred planes stay on chip).
  Blur5DynamicsKernel<<<dim3((s.w + kB5W - 1) / kB5W, (s.h + kB5H - 1) / kB5H),
                        dim3(kB5W, kB5Rows), 0, stream>>>(dense, s.xyb, s.w, s.h, n,
                                                          st.k_opsin, st.intensity_target,
                                                          st.error);
  // LF: 33-tap blur of the three XYB planes straight into the LF planes.
  BlurPlanes<16>(s.xyb, s.tmp, psycho + kLF * n, s.w, s.h, n, 3, st.k_low, stream);
  FrequencyLowKernel<<<Blocks(n), kThreads, 0, stream>>>(s.xyb, psycho, static_cast<int>(n), n,
                                                         st.error);
  // 15-tap blur of MF (3 planes) into blur3.
  BlurPlanes<7>(psycho + kMF * n, s.tmp, s.blur3, s.w, s.h, n, 3, st.k_high, stream);
  FrequencyHighKernel<<<Blocks(n), kThreads, 0, stream>>>(s.blur3, psycho, static_cast<int>(n), n,
                                                          st.error, mp);
  // 7-tap blur of HF (2 planes) into blur3.
  BlurPlanes<3>(psycho + kHF * n, s.tmp, s.blur3, s.w, s.h, n, 2, st.k_ultra, stream);
  FrequencyUltraKernel<<<Blocks(n), kThreads, 0, stream>>>(s.blur3, psycho, static_cast<int>(n),
                                                           n, st.error, mp);
}

// Difference stages of one scale into s.final_map; with `reference_side`
// the reference's mask planes are computed (prepare), otherwise reused.
void Differences(ButteraugliState& st, Scale& s, bool reference_side, cudaStream_t stream) {
  const size_t n = s.n;
  const float asym = st.hf_asymmetry;
  // Stage inputs (computed beside the distorted image's final planes):
  // MF_Y, MF_X, HF_Y, HF_X, UHF_Y, UHF_X.
  // The first stage of each channel (4, 5) writes its plane; the B plane is
  // written by the L2 terms.
  const int order[6] = {4, 5, 2, 3, 0, 1};
  const int tiles_x = (s.w + kMaltaTileW - 1) / kMaltaTileW;
  const int tiles_y = (s.h + kMaltaTileH - 1) / kMaltaTileH;
  // Three CTAs per SM walk the tiles.
  const unsigned malta_grid = static_cast<unsigned>(
    st.sm_count > 0 ? std::min(tiles_x * tiles_y, st.sm_count * 3) : tiles_x * tiles_y);
  if (s.malta_tma) {
    // Channel 1 (Y) from stage planes 4, 2, 0 and channel 0 (X) from 5, 3, 1.
    for (int channel = 1; channel >= 0; --channel) {
      MaltaChannelParams cp;
      cp.accumulate = s.ac + channel * n;
      cp.w = s.w;
      cp.h = s.h;
      cp.tiles_x = tiles_x;
      cp.tiles_y = tiles_y;
      cp.error = st.error;
      const int base = channel == 1 ? 0 : 1;
      // Two CTAs per SM (103 registers per thread).
      const unsigned channel_grid = static_cast<unsigned>(
        st.sm_count > 0 ? std::min(tiles_x * tiles_y, st.sm_count * 2) : tiles_x * tiles_y);
      MaltaChannelKernel<<<channel_grid, kMaltaThreads, 0, stream>>>(
        cp, s.malta_map[base + 4], s.malta_map[base + 2], s.malta_map[base]);
    }
  }
  for (int index : order) {
    if (s.malta_tma) break;
    MaltaParams mp;
    mp.scaled = s.malta + index * n;
    const int channel = index % 2 == 0 ? 1 : 0;
    mp.accumulate = s.ac + channel * n;
    mp.w = s.w;
    mp.h = s.h;
    mp.tiles_x = tiles_x;
    mp.tiles_y = tiles_y;
    mp.first = index >= 4 ? 1 : 0;
    mp.tma = s.malta_tma ? 1 : 0;
    mp.error = st.error;
    if (index < 4) {
      MaltaKernel<true><<<malta_grid, kMaltaThreads, 0, stream>>>(mp, s.malta_map[index]);
    } else {
      MaltaKernel<false><<<malta_grid, kMaltaThreads, 0, stream>>>(mp, s.malta_map[index]);
    }
  }
  // kL2Weights (:32-36).
  const float kL2[9] = {400.0f, 1.50815703118f, 0.0f, 2150.0f, 10.6195433239f, 16.2176043152f,
                        29.2353797994f, 0.844626970982f, 0.703646627719f};
  L2Params lp;
  lp.ref = s.ref_psycho;
  lp.dist = s.dist_psycho;
  lp.pitch = n;
  lp.n = static_cast<int>(n);
  lp.ac = s.ac;
  lp.dc = s.dc;
  lp.pre0 = reference_side ? s.pre0 : nullptr;
  lp.pre1 = s.pre1;
  for (int c = 0; c < 2; ++c) {
    lp.asym_gt[c] = kL2[c] * asym;
    lp.asym_lt[c] = kL2[c] / asym;
  }
  for (int c = 0; c < 3; ++c) {
    lp.mf_weight[c] = kL2[3 + c];
    lp.lf_weight[c] = kL2[6 + c];
  }
  lp.mask_multiplier = 6.19424080439f;
  lp.mask_bias = 6.19424080439f * 12.61050594197f;
  lp.mask_sqrt_bias = std::sqrt(lp.mask_bias);
  L2MaskKernel<<<Blocks(n), kThreads, 0, stream>>>(lp);
  if (reference_side) {
    BlurPlanes<6>(s.pre0, s.tmp, s.ref_blurred, s.w, s.h, n, 1, st.k_mask, stream);
    FuzzyErosionKernel<<<Blocks(n), kThreads, 0, stream>>>(s.ref_blurred, s.ref_mask, s.w, s.h);
  }
  BlurPlanes<6>(s.pre1, s.tmp, s.blurred1, s.w, s.h, n, 1, st.k_mask, stream);
  FinalCompositionKernel<<<Blocks(n), kThreads, 0, stream>>>(
    s.ref_mask, s.ref_blurred, s.blurred1, s.ac, s.dc, n, static_cast<int>(n), st.x_multiplier,
    s.final_map, st.error);
}

void TransformMain(ButteraugliState& st, const float* linear, size_t stride, size_t pitch,
                   bool reference, cudaStream_t stream) {
  const float* main_in = linear;
  size_t main_stride = stride, main_pitch = pitch;
  if (st.expanded) {
    ExpandKernel<<<dim3(Blocks(st.main.n), 3), kThreads, 0, stream>>>(
      linear, stride, pitch, st.width, st.height, st.main.linear_tmp, st.main.w, st.main.h,
      st.xborder, st.yborder, st.main.n);
    main_in = st.main.linear_tmp;
    main_stride = st.main.w;
    main_pitch = st.main.n;
  }
  Psycho(st, st.main, main_in, main_stride, main_pitch,
         reference ? st.main.ref_psycho : st.main.dist_psycho,
         reference ? nullptr : st.main.ref_psycho, stream);
}

void TransformSub(ButteraugliState& st, const float* linear, size_t stride, size_t pitch,
                  bool reference, cudaStream_t stream) {
  Subsample2xKernel<<<dim3(Blocks(st.sub.n), 3), kThreads, 0, stream>>>(
    linear, stride, pitch, st.width, st.height, st.sub.linear_tmp, st.sub.w, st.sub.h,
    st.sub.n);
  Psycho(st, st.sub, st.sub.linear_tmp, st.sub.w, st.sub.n,
         reference ? st.sub.ref_psycho : st.sub.dist_psycho,
         reference ? nullptr : st.sub.ref_psycho, stream);
}

// The side stream starts after everything queued on `stream` so far.
void Fork(ButteraugliState& st, cudaStream_t stream) {
  cudaEventRecord(st.fork, stream);
  cudaStreamWaitEvent(st.side, st.fork, 0);
}
void Join(ButteraugliState& st, cudaStream_t stream) {
  cudaEventRecord(st.join, st.side);
  cudaStreamWaitEvent(stream, st.join, 0);
}

}  // namespace

namespace {

struct ScaleExtents {
  size_t main_n = 0, sub_n = 0;
};

ScaleExtents Extents(size_t width, size_t height) {
  ScaleExtents e;
  const bool expanded = width < 8 || height < 8;
  e.main_n = std::max<size_t>(8, width) * std::max<size_t>(8, height);
  if (!expanded && width >= 15 && height >= 15) e.sub_n = ((width + 1) / 2) * ((height + 1) / 2);
  return e;
}

using TensorMapEncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                             const cuuint64_t*, const cuuint64_t*,
                                             const cuuint32_t*, const cuuint32_t*,
                                             CUtensorMapInterleave, CUtensorMapSwizzle,
                                             CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tiled tensor-map encoder, looked up once through the runtime
// (no link against the driver library); null when the driver lacks it.
TensorMapEncodeTiledFn TensorMapEncoder() {
  static TensorMapEncodeTiledFn encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult found;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &found) ==
          cudaSuccess &&
        found == cudaDriverEntryPointSuccess) {
      encode = reinterpret_cast<TensorMapEncodeTiledFn>(fn);
    }
    cudaGetLastError();
  });
  return encode;
}

// Describes each Malta input plane of `s` as a 2D FP32 tensor (w x h, rows
// w floats apart) read in 72 x 24 boxes with zero fill outside it. The
// copies need a 16-byte aligned plane and a row pitch of a multiple of 16
// bytes; other scales keep the per-thread staging.
void EncodeMaltaMaps(Scale& s) {
  s.malta_tma = false;
  std::memset(s.malta_map, 0, sizeof(s.malta_map));
  const TensorMapEncodeTiledFn encode = TensorMapEncoder();
  if (encode == nullptr || s.malta == nullptr || s.w % 4 != 0 ||
      reinterpret_cast<uintptr_t>(s.malta) % 16 != 0 || (s.n * sizeof(float)) % 16 != 0) {
    return;
  }
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(s.w), static_cast<cuuint64_t>(s.h)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(s.w) * sizeof(float)};
  const cuuint32_t box[2] = {kMaltaSpanW, kMaltaSpanH};
  const cuuint32_t unit[2] = {1, 1};
  for (int i = 0; i < 6; ++i) {
    if (encode(&s.malta_map[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, s.malta + i * s.n, dims,
               strides, box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      std::memset(s.malta_map, 0, sizeof(s.malta_map));
      return;
    }
  }
  s.malta_tma = true;
}

}  // namespace

size_t ButteraugliArenaBytes(size_t width, size_t height) {
  const ScaleExtents e = Extents(width, height);
  return (ScaleFloats(e.main_n) + ScaleFloats(e.sub_n) + 64) * sizeof(float);
}

int ButteraugliCreate(size_t width, size_t height, float intensity_target, void* external,
                      ButteraugliState** out) {
  auto* st = new (std::nothrow) ButteraugliState();
  if (st == nullptr) return SetError(GJXL_B200_OUT_OF_MEMORY, "butteraugli: host allocation");
  st->width = static_cast<int>(width);
  st->height = static_cast<int>(height);
  st->intensity_target = intensity_target;
  st->expanded = width < 8 || height < 8;
  st->main.w = static_cast<int>(std::max<size_t>(8, width));
  st->main.h = static_cast<int>(std::max<size_t>(8, height));
  if (st->expanded) {
    st->xborder = width < 8 ? static_cast<int>((8 - width) / 2) : 0;
    st->yborder = height < 8 ? static_cast<int>((8 - height) / 2) : 0;
  }
  st->main.n = static_cast<size_t>(st->main.w) * st->main.h;
  st->has_sub = !st->expanded && width >= 15 && height >= 15;
  if (st->has_sub) {
    st->sub.w = static_cast<int>((width + 1) / 2);
    st->sub.h = static_cast<int>((height + 1) / 2);
    st->sub.n = static_cast<size_t>(st->sub.w) * st->sub.h;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess ||
      cudaDeviceGetAttribute(&st->sm_count, cudaDevAttrMultiProcessorCount, device) !=
        cudaSuccess) {
    st->sm_count = 0;  // the Malta grid then takes one CTA per tile
  }
  const size_t floats = ScaleFloats(st->main.n) + ScaleFloats(st->sub.n) + 64;
  if (external != nullptr) {
    st->arena = static_cast<float*>(external);
    st->external_arena = true;
  } else {
    const int status = CheckCuda(DeviceMalloc(reinterpret_cast<void**>(&st->arena),
                                              floats * sizeof(float)),
                                 "butteraugli: cudaMalloc");
    if (status != GJXL_B200_OK) {
      delete st;
      return status;
    }
  }
  AssignScale(st->main, st->arena);
  if (st->has_sub) AssignScale(st->sub, st->arena + ScaleFloats(st->main.n));
  st->maximum = st->arena + ScaleFloats(st->main.n) + ScaleFloats(st->sub.n);
  st->error = reinterpret_cast<uint32_t*>(st->maximum + 32);
  EncodeMaltaMaps(st->main);
  if (st->has_sub) EncodeMaltaMaps(st->sub);
  if (CheckCuda(cudaStreamCreateWithFlags(&st->side, cudaStreamNonBlocking),
                "butteraugli: side stream") != GJXL_B200_OK ||
      CheckCuda(cudaEventCreateWithFlags(&st->fork, cudaEventDisableTiming),
                "butteraugli: event") != GJXL_B200_OK ||
      CheckCuda(cudaEventCreateWithFlags(&st->join, cudaEventDisableTiming),
                "butteraugli: event") != GJXL_B200_OK) {
    delete st;
    return GJXL_B200_OUT_OF_MEMORY;
  }
  st->k_opsin = MakeKernel(kOpsinSigma);
  st->k_low = MakeKernel(kLowSigma);
  st->k_high = MakeKernel(kHighSigma);
  st->k_ultra = MakeKernel(kUltraSigma);
  st->k_mask = MakeKernel(kMaskSigma);
  *out = st;
  return GJXL_B200_OK;
}

int ButteraugliPrepare(ButteraugliState* st, const float* linear, size_t stride, size_t pitch,
                       cudaStream_t stream) {
  cudaMemsetAsync(st->error, 0, sizeof(uint32_t), stream);
  if (st->has_sub) {
    Fork(*st, stream);
    TransformSub(*st, linear, stride, pitch, true, st->side);
  }
  TransformMain(*st, linear, stride, pitch, true, stream);
  if (st->has_sub) Join(*st, stream);
  st->prepared = true;
  st->reference_mask_ready = false;
  return CheckLaunch("butteraugli prepare");
}

int ButteraugliCompare(ButteraugliState* st, const float* linear, size_t stride, size_t pitch,
                       float* map, size_t map_stride, double* score, cudaStream_t stream) {
  if (!st->prepared) {
    return SetError(GJXL_B200_FAILED_PRECONDITION, "butteraugli: reference not prepared");
  }
  // The reference's mask planes depend only on the reference image; the
  // first comparison after a prepare computes them, later ones reuse them.
  const bool reference_side = !st->reference_mask_ready;
  if (st->has_sub) {
    Fork(*st, stream);
    TransformSub(*st, linear, stride, pitch, false, st->side);
    Differences(*st, st->sub, reference_side, st->side);
  }
  TransformMain(*st, linear, stride, pitch, false, stream);
  Differences(*st, st->main, reference_side, stream);
  if (st->has_sub) Join(*st, stream);
  st->reference_mask_ready = true;
  cudaMemsetAsync(st->maximum, 0, sizeof(float), stream);
  const size_t n = static_cast<size_t>(st->width) * st->height;
  CombineKernel<<<std::min<unsigned>(Blocks(n), 148 * 8), kThreads, 0, stream>>>(
    st->main.final_map, st->main.w, st->has_sub ? st->sub.final_map : nullptr, st->sub.w,
    st->width, st->height, st->xborder, st->yborder, map, map_stride, st->maximum, st->error);
  if (score != nullptr) ScoreKernel<<<1, 1, 0, stream>>>(st->maximum, score);
  return CheckLaunch("butteraugli compare");
}

uint32_t* ButteraugliErrorWord(ButteraugliState* st) { return st->error; }
void ButteraugliDestroy(ButteraugliState* st) { delete st; }
float* ButteraugliMaximum(ButteraugliState* st) { return st->maximum; }

}  // namespace gjxl_b200

using namespace gjxl_b200;

struct gjxl_b200_butteraugli : public ButteraugliState {};

extern "C" int gjxl_b200_butteraugli_create(size_t width, size_t height, float intensity_target,
                                            gjxl_b200_butteraugli** out) {
  ClearLastError();
  if (out == nullptr || width == 0 || height == 0 || width > (1u << 20) || height > (1u << 20) ||
      !std::isfinite(intensity_target) || intensity_target <= 0.0f) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "butteraugli_create: invalid arguments");
  }
  ButteraugliState* st = nullptr;
  const int status = ButteraugliCreate(width, height, intensity_target, nullptr, &st);
  if (status != GJXL_B200_OK) return status;
  // The public handle type derives from the state without adding members.
  static_assert(sizeof(gjxl_b200_butteraugli) == sizeof(ButteraugliState), "");
  *out = static_cast<gjxl_b200_butteraugli*>(st);
  return GJXL_B200_OK;
}

extern "C" void gjxl_b200_butteraugli_destroy(gjxl_b200_butteraugli* b) {
  delete static_cast<ButteraugliState*>(b);
}

extern "C" int gjxl_b200_butteraugli_prepare(gjxl_b200_butteraugli* b, const float* reference,
                                             size_t stride, size_t plane_pitch, void* stream) {
  ClearLastError();
  if (b == nullptr || reference == nullptr || stride < static_cast<size_t>(b->width) ||
      plane_pitch < stride * b->height) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "butteraugli_prepare: invalid arguments");
  }
  return ButteraugliPrepare(b, reference, stride, plane_pitch, static_cast<cudaStream_t>(stream));
}

extern "C" int gjxl_b200_butteraugli_compare(gjxl_b200_butteraugli* b, const float* distorted,
                                             size_t stride, size_t plane_pitch,
                                             float* distance_map, size_t map_stride,
                                             double* score, uint32_t* device_error, void* stream) {
  ClearLastError();
  if (b == nullptr || distorted == nullptr || distance_map == nullptr ||
      stride < static_cast<size_t>(b->width) || plane_pitch < stride * b->height ||
      map_stride < static_cast<size_t>(b->width)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "butteraugli_compare: invalid arguments");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int status = ButteraugliCompare(b, distorted, stride, plane_pitch, distance_map,
                                        map_stride, score, s);
  if (status == GJXL_B200_OK && device_error != nullptr) {
    cudaMemcpyAsync(device_error, b->error, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
  }
  return status == GJXL_B200_OK ? CheckLaunch("butteraugli compare") : status;
}
