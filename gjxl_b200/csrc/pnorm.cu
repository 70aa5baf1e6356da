// Global Butteraugli p-norm of a distance map, accumulated in FP64.
//
// The reference summarises a distance map by its maximum only
// (src/gpu/cuda/cuda_butteraugli_kernels.cu:4063-4065,
// src/codec/butteraugli.cpp:60); it has no p-norm. This is libjxl's published
// summary (ComputeDistanceP of its Butteraugli p-norm comparator): the mean
// of the p-, 2p- and 4p-norms of the map,
//   ((S_p / n)^(1/p) + (S_2p / n)^(1/(2p)) + (S_4p / n)^(1/(4p))) / 3,
//   S_q = sum over the n pixels of d^q,
// with every power and sum in double precision (each pixel's d^p in double,
// squared for 2p and again for 4p).
//
// Two launches with a fixed geometry, so the result is reproducible to the
// bit: kPartials CTAs each sum a grid-strided share of the pixels (one
// double per thread, then a fixed shared-memory tree), and one CTA reduces
// the partials in a fixed tree and applies the roots.

#include <cmath>

#include "host_util.h"
#include "session.h"

namespace gjxl_b200 {
namespace {

constexpr int kPnormThreads = 256;
constexpr int kPartials = 592;  // 4 CTAs per SM of a B200

// Fixed-order tree over the CTA's threads for the three sums.
__device__ __forceinline__ void TreeSum3(double (*sums)[kPnormThreads], double a, double b,
                                         double c) {
  const int t = threadIdx.x;
  sums[0][t] = a;
  sums[1][t] = b;
  sums[2][t] = c;
  __syncthreads();
  for (int half = kPnormThreads / 2; half >= 1; half >>= 1) {
    if (t < half) {
      sums[0][t] += sums[0][t + half];
      sums[1][t] += sums[1][t + half];
      sums[2][t] += sums[2][t + half];
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double PowerP(double d, double p) {
  // d^3 by multiplications for the usual p = 3 (libjxl's default), else pow.
  return p == 3.0 ? d * d * d : pow(d, p);
}

__global__ void __launch_bounds__(kPnormThreads)
PnormPartialKernel(const float* map, size_t stride, uint32_t width, uint32_t height, double p,
                   double* partials) {
  __shared__ double sums[3][kPnormThreads];
  double s1 = 0.0, s2 = 0.0, s4 = 0.0;
  const size_t n = static_cast<size_t>(width) * height;
  for (size_t i = static_cast<size_t>(blockIdx.x) * kPnormThreads + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * kPnormThreads) {
    const size_t y = i / width, x = i % width;
    const double d = static_cast<double>(map[y * stride + x]);
    const double dp = PowerP(d, p);
    const double d2p = dp * dp;
    s1 += dp;
    s2 += d2p;
    s4 += d2p * d2p;
  }
  TreeSum3(sums, s1, s2, s4);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x + 0] = sums[0][0];
    partials[3 * blockIdx.x + 1] = sums[1][0];
    partials[3 * blockIdx.x + 2] = sums[2][0];
  }
}

__global__ void __launch_bounds__(kPnormThreads)
PnormFinalKernel(const double* partials, int count, uint32_t width, uint32_t height, double p,
                 double* out) {
  __shared__ double sums[3][kPnormThreads];
  double s1 = 0.0, s2 = 0.0, s4 = 0.0;
  for (int i = threadIdx.x; i < count; i += kPnormThreads) {
    s1 += partials[3 * i + 0];
    s2 += partials[3 * i + 1];
    s4 += partials[3 * i + 2];
  }
  TreeSum3(sums, s1, s2, s4);
  if (threadIdx.x == 0) {
    const double per_pixel = 1.0 / (static_cast<double>(width) * static_cast<double>(height));
    const double v = pow(sums[0][0] * per_pixel, 1.0 / p) +
                     pow(sums[1][0] * per_pixel, 1.0 / (2.0 * p)) +
                     pow(sums[2][0] * per_pixel, 1.0 / (4.0 * p));
    *out = v / 3.0;
  }
}

}  // namespace

size_t PnormScratchBytes() { return static_cast<size_t>(kPartials) * 3 * sizeof(double); }

int LaunchPnorm(const float* map, size_t stride, size_t width, size_t height, double p,
                double* scratch, double* out, cudaStream_t stream) {
  PnormPartialKernel<<<kPartials, kPnormThreads, 0, stream>>>(
    map, stride, static_cast<uint32_t>(width), static_cast<uint32_t>(height), p, scratch);
  PnormFinalKernel<<<1, kPnormThreads, 0, stream>>>(scratch, kPartials,
                                                   static_cast<uint32_t>(width),
                                                   static_cast<uint32_t>(height), p, out);
  return CheckLaunch("butteraugli p-norm");
}

}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" size_t gjxl_b200_butteraugli_pnorm_scratch_bytes(void) { return PnormScratchBytes(); }

extern "C" int gjxl_b200_butteraugli_pnorm(const float* distance_map, size_t map_stride,
                                           size_t width, size_t height, double p,
                                           double* scratch, size_t scratch_bytes,
                                           double* pnorm, void* stream) {
  ClearLastError();
  if (distance_map == nullptr || scratch == nullptr || pnorm == nullptr || width == 0 ||
      height == 0 || map_stride < width || width > (1u << 20) || height > (1u << 20) ||
      !(p >= 1.0 && p <= 64.0) || scratch_bytes < PnormScratchBytes()) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "butteraugli_pnorm: invalid arguments");
  }
  return LaunchPnorm(distance_map, map_stride, width, height, p, scratch, pnorm,
                     static_cast<cudaStream_t>(stream));
}
