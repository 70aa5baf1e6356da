// Shared transform machinery for the per-transform kernels: strategy
// geometry (src/core/ac_strategy.h:63-143) and the reference CPU DCT in
// double precision with sequential sums (src/codec/dct.cpp:135-230),
// register-tiled four outputs per work item.
#pragma once

#include "common.cuh"

namespace gjxl_b200 {

// Strategy ids (reference src/core/ac_strategy.h:25-53).
constexpr int kStrategyDct8 = 0, kStrategyDct16x16 = 4, kStrategyDct32x32 = 5,
              kStrategyDct16x8 = 6, kStrategyDct8x16 = 7, kStrategyDct32x16 = 10,
              kStrategyDct16x32 = 11;

// Family order of the reference's candidate stages.
constexpr int kFamilyCountT = 7;
__host__ __device__ constexpr int FamilyStrategy(int f) {
  return f == 0 ? kStrategyDct8 : f == 1 ? kStrategyDct16x8 : f == 2 ? kStrategyDct8x16
       : f == 3 ? kStrategyDct16x16 : f == 4 ? kStrategyDct32x16 : f == 5 ? kStrategyDct16x32
       : kStrategyDct32x32;
}
__host__ __device__ constexpr int StrategyFamily(int s) {
  return s == kStrategyDct8 ? 0 : s == kStrategyDct16x8 ? 1 : s == kStrategyDct8x16 ? 2
       : s == kStrategyDct16x16 ? 3 : s == kStrategyDct32x16 ? 4 : s == kStrategyDct16x32 ? 5
       : s == kStrategyDct32x32 ? 6 : -1;
}
// Covered blocks (width, height) per family.
__host__ __device__ constexpr int FamilyCoveredW(int f) {
  return f == 0 ? 1 : f == 1 ? 1 : f == 2 ? 2 : f == 3 ? 2 : f == 4 ? 2 : 4;
}
__host__ __device__ constexpr int FamilyCoveredH(int f) {
  return f == 0 ? 1 : f == 1 ? 2 : f == 2 ? 1 : f == 3 ? 2 : f == 4 ? 4 : f == 5 ? 2 : 4;
}

template <int W, int H>
struct TransformShape {
  static constexpr int N = W * H;
  static constexpr int CW = W / 8, CH = H / 8;  // covered blocks
  // Physical coefficient storage, longer frequency axis contiguous.
  static constexpr int SW = W >= H ? W : H;  // coefficient extent width
  static constexpr int SH = W >= H ? H : W;  // coefficient extent height
  // AcStrategyInfo::coefficient_index.
  __device__ static int Index(int v, int u) { return H < W ? v * W + u : u * H + v; }
};

// Forward pass: out[index(v,u)] = float(sum_y bh[v][y] * (sum_x px[y][x] * bw[u][x])).
// `pixels` (float, N, row-major W) and `tmp` (double, N) in shared memory;
// `bw_t` is the width-length forward basis transposed [x][u], `bh` the
// height-length basis [v][y]. Work items: `channels` x N / 4, strided by
// `threads` from `tid`. Caller synchronizes between passes.
template <int W, int H>
__device__ __forceinline__ void ForwardRows(const float* pixels, double* tmp, const double* bw_t,
                                            int channels, int tid, int threads) {
  constexpr int N = W * H;
  for (int item = tid; item < channels * N / 4; item += threads) {
    const int i = item * 4, c = i / N, yu = i % N, y = yu / W, u0 = yu % W;
    const float* row = pixels + c * N + y * W;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll 8
    for (int x = 0; x < W; ++x) {
      const double p = static_cast<double>(row[x]);
      const double2 b01 = __ldg(reinterpret_cast<const double2*>(bw_t + x * W + u0));
      const double2 b23 = __ldg(reinterpret_cast<const double2*>(bw_t + x * W + u0 + 2));
      s0 += p * b01.x;
      s1 += p * b01.y;
      s2 += p * b23.x;
      s3 += p * b23.y;
    }
    double* out = tmp + i;
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
    out[3] = s3;
  }
}

template <int W, int H>
__device__ __forceinline__ void ForwardColumns(const double* tmp, float* coef, const double* bh,
                                               int channels, int tid, int threads) {
  using S = TransformShape<W, H>;
  constexpr int N = W * H;
  for (int item = tid; item < channels * N / 4; item += threads) {
    const int i = item * 4, c = i / N, vu = i % N, v = vu / W, u0 = vu % W;
    const double* col = tmp + c * N + u0;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll 8
    for (int y = 0; y < H; ++y) {
      const double b = __ldg(bh + v * H + y);
      const double2 t01 = *reinterpret_cast<const double2*>(col + y * W);
      const double2 t23 = *reinterpret_cast<const double2*>(col + y * W + 2);
      s0 += b * t01.x;
      s1 += b * t01.y;
      s2 += b * t23.x;
      s3 += b * t23.y;
    }
    float* out = coef + c * N;
    out[S::Index(v, u0 + 0)] = static_cast<float>(s0);
    out[S::Index(v, u0 + 1)] = static_cast<float>(s1);
    out[S::Index(v, u0 + 2)] = static_cast<float>(s2);
    out[S::Index(v, u0 + 3)] = static_cast<float>(s3);
  }
}

// Inverse passes (src/codec/dct.cpp:184-230): tmp[v][x] = sum_u coef[index(v,u)] *
// iw[u][x]; pixels[y][x] = float(sum_v ih[v][y] * tmp[v][x]).
template <int W, int H>
__device__ __forceinline__ void InverseRows(const float* coef, double* tmp, const double* iw,
                                            int channels, int tid, int threads) {
  using S = TransformShape<W, H>;
  constexpr int N = W * H;
  for (int item = tid; item < channels * N / 4; item += threads) {
    const int i = item * 4, c = i / N, vx = i % N, v = vx / W, x0 = vx % W;
    const float* cf = coef + c * N;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll 8
    for (int u = 0; u < W; ++u) {
      const double k = static_cast<double>(cf[S::Index(v, u)]);
      const double2 b01 = __ldg(reinterpret_cast<const double2*>(iw + u * W + x0));
      const double2 b23 = __ldg(reinterpret_cast<const double2*>(iw + u * W + x0 + 2));
      s0 += k * b01.x;
      s1 += k * b01.y;
      s2 += k * b23.x;
      s3 += k * b23.y;
    }
    double* out = tmp + i;
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
    out[3] = s3;
  }
}

template <int W, int H>
__device__ __forceinline__ void InverseColumns(const double* tmp, float* pixels, const double* ih,
                                               int channels, int tid, int threads) {
  constexpr int N = W * H;
  for (int item = tid; item < channels * N / 4; item += threads) {
    const int i = item * 4, c = i / N, yx = i % N, y = yx / W, x0 = yx % W;
    const double* col = tmp + c * N + x0;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll 8
    for (int v = 0; v < H; ++v) {
      const double b = __ldg(ih + v * H + y);
      const double2 t01 = *reinterpret_cast<const double2*>(col + v * W);
      const double2 t23 = *reinterpret_cast<const double2*>(col + v * W + 2);
      s0 += b * t01.x;
      s1 += b * t01.y;
      s2 += b * t23.x;
      s3 += b * t23.y;
    }
    float* out = pixels + i;
    out[0] = static_cast<float>(s0);
    out[1] = static_cast<float>(s1);
    out[2] = static_cast<float>(s2);
    out[3] = static_cast<float>(s3);
  }
}

}  // namespace gjxl_b200
