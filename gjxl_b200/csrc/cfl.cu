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
// One CTA of four warps per tile; both maps of the tile stay in shared memory.
//
// Phase 1 (all four warps): each warp transforms whole blocks, channel by
// channel. The block's pixels are staged in shared memory as doubles, lane l
// owns row-pass and column-pass outputs (l >> 3, l & 7) and (l >> 3 + 4,
// l & 7), and keeps its three rows of the DCT basis in registers. Each map's
// (a, b) pairs go to shared memory grouped by the reference's lane
// (element i at [i & 3][i >> 2]).
//
// Phase 2 (warps 0-2): the Newton iterations. The derivative sums are twelve
// sequential float chains per map (3 sums x the reference's 4 lanes), so
// their additions cannot be spread out; the per-element terms can. Warps 1
// and 2 (one per map) evaluate the terms of 128-element chunks with all 32
// lanes into a double buffer; warp 0 adds them, lanes 0-11 for y_to_x and
// 16-27 for y_to_b, each lane one chain in element order, then takes the
// Newton step. Named barriers pair the warps: FULL/EMPTY per buffer, and
// XREADY when a new x is published. All three warps run the same loop
// counts (the chunk count follows from the tile, the iteration count from
// flags read after XREADY), so every barrier is met.

#include <cmath>
#include <cstring>

#include "common.cuh"
#include "host_util.h"
#include "tables.h"

namespace gjxl_b200 {
namespace {

constexpr int kTileValues = 64 * 64;  // up to 64 blocks of 64 coefficients
constexpr int kCflThreads = 128;
constexpr int kChunk = 32;           // elements per lane chain in one chunk
constexpr int kTermStride = kChunk + 4;  // floats per term row (bank spread)
constexpr int kTermRows = 24;        // 2 maps x 3 sums x 4 lanes
constexpr size_t kPairBytes = 2 * kTileValues * sizeof(float2);
constexpr size_t kTermBytes = 2 * kTermRows * kTermStride * sizeof(float);
constexpr size_t kPhase1Bytes = 4 * (64 * sizeof(double) * 2 + 64 * sizeof(float));
constexpr size_t kScratchBytes = kTermBytes > kPhase1Bytes ? kTermBytes : kPhase1Bytes;
constexpr size_t kCflSmem = kPairBytes + kScratchBytes + 16;

// Named barrier ids (0 is __syncthreads) and the phase-2 participants.
constexpr int kBarFull = 1;    // + buffer
constexpr int kBarEmpty = 3;   // + buffer
constexpr int kBarXReady = 5;
constexpr int kPhase2Threads = 96;

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

// Barrier ids are immediates, so that the kernel reserves only the six it
// uses; `id` is warp-uniform.
__device__ __forceinline__ void BarSync(int id) {
  switch (id) {
    case kBarFull: asm volatile("bar.sync 1, %0;" :: "n"(kPhase2Threads) : "memory"); break;
    case kBarFull + 1: asm volatile("bar.sync 2, %0;" :: "n"(kPhase2Threads) : "memory"); break;
    case kBarEmpty: asm volatile("bar.sync 3, %0;" :: "n"(kPhase2Threads) : "memory"); break;
    case kBarEmpty + 1: asm volatile("bar.sync 4, %0;" :: "n"(kPhase2Threads) : "memory"); break;
    default: asm volatile("bar.sync 5, %0;" :: "n"(kPhase2Threads) : "memory"); break;
  }
}
__device__ __forceinline__ void BarArrive(int id) {
  switch (id) {
    case kBarFull: asm volatile("bar.arrive 1, %0;" :: "n"(kPhase2Threads) : "memory"); break;
    case kBarFull + 1: asm volatile("bar.arrive 2, %0;" :: "n"(kPhase2Threads) : "memory"); break;
    case kBarEmpty: asm volatile("bar.arrive 3, %0;" :: "n"(kPhase2Threads) : "memory"); break;
    case kBarEmpty + 1: asm volatile("bar.arrive 4, %0;" :: "n"(kPhase2Threads) : "memory"); break;
    default: asm volatile("bar.arrive 5, %0;" :: "n"(kPhase2Threads) : "memory"); break;
  }
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

// The derivative terms of one element for the three sums (center, +eps,
// -eps) at the current x: d = (2/3 a) (|r| + 1) signed like r, r = a x_k + b,
// skipped (zero) where |a x + b| >= 100. A skipped term is a signed zero
// here and +0.0 in the reference; adding either leaves the sum unchanged,
// since a sum that starts at +0.0 is never -0.0.
__device__ __forceinline__ void Terms(float2 v, float x, float xp, float xm, float& t0, float& t1,
                                      float& t2) {
  const float center = fmaf(v.x, x, v.y);
  const float scale = fabsf(center) >= 100.0f ? 0.0f : (2.0f / 3.0f) * v.x;
  const float rp = fmaf(v.x, xp, v.y);
  const float rm = fmaf(v.x, xm, v.y);
  const float d0 = scale * (fabsf(center) + 1.0f);
  const float dp = scale * (fabsf(rp) + 1.0f);
  const float dm = scale * (fabsf(rm) + 1.0f);
  t0 = center < 0.0f ? -d0 : d0;
  t1 = rp < 0.0f ? -dp : dp;
  t2 = rm < 0.0f ? -dm : dm;
}

__global__ void __launch_bounds__(kCflThreads, 3) CflTileKernel(const __grid_constant__ CflParams p) {
  extern __shared__ __align__(16) unsigned char cfl_smem[];
  float2* pairs = reinterpret_cast<float2*>(cfl_smem);  // [map][4][js]
  unsigned char* scratch = cfl_smem + kPairBytes;
  float* xs = reinterpret_cast<float*>(cfl_smem + kPairBytes + kScratchBytes);
  int* dones = reinterpret_cast<int*>(xs + 2);

  const int tile = blockIdx.x;
  const int tx = tile % p.tiles_x, ty = tile / p.tiles_x;
  const int bx0 = tx * 8, by0 = ty * 8;
  const int tw = min(8, static_cast<int>(p.blocks_x) - bx0);
  const int th = min(8, static_cast<int>(p.blocks_y) - by0);
  const int blocks = tw * th;
  const int js = blocks * 16;  // elements per reference lane
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // ---- Phase 1: transforms and pairs.
  {
    double* px = reinterpret_cast<double*>(scratch) + warp * 128;  // 64 pixels
    double* tm = px + 64;                                          // row-pass output
    float* ycoef = reinterpret_cast<float*>(reinterpret_cast<double*>(scratch) + 4 * 128) +
                   warp * 64;
    const int y0 = lane >> 3, u = lane & 7;
    double basis_u[8], basis_v0[8], basis_v1[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      basis_u[i] = __ldg(p.fwd + u * 8 + i);
      basis_v0[i] = __ldg(p.fwd + y0 * 8 + i);
      basis_v1[i] = __ldg(p.fwd + (y0 + 4) * 8 + i);
    }
    // Lane's two coefficients: storage index u * 8 + v, v = y0 and y0 + 4.
    const int index0 = u * 8 + y0, index1 = index0 + 4;
    const float inv_x0 = __ldg(p.inv_x + index0), inv_x1 = __ldg(p.inv_x + index1);
    const float inv_b0 = __ldg(p.inv_b + index0), inv_b1 = __ldg(p.inv_b + index1);
    // The lane's pixels (row lane >> 2, columns 2 (lane & 3) + 0, 1) of the
    // three channels, Y first, then X and B; the next block's are loaded
    // while this one is transformed.
    auto load_block = [&](int b, float2 (&pix)[3]) {
      if (b >= blocks) return;
      const int bx = bx0 + b % tw, by = by0 + b / tw;
      const size_t at = static_cast<size_t>(by * 8 + (lane >> 2)) * p.stride + bx * 8 +
                        (lane & 3) * 2;
      pix[0] = *reinterpret_cast<const float2*>(p.opsin + p.pitch + at);
      pix[1] = *reinterpret_cast<const float2*>(p.opsin + at);
      pix[2] = *reinterpret_cast<const float2*>(p.opsin + 2 * p.pitch + at);
    };
    float2 current[3], next[3];
    load_block(warp, current);
    for (int b = warp; b < blocks; b += 4) {
      load_block(b + 4, next);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int ch = c == 0 ? 1 : c == 1 ? 0 : 2;  // Y first, then X and B
        const float2 pix = current[c];
        __syncwarp();
        reinterpret_cast<double2*>(px)[lane] = make_double2(pix.x, pix.y);
        __syncwarp();
        // Row pass: T[y][u] = sum_x pixel[y][x] * basis[u][x].
        double t0 = 0.0, t1 = 0.0;
#pragma unroll
        for (int x = 0; x < 8; x += 2) {
          const double2 a = reinterpret_cast<const double2*>(px + y0 * 8)[x / 2];
          const double2 e = reinterpret_cast<const double2*>(px + (y0 + 4) * 8)[x / 2];
          t0 += a.x * basis_u[x];
          t0 += a.y * basis_u[x + 1];
          t1 += e.x * basis_u[x];
          t1 += e.y * basis_u[x + 1];
        }
        tm[y0 * 8 + u] = t0;
        tm[(y0 + 4) * 8 + u] = t1;
        __syncwarp();
        // Column pass: coef[v][u] = sum_y basis[v][y] * T[y][u].
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int y = 0; y < 8; ++y) {
          const double t = tm[y * 8 + u];
          s0 += basis_v0[y] * t;
          s1 += basis_v1[y] * t;
        }
        const float c0 = index0 == 0 ? 0.0f : static_cast<float>(s0);  // LLF zeroed
        const float c1 = static_cast<float>(s1);
        if (ch == 1) {
          ycoef[index0] = c0;
          ycoef[index1] = c1;
          __syncwarp();
          continue;
        }
        // Element i = b * 64 + index; reference lane s = index & 3 = y0,
        // position j = i >> 2 = b * 16 + 2u (+1 for index1).
        const bool is_b = ch == 2;
        const float w0 = is_b ? inv_b0 : inv_x0, w1 = is_b ? inv_b1 : inv_x1;
        const float luma0 = ycoef[index0] * w0, luma1 = ycoef[index1] * w1;
        const float chroma0 = c0 * w0, chroma1 = c1 * w1;
        const float base = is_b ? 1.0f : 0.0f;
        float4 out;
        out.x = luma0 / 84.0f;
        out.y = base * luma0 - chroma0;
        out.z = luma1 / 84.0f;
        out.w = base * luma1 - chroma1;
        float2* map_pairs = pairs + (is_b ? kTileValues : 0);
        *reinterpret_cast<float4*>(map_pairs + y0 * js + b * 16 + 2 * u) = out;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) current[c] = next[c];
    }
  }
  __syncthreads();
  if (warp == 3) return;

  // ---- Phase 2: Newton iterations.
  const float kDistanceMultiplierAc = 1.0e-9f;
  const float kEpsilon = 100.0f;
  float* terms = reinterpret_cast<float*>(scratch);  // [buffer][row][kTermStride]
  const int chunks = (js + kChunk - 1) / kChunk;
  if (warp == 0) {
    // Consumer. Lane 16 * map + 4 * kind + slot, kind < 3, owns one chain.
    const int map = lane >> 4, row_in_map = lane & 15;
    const bool chain = row_in_map < 12;
    const int row = map * 12 + (chain ? row_in_map : 0);
    float x = 0.0f;
    bool done = false, all_done = false;
    int g = 0;
    for (int iteration = 0; iteration < p.iterations; ++iteration) {
      if ((lane & 15) == 0) {
        xs[map] = x;
        dones[map] = done ? 1 : 0;
      }
      BarArrive(kBarXReady);
      if (all_done) break;
      float lane_sum = 0.0f;
      for (int c = 0; c < chunks; ++c, ++g) {
        const int buffer = g & 1;
        BarSync(kBarFull + buffer);
        const float4* src = reinterpret_cast<const float4*>(
          terms + (buffer * kTermRows + row) * kTermStride);
        // All of the chunk's terms into registers first (the loads overlap),
        // which also frees the buffer for the producers before the adds.
        // A chunk holds 32 terms per chain, or 16 in a ragged tile's last.
        float4 t[kChunk / 4];
        const bool half = js - c * kChunk < kChunk;
#pragma unroll
        for (int q = 0; q < kChunk / 8; ++q) t[q] = src[q];
        if (!half) {
#pragma unroll
          for (int q = kChunk / 8; q < kChunk / 4; ++q) t[q] = src[q];
        }
        BarArrive(kBarEmpty + buffer);
#pragma unroll
        for (int q = 0; q < kChunk / 8; ++q) {
          lane_sum += t[q].x;
          lane_sum += t[q].y;
          lane_sum += t[q].z;
          lane_sum += t[q].w;
        }
        if (!half) {
#pragma unroll
          for (int q = kChunk / 8; q < kChunk / 4; ++q) {
            lane_sum += t[q].x;
            lane_sum += t[q].y;
            lane_sum += t[q].z;
            lane_sum += t[q].w;
          }
        }
      }
      // Horizontal sums (l0 + l1) + (l2 + l3) for each kind, per map.
      float sums[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int first = (lane & 16) + 4 * k;
        const float l0 = __shfl_sync(0xffffffffu, lane_sum, first + 0);
        const float l1 = __shfl_sync(0xffffffffu, lane_sum, first + 1);
        const float l2 = __shfl_sync(0xffffffffu, lane_sum, first + 2);
        const float l3 = __shfl_sync(0xffffffffu, lane_sum, first + 3);
        sums[k] = (l0 + l1) + (l2 + l3);
      }
      if (!done) {
        const float n = static_cast<float>(blocks * 64);
        const float center = 2.0f * kDistanceMultiplierAc * n * x + sums[0];
        const float plus = 2.0f * kDistanceMultiplierAc * n * (x + kEpsilon) + sums[1];
        const float minus = 2.0f * kDistanceMultiplierAc * n * (x - kEpsilon) + sums[2];
        const float second = (plus - minus) / (2.0f * kEpsilon);
        const float step = center / (second + 0.85f);
        x = x - fminf(fmaxf(step, -20.0f), 20.0f);
        if (fabsf(step) < 3.0e-3f) done = true;
      }
      // Every lane of a map half holds the same sums, x and flag.
      all_done = __shfl_sync(0xffffffffu, done, 0) && __shfl_sync(0xffffffffu, done, 16);
    }
    if (lane == 0) p.y_to_x[tile] = QuantizeMultiplier(x);
    if (lane == 16) p.y_to_b[tile] = QuantizeMultiplier(x);
    return;
  }
  // Producers: warp 1 for y_to_x, warp 2 for y_to_b. Lane (slot s, quad q)
  // evaluates elements j = chunk * 32 + 4q .. 4q + 3 of reference lane s.
  const int map = warp - 1;
  const float2* map_pairs = pairs + map * kTileValues;
  const int s = lane >> 3, q = lane & 7;
  int g = 0;
  for (int iteration = 0; iteration < p.iterations; ++iteration) {
    BarSync(kBarXReady);
    const float x = xs[map];
    const bool skip = dones[map] != 0;
    if (dones[0] != 0 && dones[1] != 0) break;
    const float xp = x + kEpsilon, xm = x - kEpsilon;
    for (int c = 0; c < chunks; ++c, ++g) {
      const int buffer = g & 1;
      if (g >= 2) BarSync(kBarEmpty + buffer);
      const int j = c * kChunk + 4 * q;
      if (!skip && j < js) {
        const float4* src = reinterpret_cast<const float4*>(map_pairs + s * js + j);
        const float4 ab01 = src[0], ab23 = src[1];
        float4 o0, o1, o2;
        Terms(make_float2(ab01.x, ab01.y), x, xp, xm, o0.x, o1.x, o2.x);
        Terms(make_float2(ab01.z, ab01.w), x, xp, xm, o0.y, o1.y, o2.y);
        Terms(make_float2(ab23.x, ab23.y), x, xp, xm, o0.z, o1.z, o2.z);
        Terms(make_float2(ab23.z, ab23.w), x, xp, xm, o0.w, o1.w, o2.w);
        float* dst = terms + (buffer * kTermRows + map * 12 + s) * kTermStride + 4 * q;
        *reinterpret_cast<float4*>(dst) = o0;
        *reinterpret_cast<float4*>(dst + 4 * kTermStride) = o1;
        *reinterpret_cast<float4*>(dst + 8 * kTermStride) = o2;
      }
      __syncwarp();
      BarArrive(kBarFull + buffer);
    }
  }
  // Meet the consumer's last two EMPTY arrivals.
  for (int last = max(0, g - 2); last < g; ++last) BarSync(kBarEmpty + (last & 1));
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
  status = CheckCuda(cudaFuncSetAttribute(CflTileKernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(kCflSmem)),
                     "initial_cfl smem attribute");
  if (status != GJXL_B200_OK) return status;
  CflTileKernel<<<p.tiles_x * p.tiles_y, kCflThreads, kCflSmem, stream>>>(p);
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
      opsin_stride < padded_width || opsin_stride % 2 ||
      opsin_plane_pitch < opsin_stride * padded_height || opsin_plane_pitch % 2 ||
      reinterpret_cast<uintptr_t>(opsin) % 8) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "initial_cfl: invalid arguments");
  }
  return LaunchInitialCfl(opsin, opsin_stride, opsin_plane_pitch, padded_width, padded_height,
                          y_to_x, y_to_b, static_cast<cudaStream_t>(stream));
}
