// Row N4: the learned proposal network and its training kernels.
//
// The reference has no learned component. The network proposes, for every
// 8x8 block of a 64x64 tile, the AC strategies most likely chosen by the
// plain search and a log-scale correction of the adjusted quant field (the
// field the refinement loop starts from) towards the loop's final field:
//
//   input  80 x 80 x 4: the tile's Gaborish-inverted XYB with an 8-px halo
//          (edge-clamped), scaled per channel, and log2 of the distance
//   conv1  3x3 stride 2, 4 -> 32, ReLU     (40 x 40)
//   conv2  3x3 stride 2, 32 -> 32, ReLU    (20 x 20)
//   conv3  3x3 stride 2, 32 -> 32, ReLU    (10 x 10)
//   conv4  3x3 stride 1, 32 -> 32, ReLU    (10 x 10)
//   head   1x1, 32 -> 28 on the centre 8 x 8 cells (one per block): 27
//          strategy logits and the log field scale.
//
// Arithmetic: weights and activations are rounded to BF16, products are
// accumulated in FP32 (bias first, then taps in (ky, kx, ci) order), FP32
// master weights and gradients. Activations are NHWC (32 channels = 64 bytes
// per pixel); weights are [co][ky][kx][ci] and staged in shared memory as
// [tap][ci][co], so that one 16-byte load feeds four output channels.
//
// Training kernels: the loss (softmax cross-entropy over the 27 logits plus
// the squared error of the field scale, averaged over all block slots, with
// per-block weights 0 for blocks outside the image), the head and
// convolution backward passes (input gradients per input pixel; weight
// gradients as per-chunk partial sums reduced in a fixed order, so a step is
// deterministic), and AdamW with decoupled weight decay.

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "cnn.h"
#include "common.cuh"
#include "host_util.h"
#include "umma.cuh"

namespace gjxl_b200 {
namespace {

size_t Align(size_t v, size_t a) { return (v + a - 1) / a * a; }

__device__ __forceinline__ float RoundBf16(float v) {
  return __bfloat162float(__float2bfloat16_rn(v));
}

struct LayerShape {
  int cin, in_size, out_size, stride, w_offset, b_offset;
};

__host__ __device__ inline LayerShape Layer(int l) {
  switch (l) {
    case 0: return {kCnnInChannels, kCnnIn, 40, 2, kCnnW1, kCnnB1};
    case 1: return {kCnnC, 40, 20, 2, kCnnW2, kCnnB2};
    case 2: return {kCnnC, 20, 10, 2, kCnnW3, kCnnB3};
    default: return {kCnnC, 10, 10, 1, kCnnW4, kCnnB4};
  }
}

// ---------------------------------------------------------------------------
// Input tiles.

struct GatherParams {
  const float* opsin;  // Gaborish-inverted padded XYB
  size_t stride, pitch;
  int pw, ph, tiles_x;
  const int* tile_list;  // tile indices (null: tile i = i)
  float log2_distance;
  __nv_bfloat16* out;    // [n][80][80][4]
  int n;
};

// Per-channel input scaling: X is small around 0, Y and B lie in [0, ~1].
__global__ void GatherKernel(const __grid_constant__ GatherParams p) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(p.n) * kCnnIn * kCnnIn) return;
  const int t = static_cast<int>(i / (kCnnIn * kCnnIn));
  const int pix = static_cast<int>(i % (kCnnIn * kCnnIn));
  const int tile = p.tile_list != nullptr ? p.tile_list[t] : t;
  const int tx = tile % p.tiles_x, ty = tile / p.tiles_x;
  const int x = min(max(tx * 64 - 8 + pix % kCnnIn, 0), p.pw - 1);
  const int y = min(max(ty * 64 - 8 + pix / kCnnIn, 0), p.ph - 1);
  const size_t at = static_cast<size_t>(y) * p.stride + x;
  const float xv = p.opsin[at], yv = p.opsin[p.pitch + at], bv = p.opsin[2 * p.pitch + at];
  __nv_bfloat16* o = p.out + i * kCnnInChannels;
  o[0] = __float2bfloat16_rn(xv * 24.0f);
  o[1] = __float2bfloat16_rn(yv * 2.0f - 1.0f);
  o[2] = __float2bfloat16_rn((bv - yv) * 4.0f);
  o[3] = __float2bfloat16_rn(p.log2_distance);
}

// ---------------------------------------------------------------------------
// Forward convolution: one thread per output pixel, all 32 output channels.

template <int CIN>
__global__ void __launch_bounds__(128)
ConvForwardKernel(const __nv_bfloat16* in, const float* params, int layer, int n,
                  __nv_bfloat16* out) {
  const LayerShape L = Layer(layer);
  __shared__ __align__(16) float ws[9 * CIN * kCnnC];
  __shared__ float bs[kCnnC];
  for (int i = threadIdx.x; i < 9 * CIN * kCnnC; i += blockDim.x) {
    const int co = i % kCnnC, ci = (i / kCnnC) % CIN, tap = i / (kCnnC * CIN);
    ws[i] = RoundBf16(params[L.w_offset + (co * 9 + tap) * CIN + ci]);
  }
  if (threadIdx.x < kCnnC) bs[threadIdx.x] = params[L.b_offset + threadIdx.x];
  __syncthreads();
  const size_t pixel = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t per_tile = static_cast<size_t>(L.out_size) * L.out_size;
  if (pixel >= static_cast<size_t>(n) * per_tile) return;
  const size_t t = pixel / per_tile;
  const int oy = static_cast<int>(pixel % per_tile) / L.out_size;
  const int ox = static_cast<int>(pixel % per_tile) % L.out_size;
  float acc[kCnnC];
#pragma unroll
  for (int co = 0; co < kCnnC; ++co) acc[co] = bs[co];
  for (int tap = 0; tap < 9; ++tap) {
    const int iy = oy * L.stride + tap / 3 - 1, ix = ox * L.stride + tap % 3 - 1;
    if (iy < 0 || iy >= L.in_size || ix < 0 || ix >= L.in_size) continue;
    const __nv_bfloat16* x = in + ((t * L.in_size + iy) * L.in_size + ix) * CIN;
    for (int c8 = 0; c8 < CIN; c8 += (CIN < 8 ? CIN : 8)) {
      float xv[CIN < 8 ? CIN : 8];
      if constexpr (CIN >= 8) {
        const uint4 raw = *reinterpret_cast<const uint4*>(x + c8);
        const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&raw);
#pragma unroll
        for (int k = 0; k < 8; ++k) xv[k] = __bfloat162float(h[k]);
      } else {
#pragma unroll
        for (int k = 0; k < CIN; ++k) xv[k] = __bfloat162float(x[k]);
      }
#pragma unroll
      for (int k = 0; k < (CIN < 8 ? CIN : 8); ++k) {
        const float4* w4 = reinterpret_cast<const float4*>(ws + (tap * CIN + c8 + k) * kCnnC);
#pragma unroll
        for (int q = 0; q < kCnnC / 4; ++q) {
          const float4 w = w4[q];
          acc[4 * q + 0] = fmaf(w.x, xv[k], acc[4 * q + 0]);
          acc[4 * q + 1] = fmaf(w.y, xv[k], acc[4 * q + 1]);
          acc[4 * q + 2] = fmaf(w.z, xv[k], acc[4 * q + 2]);
          acc[4 * q + 3] = fmaf(w.w, xv[k], acc[4 * q + 3]);
        }
      }
    }
  }
  __align__(16) __nv_bfloat16 o[kCnnC];
#pragma unroll
  for (int co = 0; co < kCnnC; ++co) o[co] = __float2bfloat16_rn(fmaxf(acc[co], 0.0f));
  uint4* dst = reinterpret_cast<uint4*>(out + pixel * kCnnC);
#pragma unroll
  for (int q = 0; q < 4; ++q) dst[q] = reinterpret_cast<const uint4*>(o)[q];
}

// The same convolution as implicit GEMMs on the fifth-generation tensor
// cores, for inference: rows are output pixels (M = 128 per MMA tile), K the
// 3x3 x Cin patch (tap-major, padded to a multiple of 16), N the 32 output
// channels. Each thread gathers its row's patch from the NHWC input into the
// canonical no-swizzle K-major layout in shared memory (16-byte pieces: one
// pixel's 8 channels, or two taps of the 4-channel input); one thread issues
// the K / 16 MMAs into a 32-column tensor-memory accumulator; each thread
// reads its row back (tcgen05.ld), adds the bias, applies the ReLU and
// stores 64 bytes of BF16. Persistent CTAs walk the M tiles. The products
// are the SIMT kernel's (BF16 x BF16); only the FP32 summation order differs.
constexpr int kConvTcThreads = 128;
constexpr uint32_t kConvWaitPolls = 1u << 22;

template <int CIN>
struct ConvTcShape {
  static constexpr int K = 9 * CIN;
  static constexpr int KP = (K + 15) / 16 * 16;  // 48 or 288
  static constexpr int kABytes = 128 * KP * 2;
  static constexpr int kBBytes = kCnnC * KP * 2;
  static constexpr size_t kSmem = static_cast<size_t>(kABytes) + kBBytes;
};

template <int KP>
__device__ __forceinline__ int KMajor(int row, int k) {
  return (row >> 3) * (KP / 8) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

template <int CIN>
__global__ void __launch_bounds__(kConvTcThreads)
ConvTcKernel(const __nv_bfloat16* in, const float* params, int layer, int n, __nv_bfloat16* out,
             uint32_t* error) {
  using T = ConvTcShape<CIN>;
  constexpr int KP = T::KP;
  const LayerShape L = Layer(layer);
  extern __shared__ __align__(128) unsigned char conv_smem[];
  unsigned char* a_tile = conv_smem;
  unsigned char* b_tile = conv_smem + T::kABytes;
  __shared__ __align__(8) uint64_t barrier;
  __shared__ uint32_t tmem_slot;
  __shared__ float bias[kCnnC];
  __shared__ int aborted;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) umma::Allocate(&tmem_slot, 32);
  if (tid == 0) {
    umma::InitBarrier(&barrier, 1);
    aborted = 0;
  }
  // B: the weights rounded to BF16, K-major [co][k], zero past K.
  for (int i = tid; i < kCnnC * KP; i += kConvTcThreads) {
    const int co = i / KP, k = i % KP;
    const float wv = k < T::K ? params[L.w_offset + (co * 9 + k / CIN) * CIN + k % CIN] : 0.0f;
    *reinterpret_cast<__nv_bfloat16*>(b_tile + KMajor<KP>(co, k)) = __float2bfloat16_rn(wv);
  }
  if (tid < kCnnC) bias[tid] = params[L.b_offset + tid];
  umma::FenceAsyncShared();
  umma::FenceBeforeSync();
  __syncthreads();
  umma::FenceAfterSync();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = tmem + (static_cast<uint32_t>(warp * 32) << 16);
  const uint32_t a_address = umma::SmemAddress(a_tile), b_address = umma::SmemAddress(b_tile);
  constexpr uint32_t kInstr = umma::InstrBf16F32(128, kCnnC, false, false);
  const size_t per_tile = static_cast<size_t>(L.out_size) * L.out_size;
  const size_t total = static_cast<size_t>(n) * per_tile;
  const size_t m_tiles = (total + 127) / 128;
  uint32_t phase = 0;
  for (size_t mt = blockIdx.x; mt < m_tiles; mt += gridDim.x) {
    const size_t m = mt * 128 + tid;
    if (m < total) {
      const size_t t = m / per_tile;
      const int oy = static_cast<int>(m % per_tile) / L.out_size;
      const int ox = static_cast<int>(m % per_tile) % L.out_size;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const int iy = oy * L.stride + tap / 3 - 1, ix = ox * L.stride + tap % 3 - 1;
        const bool valid = iy >= 0 && iy < L.in_size && ix >= 0 && ix < L.in_size;
        const __nv_bfloat16* src = in + ((t * L.in_size + (valid ? iy : 0)) * L.in_size +
                                         (valid ? ix : 0)) * CIN;
        if constexpr (CIN == kCnnC) {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const uint4 v = valid ? *reinterpret_cast<const uint4*>(src + 8 * c)
                                  : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4*>(a_tile + KMajor<KP>(tid, tap * CIN + 8 * c)) = v;
          }
        } else {
          const uint2 v = valid ? *reinterpret_cast<const uint2*>(src) : make_uint2(0, 0);
          *reinterpret_cast<uint2*>(a_tile + KMajor<KP>(tid, tap * CIN)) = v;
        }
      }
      if constexpr (T::K < KP) {
        // K = 36 .. 47 of the 4-channel input.
        *reinterpret_cast<uint2*>(a_tile + KMajor<KP>(tid, T::K)) = make_uint2(0, 0);
        for (int k = (T::K + 8) / 8 * 8; k < KP; k += 8)
          *reinterpret_cast<uint4*>(a_tile + KMajor<KP>(tid, k)) = make_uint4(0, 0, 0, 0);
      }
    }
    umma::FenceAsyncShared();
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
    if (tid == 0) {
#pragma unroll
      for (int kc = 0; kc < KP / 16; ++kc) {
        const uint64_t a = umma::Descriptor(a_address + kc * 256, 128, (KP / 8) * 128);
        const uint64_t b = umma::Descriptor(b_address + kc * 256, 128, (KP / 8) * 128);
        umma::Mma(tmem, a, b, kInstr, kc > 0);
      }
      umma::Commit(&barrier);
    }
    const bool ok = umma::WaitParity(&barrier, phase, kConvWaitPolls);
    phase ^= 1u;
    umma::FenceAfterSync();
    if (!__syncthreads_and(ok ? 1 : 0)) {
      if (tid == 0) {
        aborted = 1;
        RaiseError(error, kErrorInternal);
      }
      break;
    }
    float acc[kCnnC];
    umma::Load<32>(lane_base, acc);
    if (m < total) {
      __align__(16) __nv_bfloat16 o[kCnnC];
#pragma unroll
      for (int co = 0; co < kCnnC; ++co)
        o[co] = __float2bfloat16_rn(fmaxf(acc[co] + bias[co], 0.0f));
      uint4* dst = reinterpret_cast<uint4*>(out + m * kCnnC);
#pragma unroll
      for (int q = 0; q < 4; ++q) dst[q] = reinterpret_cast<const uint4*>(o)[q];
    }
    // The next tile's gather and MMA overwrite the operand and accumulator.
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
  }
  // A CTA that gave up waits once more (bounded) for the tensor core to
  // finish with its tensor memory before releasing it.
  __syncthreads();
  if (aborted) umma::WaitParity(&barrier, phase ^ 1u, kConvWaitPolls);
  umma::FenceBeforeSync();
  __syncthreads();
  umma::FenceAfterSync();
  if (warp == 0) umma::Deallocate(tmem, 32);
}

// Head: 28 outputs per centre cell (FP32).
__global__ void HeadForwardKernel(const __nv_bfloat16* a4, const float* params, int n,
                                  float* out) {
  __shared__ float wh[kCnnHead * kCnnC];
  __shared__ float bh[kCnnHead];
  for (int i = threadIdx.x; i < kCnnHead * kCnnC; i += blockDim.x)
    wh[i] = RoundBf16(params[kCnnWh + i]);
  if (threadIdx.x < kCnnHead) bh[threadIdx.x] = params[kCnnBh + threadIdx.x];
  __syncthreads();
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(n) * 64) return;
  const size_t t = i / 64;
  const int cell = static_cast<int>(i % 64);
  const int cy = cell / 8 + 1, cx = cell % 8 + 1;
  const __nv_bfloat16* x = a4 + ((t * 10 + cy) * 10 + cx) * kCnnC;
  float xv[kCnnC];
#pragma unroll
  for (int c = 0; c < kCnnC; ++c) xv[c] = __bfloat162float(x[c]);
  for (int k = 0; k < kCnnHead; ++k) {
    float acc = bh[k];
#pragma unroll
    for (int c = 0; c < kCnnC; ++c) acc = fmaf(wh[k * kCnnC + c], xv[c], acc);
    out[i * kCnnHead + k] = acc;
  }
}

// ---------------------------------------------------------------------------
// Loss and its gradient with respect to the head outputs.

__global__ void LossKernel(const float* head, const uint8_t* labels, const float* targets,
                           const float* weights, int n, float qf_weight, float* dhead,
                           float* partial) {
  __shared__ float sums[256];
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  float loss = 0.0f;
  if (i < static_cast<size_t>(n) * 64) {
    const float* h = head + i * kCnnHead;
    const float w = weights[i];
    const float scale = w / (static_cast<float>(n) * 64.0f);
    float m = h[0];
    for (int k = 1; k < kCnnStrategies; ++k) m = fmaxf(m, h[k]);
    float z = 0.0f;
    for (int k = 0; k < kCnnStrategies; ++k) z += expf(h[k] - m);
    const int label = labels[i];
    const float lse = m + logf(z);
    const float e = h[kCnnStrategies] - targets[i];
    loss = w * ((lse - h[label]) + qf_weight * e * e);
    float* d = dhead + i * kCnnHead;
    for (int k = 0; k < kCnnStrategies; ++k)
      d[k] = scale * (expf(h[k] - lse) - (k == label ? 1.0f : 0.0f));
    d[kCnnStrategies] = scale * 2.0f * qf_weight * e;
  }
  sums[threadIdx.x] = loss;
  __syncthreads();
  for (int half = 128; half >= 1; half >>= 1) {
    if (threadIdx.x < half) sums[threadIdx.x] += sums[threadIdx.x + half];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sums[0];
}

__global__ void LossReduceKernel(const float* partial, int count, int n, float* loss) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float s = 0.0f;
  for (int i = 0; i < count; ++i) s += partial[i];
  *loss = s / (static_cast<float>(n) * 64.0f);
}

// Head backward: input gradient of the conv4 output (zero off the centre)
// and per-chunk weight-gradient partials.
__global__ void HeadBackwardInputKernel(const float* dhead, const float* params, int n,
                                        float* da4) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(n) * 100) return;
  const size_t t = i / 100;
  const int cy = static_cast<int>(i % 100) / 10, cx = static_cast<int>(i % 100) % 10;
  float* d = da4 + i * kCnnC;
  if (cy < 1 || cy > 8 || cx < 1 || cx > 8) {
    for (int c = 0; c < kCnnC; ++c) d[c] = 0.0f;
    return;
  }
  const float* g = dhead + (t * 64 + (cy - 1) * 8 + (cx - 1)) * kCnnHead;
  for (int c = 0; c < kCnnC; ++c) {
    float acc = 0.0f;
    for (int k = 0; k < kCnnHead; ++k) acc = fmaf(RoundBf16(params[kCnnWh + k * kCnnC + c]), g[k], acc);
    d[c] = acc;
  }
}

constexpr int kHeadChunk = 256;  // cells per partial

__global__ void HeadBackwardWeightKernel(const float* dhead, const __nv_bfloat16* a4, int n,
                                         float* partial) {
  // One CTA per chunk of cells; thread j < 28 * 33 owns dWh[k][c] (c < 32)
  // or dbh[k] (c == 32).
  const int j = threadIdx.x;
  if (j >= kCnnHead * (kCnnC + 1)) return;
  const int k = j / (kCnnC + 1), c = j % (kCnnC + 1);
  const size_t begin = static_cast<size_t>(blockIdx.x) * kHeadChunk;
  const size_t end = min(begin + kHeadChunk, static_cast<size_t>(n) * 64);
  float acc = 0.0f;
  for (size_t i = begin; i < end; ++i) {
    const size_t t = i / 64;
    const int cell = static_cast<int>(i % 64);
    const float g = dhead[i * kCnnHead + k];
    const float x = c == kCnnC ? 1.0f
                               : __bfloat162float(a4[((t * 10 + cell / 8 + 1) * 10 + cell % 8 + 1) *
                                                        kCnnC + c]);
    acc = fmaf(g, x, acc);
  }
  partial[static_cast<size_t>(blockIdx.x) * kCnnHead * (kCnnC + 1) + j] = acc;
}

// Convolution backward. dz = dy * (y > 0) is formed on the fly.
constexpr int kConvChunk = 512;  // output pixels per weight-gradient partial

template <int CIN>
__global__ void __launch_bounds__(256)
ConvBackwardWeightKernel(const float* dy, const __nv_bfloat16* y, const __nv_bfloat16* x,
                         int layer, int n, float* partial) {
  // Thread (cg, pg): output channels 4cg..4cg+3 x patch entries 9pg..9pg+8
  // (patch entry = tap * CIN + ci); thread 0..31 also sums the bias of its co.
  constexpr int kPatch = 9 * CIN;
  constexpr int kGroups = kPatch / 9;
  const LayerShape L = Layer(layer);
  __shared__ float dz[kCnnC];
  __shared__ float patch[kPatch];
  const int tid = threadIdx.x;
  const int cg = tid / kGroups, pg = tid % kGroups;
  const bool active = tid < 8 * kGroups;
  float acc[4][9] = {};
  float bias = 0.0f;
  const size_t per_tile = static_cast<size_t>(L.out_size) * L.out_size;
  const size_t total = static_cast<size_t>(n) * per_tile;
  const size_t begin = static_cast<size_t>(blockIdx.x) * kConvChunk;
  const size_t end = min(begin + kConvChunk, total);
  for (size_t pixel = begin; pixel < end; ++pixel) {
    const size_t t = pixel / per_tile;
    const int oy = static_cast<int>(pixel % per_tile) / L.out_size;
    const int ox = static_cast<int>(pixel % per_tile) % L.out_size;
    __syncthreads();
    if (tid < kCnnC) {
      const float yv = __bfloat162float(y[pixel * kCnnC + tid]);
      dz[tid] = yv > 0.0f ? dy[pixel * kCnnC + tid] : 0.0f;
    }
    for (int e = tid; e < kPatch; e += blockDim.x) {
      const int tap = e / CIN, ci = e % CIN;
      const int iy = oy * L.stride + tap / 3 - 1, ix = ox * L.stride + tap % 3 - 1;
      patch[e] = (iy < 0 || iy >= L.in_size || ix < 0 || ix >= L.in_size)
                   ? 0.0f
                   : __bfloat162float(x[((t * L.in_size + iy) * L.in_size + ix) * CIN + ci]);
    }
    __syncthreads();
    if (active) {
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const float g = dz[4 * cg + a];
#pragma unroll
        for (int b = 0; b < 9; ++b) acc[a][b] = fmaf(g, patch[9 * pg + b], acc[a][b]);
      }
    }
    if (tid < kCnnC) bias += dz[tid];
  }
  float* out = partial + static_cast<size_t>(blockIdx.x) * (kCnnC * kPatch + kCnnC);
  if (active) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 9; ++b) {
        const int co = 4 * cg + a, e = 9 * pg + b;
        // Stored in the parameter layout [co][tap][ci].
        out[co * kPatch + e] = acc[a][b];
      }
  }
  if (tid < kCnnC) out[kCnnC * kPatch + tid] = bias;
}

template <int CIN>
__global__ void __launch_bounds__(128)
ConvBackwardInputKernel(const float* dy, const __nv_bfloat16* y, const float* params, int layer,
                        int n, float* dx) {
  const LayerShape L = Layer(layer);
  __shared__ __align__(16) float ws[9 * CIN * kCnnC];
  for (int i = threadIdx.x; i < 9 * CIN * kCnnC; i += blockDim.x) {
    const int co = i % kCnnC, ci = (i / kCnnC) % CIN, tap = i / (kCnnC * CIN);
    ws[i] = RoundBf16(params[L.w_offset + (co * 9 + tap) * CIN + ci]);
  }
  __syncthreads();
  const size_t pixel = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t per_tile = static_cast<size_t>(L.in_size) * L.in_size;
  if (pixel >= static_cast<size_t>(n) * per_tile) return;
  const size_t t = pixel / per_tile;
  const int iy = static_cast<int>(pixel % per_tile) / L.in_size;
  const int ix = static_cast<int>(pixel % per_tile) % L.in_size;
  float acc[CIN];
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.0f;
  for (int tap = 0; tap < 9; ++tap) {
    const int ny = iy + 1 - tap / 3, nx = ix + 1 - tap % 3;
    if (ny < 0 || nx < 0 || ny % L.stride || nx % L.stride) continue;
    const int oy = ny / L.stride, ox = nx / L.stride;
    if (oy >= L.out_size || ox >= L.out_size) continue;
    const size_t o = (t * L.out_size + oy) * L.out_size + ox;
    float dz[kCnnC];
#pragma unroll
    for (int co = 0; co < kCnnC; ++co) {
      const float yv = __bfloat162float(y[o * kCnnC + co]);
      dz[co] = yv > 0.0f ? dy[o * kCnnC + co] : 0.0f;
    }
#pragma unroll
    for (int ci = 0; ci < CIN; ++ci) {
      const float4* w4 = reinterpret_cast<const float4*>(ws + (tap * CIN + ci) * kCnnC);
#pragma unroll
      for (int q = 0; q < kCnnC / 4; ++q) {
        const float4 w = w4[q];
        acc[ci] = fmaf(w.x, dz[4 * q + 0], acc[ci]);
        acc[ci] = fmaf(w.y, dz[4 * q + 1], acc[ci]);
        acc[ci] = fmaf(w.z, dz[4 * q + 2], acc[ci]);
        acc[ci] = fmaf(w.w, dz[4 * q + 3], acc[ci]);
      }
    }
  }
  float* d = dx + pixel * CIN;
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) d[ci] = acc[ci];
}

__global__ void HeadGradScatterKernel(const float* reduced, float* grads) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= kCnnHead * (kCnnC + 1)) return;
  const int k = j / (kCnnC + 1), c = j % (kCnnC + 1);
  if (c == kCnnC) {
    grads[kCnnBh + k] = reduced[j];
  } else {
    grads[kCnnWh + k * kCnnC + c] = reduced[j];
  }
}

// Fixed-order sum of `chunks` partial rows of `width` values into grads.
__global__ void ReducePartialsKernel(const float* partial, int chunks, int width,
                                     float* grads) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= width) return;
  float s = 0.0f;
  for (int c = 0; c < chunks; ++c) s += partial[static_cast<size_t>(c) * width + j];
  grads[j] = s;
}

__global__ void AdamWKernel(float* params, const float* grads, float* m, float* v, int count,
                            float lr, float beta1, float beta2, float eps, float weight_decay,
                            float bias1, float bias2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float g = grads[i];
  const float mi = beta1 * m[i] + (1.0f - beta1) * g;
  const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float mhat = mi / bias1, vhat = vi / bias2;
  params[i] -= lr * (mhat / (sqrtf(vhat) + eps) + weight_decay * params[i]);
}

// ---------------------------------------------------------------------------
// Proposals of the analysis.

// Per block: the three most likely of the seven searched strategies (by
// logit), the probability mass of those three (softmax over all 27), and
// the predicted log field scale.
__global__ void ProposeKernel(const float* head, int n, int tiles_x, int blocks_x, int blocks_y,
                              uint8_t* proposals, float* confidence, float* log_scale) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(n) * 64) return;
  const int tile = static_cast<int>(i / 64), cell = static_cast<int>(i % 64);
  const int bx = (tile % tiles_x) * 8 + cell % 8, by = (tile / tiles_x) * 8 + cell / 8;
  if (bx >= blocks_x || by >= blocks_y) return;
  const float* h = head + i * kCnnHead;
  float m = h[0];
  for (int k = 1; k < kCnnStrategies; ++k) m = fmaxf(m, h[k]);
  float z = 0.0f;
  for (int k = 0; k < kCnnStrategies; ++k) z += expf(h[k] - m);
  constexpr int kSearched[7] = {0, 6, 7, 4, 10, 11, 5};
  int best[3] = {-1, -1, -1};
  for (int r = 0; r < 3; ++r) {
    float top = -INFINITY;
    for (int s : kSearched) {
      if (s == best[0] || s == best[1]) continue;
      if (best[r] < 0 || h[s] > top) {
        top = h[s];
        best[r] = s;
      }
    }
  }
  float mass = 0.0f;
  for (int r = 0; r < 3; ++r) mass += expf(h[best[r]] - m) / z;
  const size_t b = static_cast<size_t>(by) * blocks_x + bx;
  for (int r = 0; r < 3; ++r) proposals[3 * b + r] = static_cast<uint8_t>(best[r]);
  confidence[b] = mass;
  log_scale[b] = h[kCnnStrategies];
}

}  // namespace

size_t CnnWorkspaceBytes(int n) {
  const size_t a0 = static_cast<size_t>(n) * kCnnIn * kCnnIn * kCnnInChannels * 2;
  const size_t a1 = static_cast<size_t>(n) * 40 * 40 * kCnnC * 2;
  const size_t a2 = static_cast<size_t>(n) * 20 * 20 * kCnnC * 2;
  const size_t a3 = static_cast<size_t>(n) * 10 * 10 * kCnnC * 2;
  const size_t head = static_cast<size_t>(n) * 64 * kCnnHead * 4;
  return Align(a0, 256) + Align(a1, 256) + Align(a2, 256) + 2 * Align(a3, 256) + Align(head, 256);
}

CnnActivations CnnLayout(void* workspace, int n) {
  CnnActivations a;
  unsigned char* p = static_cast<unsigned char*>(workspace);
  const size_t sizes[6] = {static_cast<size_t>(n) * kCnnIn * kCnnIn * kCnnInChannels * 2,
                           static_cast<size_t>(n) * 40 * 40 * kCnnC * 2,
                           static_cast<size_t>(n) * 20 * 20 * kCnnC * 2,
                           static_cast<size_t>(n) * 10 * 10 * kCnnC * 2,
                           static_cast<size_t>(n) * 10 * 10 * kCnnC * 2,
                           static_cast<size_t>(n) * 64 * kCnnHead * 4};
  void* ptrs[6];
  for (int i = 0; i < 6; ++i) {
    ptrs[i] = p;
    p += Align(sizes[i], 256);
  }
  for (int i = 0; i < 5; ++i) a.act[i] = static_cast<__nv_bfloat16*>(ptrs[i]);
  a.head = static_cast<float*>(ptrs[5]);
  return a;
}

int CnnGather(const float* opsin, size_t stride, size_t pitch, size_t pw, size_t ph,
              const int* tile_list, int n, float distance, __nv_bfloat16* out,
              cudaStream_t stream) {
  GatherParams p;
  p.opsin = opsin;
  p.stride = stride;
  p.pitch = pitch;
  p.pw = static_cast<int>(pw);
  p.ph = static_cast<int>(ph);
  p.tiles_x = static_cast<int>((pw / 8 + 7) / 8);
  p.tile_list = tile_list;
  p.log2_distance = std::log2(distance);
  p.out = out;
  p.n = n;
  const size_t total = static_cast<size_t>(n) * kCnnIn * kCnnIn;
  GatherKernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(p);
  return CheckLaunch("cnn gather");
}

template <int CIN>
int LaunchConvTc(const CnnActivations& a, const float* params, int layer, int n, uint32_t* error,
                 cudaStream_t stream) {
  using T = ConvTcShape<CIN>;
  int status = CheckCuda(cudaFuncSetAttribute(ConvTcKernel<CIN>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(T::kSmem)),
                         "cnn tensor-core smem attribute");
  if (status != GJXL_B200_OK) return status;
  const LayerShape L = Layer(layer);
  const size_t tiles = (static_cast<size_t>(n) * L.out_size * L.out_size + 127) / 128;
  // As many CTAs as fit on the device at once (shared memory with the static
  // part and the runtime's 1 KB per CTA, threads, and 16 x 32 tensor-memory
  // columns per SM), each walking M tiles.
  int device = 0, sms = 148, smem_per_sm = 232448;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
  cudaFuncAttributes attributes;
  status = CheckCuda(cudaFuncGetAttributes(&attributes, ConvTcKernel<CIN>),
                     "cnn tensor-core attributes");
  if (status != GJXL_B200_OK) return status;
  const int per_cta = static_cast<int>(T::kSmem + attributes.sharedSizeBytes) + 1024;
  const int per_sm = std::max(1, std::min({smem_per_sm / per_cta, 2048 / kConvTcThreads, 16}));
  const unsigned grid =
    static_cast<unsigned>(std::min<size_t>(tiles, static_cast<size_t>(sms) * per_sm));
  ConvTcKernel<CIN><<<grid, kConvTcThreads, T::kSmem, stream>>>(a.act[layer], params, layer, n,
                                                                a.act[layer + 1], error);
  return CheckLaunch("cnn tensor-core convolution");
}

int CnnForward(const float* params, const CnnActivations& a, int n, cudaStream_t stream,
               bool tensor_cores, uint32_t* error) {
  if (tensor_cores) {
    int status = LaunchConvTc<kCnnInChannels>(a, params, 0, n, error, stream);
    for (int l = 1; l < 4 && status == GJXL_B200_OK; ++l)
      status = LaunchConvTc<kCnnC>(a, params, l, n, error, stream);
    if (status != GJXL_B200_OK) return status;
    const size_t cells = static_cast<size_t>(n) * 64;
    HeadForwardKernel<<<static_cast<unsigned>((cells + 127) / 128), 128, 0, stream>>>(
      a.act[4], params, n, a.head);
    return CheckLaunch("cnn forward");
  }
  for (int l = 0; l < 4; ++l) {
    const LayerShape L = Layer(l);
    const size_t pixels = static_cast<size_t>(n) * L.out_size * L.out_size;
    const unsigned grid = static_cast<unsigned>((pixels + 127) / 128);
    if (l == 0) {
      ConvForwardKernel<kCnnInChannels><<<grid, 128, 0, stream>>>(a.act[0], params, 0, n,
                                                                  a.act[1]);
    } else {
      ConvForwardKernel<kCnnC><<<grid, 128, 0, stream>>>(a.act[l], params, l, n, a.act[l + 1]);
    }
  }
  const size_t cells = static_cast<size_t>(n) * 64;
  HeadForwardKernel<<<static_cast<unsigned>((cells + 127) / 128), 128, 0, stream>>>(
    a.act[4], params, n, a.head);
  return CheckLaunch("cnn forward");
}

int CnnPropose(const float* head, int n, size_t blocks_x, size_t blocks_y, uint8_t* proposals,
               float* confidence, float* log_scale, cudaStream_t stream) {
  const size_t cells = static_cast<size_t>(n) * 64;
  ProposeKernel<<<static_cast<unsigned>((cells + 127) / 128), 128, 0, stream>>>(
    head, n, static_cast<int>((blocks_x + 7) / 8), static_cast<int>(blocks_x),
    static_cast<int>(blocks_y), proposals, confidence, log_scale);
  return CheckLaunch("cnn propose");
}

size_t CnnTrainScratchBytes(int n) {
  // dhead, two gradient planes of the largest activation, partials.
  const size_t dhead = static_cast<size_t>(n) * 64 * kCnnHead * 4;
  const size_t plane = static_cast<size_t>(n) * 40 * 40 * kCnnC * 4;
  const size_t l1_chunks = (static_cast<size_t>(n) * 40 * 40 + kConvChunk - 1) / kConvChunk;
  const size_t partial = l1_chunks * (kCnnC * 9 * kCnnC + kCnnC) * 4;
  const size_t loss = ((static_cast<size_t>(n) * 64 + 255) / 256 + 1) * 4;
  return Align(dhead, 256) + 2 * Align(plane, 256) + Align(partial, 256) + Align(loss, 256);
}

int CnnTrainStep(const float* params, const CnnActivations& a, int n, const uint8_t* labels,
                 const float* targets, const float* weights, float qf_weight, float* grads,
                 void* scratch, float* loss, cudaStream_t stream) {
  unsigned char* p = static_cast<unsigned char*>(scratch);
  float* dhead = reinterpret_cast<float*>(p);
  p += Align(static_cast<size_t>(n) * 64 * kCnnHead * 4, 256);
  const size_t plane = static_cast<size_t>(n) * 40 * 40 * kCnnC * 4;
  float* g0 = reinterpret_cast<float*>(p);
  p += Align(plane, 256);
  float* g1 = reinterpret_cast<float*>(p);
  p += Align(plane, 256);
  const size_t l1_chunks = (static_cast<size_t>(n) * 40 * 40 + kConvChunk - 1) / kConvChunk;
  float* partial = reinterpret_cast<float*>(p);
  p += Align(l1_chunks * (kCnnC * 9 * kCnnC + kCnnC) * 4, 256);
  float* loss_partial = reinterpret_cast<float*>(p);

  const size_t cells = static_cast<size_t>(n) * 64;
  const unsigned loss_blocks = static_cast<unsigned>((cells + 255) / 256);
  LossKernel<<<loss_blocks, 256, 0, stream>>>(a.head, labels, targets, weights, n, qf_weight,
                                              dhead, loss_partial);
  LossReduceKernel<<<1, 1, 0, stream>>>(loss_partial, static_cast<int>(loss_blocks), n, loss);
  // Head.
  const unsigned head_chunks = static_cast<unsigned>((cells + kHeadChunk - 1) / kHeadChunk);
  HeadBackwardWeightKernel<<<head_chunks, kCnnHead * (kCnnC + 1), 0, stream>>>(dhead, a.act[4],
                                                                                n, partial);
  // Partials are [chunk][k][c + bias]; reduce, then scatter into Wh / bh.
  ReducePartialsKernel<<<(kCnnHead * (kCnnC + 1) + 127) / 128, 128, 0, stream>>>(
    partial, static_cast<int>(head_chunks), kCnnHead * (kCnnC + 1), g1);
  // g1 holds [k][c | bias]; scatter into the parameter layout.
  HeadGradScatterKernel<<<(kCnnHead * (kCnnC + 1) + 127) / 128, 128, 0, stream>>>(g1, grads);
  HeadBackwardInputKernel<<<static_cast<unsigned>((static_cast<size_t>(n) * 100 + 127) / 128),
                            128, 0, stream>>>(dhead, params, n, g0);
  // Convolutions, last to first. g_in holds dL/d(output of layer l).
  float* g_in = g0;
  float* g_out = g1;
  for (int l = 3; l >= 0; --l) {
    const LayerShape L = Layer(l);
    const size_t out_pixels = static_cast<size_t>(n) * L.out_size * L.out_size;
    const unsigned chunks = static_cast<unsigned>((out_pixels + kConvChunk - 1) / kConvChunk);
    const int patch = 9 * L.cin;
    if (l == 0) {
      ConvBackwardWeightKernel<kCnnInChannels><<<chunks, 256, 0, stream>>>(
        g_in, a.act[1], a.act[0], 0, n, partial);
    } else {
      ConvBackwardWeightKernel<kCnnC><<<chunks, 256, 0, stream>>>(g_in, a.act[l + 1], a.act[l],
                                                                  l, n, partial);
    }
    // Partials are [chunk][co * patch + e | 32 biases]: W then b, contiguous
    // in the parameter layout.
    const int width = kCnnC * patch + kCnnC;
    ReducePartialsKernel<<<(width + 127) / 128, 128, 0, stream>>>(partial, static_cast<int>(chunks),
                                                                  width, grads + L.w_offset);
    if (l > 0) {
      const size_t in_pixels = static_cast<size_t>(n) * L.in_size * L.in_size;
      ConvBackwardInputKernel<kCnnC><<<static_cast<unsigned>((in_pixels + 127) / 128), 128, 0,
                                       stream>>>(g_in, a.act[l + 1], params, l, n, g_out);
      float* t = g_in;
      g_in = g_out;
      g_out = t;
    }
  }
  return CheckLaunch("cnn train step");
}

int CnnAdamW(float* params, const float* grads, float* m, float* v, int step, float lr,
             float beta1, float beta2, float eps, float weight_decay, cudaStream_t stream) {
  const float bias1 = 1.0f - std::pow(beta1, static_cast<float>(step));
  const float bias2 = 1.0f - std::pow(beta2, static_cast<float>(step));
  AdamWKernel<<<(kCnnParams + 255) / 256, 256, 0, stream>>>(params, grads, m, v, kCnnParams, lr,
                                                            beta1, beta2, eps, weight_decay, bias1,
                                                            bias2);
  return CheckLaunch("cnn adamw");
}

}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" size_t gjxl_b200_cnn_param_count(void) { return kCnnParams; }
extern "C" size_t gjxl_b200_cnn_workspace_bytes(int tiles) {
  return tiles > 0 ? CnnWorkspaceBytes(tiles) : 0;
}
extern "C" size_t gjxl_b200_cnn_train_scratch_bytes(int tiles) {
  return tiles > 0 ? CnnTrainScratchBytes(tiles) : 0;
}

extern "C" int gjxl_b200_cnn_gather(const float* opsin, size_t opsin_stride,
                                    size_t opsin_plane_pitch, size_t padded_width,
                                    size_t padded_height, const int* tile_list, int tiles,
                                    float distance, void* workspace, void* stream) {
  ClearLastError();
  if (opsin == nullptr || workspace == nullptr || tiles <= 0 || padded_width % 8 ||
      padded_height % 8 || padded_width == 0 || padded_height == 0 ||
      opsin_stride < padded_width || !(distance > 0.0f)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "cnn_gather: invalid arguments");
  }
  const CnnActivations a = CnnLayout(workspace, tiles);
  return CnnGather(opsin, opsin_stride, opsin_plane_pitch, padded_width, padded_height,
                   tile_list, tiles, distance, a.act[0], static_cast<cudaStream_t>(stream));
}

extern "C" int gjxl_b200_cnn_forward(const float* params, int tiles, void* workspace,
                                     float* head_out, int tensor_cores, void* stream) {
  ClearLastError();
  if (params == nullptr || workspace == nullptr || tiles <= 0) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "cnn_forward: invalid arguments");
  }
  const CnnActivations a = CnnLayout(workspace, tiles);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  int status = CnnForward(params, a, tiles, s, tensor_cores != 0, nullptr);
  if (status == GJXL_B200_OK && head_out != nullptr) {
    status = CheckCuda(cudaMemcpyAsync(head_out, a.head,
                                       static_cast<size_t>(tiles) * 64 * kCnnHead * 4,
                                       cudaMemcpyDeviceToDevice, s),
                       "cnn_forward: head copy");
  }
  return status;
}

extern "C" int gjxl_b200_cnn_train_step(const float* params, int tiles, void* workspace,
                                        const uint8_t* labels, const float* targets,
                                        const float* weights, float qf_weight, float* grads,
                                        void* scratch, float* loss, void* stream) {
  ClearLastError();
  if (params == nullptr || workspace == nullptr || labels == nullptr || targets == nullptr ||
      weights == nullptr || grads == nullptr || scratch == nullptr || loss == nullptr ||
      tiles <= 0) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "cnn_train_step: invalid arguments");
  }
  const CnnActivations a = CnnLayout(workspace, tiles);
  return CnnTrainStep(params, a, tiles, labels, targets, weights, qf_weight, grads, scratch, loss,
                      static_cast<cudaStream_t>(stream));
}

extern "C" int gjxl_b200_cnn_adamw(float* params, const float* grads, float* m, float* v,
                                   int step, float lr, float beta1, float beta2, float eps,
                                   float weight_decay, void* stream) {
  ClearLastError();
  if (params == nullptr || grads == nullptr || m == nullptr || v == nullptr || step < 1) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "cnn_adamw: invalid arguments");
  }
  return CnnAdamW(params, grads, m, v, step, lr, beta1, beta2, eps, weight_decay,
                  static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------
// Learned analysis mode: per-tile family masks and the pruned cost table.

namespace gjxl_b200 {
namespace {

__device__ __forceinline__ int SearchedFamily(int s) {
  return s == 0 ? 0 : s == 6 ? 1 : s == 7 ? 2 : s == 4 ? 3 : s == 10 ? 4 : s == 11 ? 5
       : s == 5 ? 6 : -1;
}

// One thread per tile: the union of its blocks' proposed families (DCT8
// always), or every family when a block's top-3 mass is below `confidence`.
__global__ void TileMaskKernel(const uint8_t* proposals, const float* mass, int blocks_x,
                               int blocks_y, float confidence, uint8_t* masks) {
  const int tiles_x = (blocks_x + 7) / 8, tiles_y = (blocks_y + 7) / 8;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= tiles_x * tiles_y) return;
  const int bx0 = (t % tiles_x) * 8, by0 = (t / tiles_x) * 8;
  uint32_t mask = 1u;
  bool fallback = false;
  for (int y = by0; y < min(by0 + 8, blocks_y); ++y) {
    for (int x = bx0; x < min(bx0 + 8, blocks_x); ++x) {
      const size_t b = static_cast<size_t>(y) * blocks_x + x;
      if (mass[b] < confidence) fallback = true;
      for (int r = 0; r < 3; ++r) {
        const int f = SearchedFamily(proposals[3 * b + r]);
        if (f >= 0) mask |= 1u << f;
      }
    }
  }
  masks[t] = static_cast<uint8_t>(fallback ? 0x7fu : mask);
}

// Anchors of families outside their tile's mask get the largest finite
// cost, so the greedy merge never takes them.
__global__ void MaskCostsKernel(float* costs, const uint8_t* masks, int blocks_x, int blocks_y) {
  const size_t blocks = static_cast<size_t>(blocks_x) * blocks_y;
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 7 * blocks) return;
  const int f = static_cast<int>(i / blocks);
  const size_t b = i % blocks;
  const int bx = static_cast<int>(b % blocks_x), by = static_cast<int>(b / blocks_x);
  const int tiles_x = (blocks_x + 7) / 8;
  if (!(masks[(by / 8) * tiles_x + bx / 8] & (1u << f))) costs[i] = 3.402823466e38f;
}

// Per family, the tiles whose mask keeps it (in no particular order; each
// candidate's cost is independent of the others).
__global__ void KeptTilesKernel(const uint8_t* masks, int tiles, uint32_t* kept,
                                uint32_t* counts) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= tiles) return;
  for (int f = 0; f < 7; ++f) {
    if (masks[t] & (1u << f)) kept[static_cast<size_t>(f) * tiles + atomicAdd(&counts[f], 1u)] = t;
  }
}

__global__ void ScaleFieldKernel(float* field, const float* log_scale, size_t blocks) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < blocks) field[i] *= expf(log_scale[i]);
}

}  // namespace

int CnnTileMasks(const uint8_t* proposals, const float* mass, size_t blocks_x, size_t blocks_y,
                 float confidence, uint8_t* masks, cudaStream_t stream) {
  const size_t tiles = ((blocks_x + 7) / 8) * ((blocks_y + 7) / 8);
  TileMaskKernel<<<static_cast<unsigned>((tiles + 127) / 128), 128, 0, stream>>>(
    proposals, mass, static_cast<int>(blocks_x), static_cast<int>(blocks_y), confidence, masks);
  return CheckLaunch("cnn tile masks");
}

int CnnKeptTiles(const uint8_t* masks, size_t tiles, uint32_t* kept, uint32_t* counts,
                 cudaStream_t stream) {
  int status = CheckCuda(cudaMemsetAsync(counts, 0, 8 * sizeof(uint32_t), stream),
                         "cnn kept tiles");
  if (status != GJXL_B200_OK) return status;
  KeptTilesKernel<<<static_cast<unsigned>((tiles + 127) / 128), 128, 0, stream>>>(
    masks, static_cast<int>(tiles), kept, counts);
  return CheckLaunch("cnn kept tiles");
}

int CnnMaskCosts(float* costs, const uint8_t* masks, size_t blocks_x, size_t blocks_y,
                 cudaStream_t stream) {
  const size_t n = 7 * blocks_x * blocks_y;
  MaskCostsKernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(
    costs, masks, static_cast<int>(blocks_x), static_cast<int>(blocks_y));
  return CheckLaunch("cnn mask costs");
}

int CnnScaleField(float* field, const float* log_scale, size_t blocks, cudaStream_t stream) {
  ScaleFieldKernel<<<static_cast<unsigned>((blocks + 255) / 256), 256, 0, stream>>>(
    field, log_scale, blocks);
  return CheckLaunch("cnn scale field");
}

}  // namespace gjxl_b200
