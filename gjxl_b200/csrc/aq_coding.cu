// Rows a9-a12: adaptive-quantization field adjustment, quantizer selection,
// final chroma-from-luma, per-transform AC coefficient coding and
// prediction-aware DC quantization, on the device.
//
// Restates, with the reference's exact float/double operation order:
//   AdjustQuantField            src/codec/adaptive_quantization.cpp:740-830
//   PrepareButteraugliPolicy    src/codec/adaptive_quantization.cpp:1178-1240
//   CreateQuantizerFromField    src/codec/quantization.cpp:536-620, :59-100
//   ComputeFinalColorCorrelationMap (fast)  src/codec/chroma_from_luma.cpp:543-650
//   ComputeQuantizedCoefficientsImpl        src/codec/reconstruction.cpp:386-760
//   SelectAdjustedAcQuantization / AdjustQuantForChannel /
//   QuantizeAcBlockWithThresholds           src/codec/quantization.cpp:185-480, 740-800
//   ConvertLowFrequenciesToDc               src/codec/dc_conversion.cpp:174-236
//   QuantizeDcCoefficients (prediction-aware, weighted predictor)
//                                           src/codec/vardct/dc_quantization.cpp:120-230,
//                                           src/codec/modular/prediction.h:59-150
//   ComputeEpfInverseSigma                  src/codec/epf.cpp:207-270
//
// Coefficients live in "footprint layout": the N coefficients of a transform
// anchored at block (bx, by) occupy its own W x H pixel footprint of a padded
// plane, coefficient i at (bx*8 + i % W, by*8 + i / W).

#include <algorithm>
#include <cmath>
#include <cstring>

#include "aq.h"
#include "common.cuh"
#include "dc_tokens.cuh"
#include "host_util.h"
#include "line_dct.cuh"
#include "tables.h"
#include "transform.cuh"

namespace gjxl_b200 {
namespace {

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// Anchor lists.

__global__ void AnchorListKernel(const uint8_t* cells, uint32_t blocks_x, uint32_t blocks,
                                 int2* lists, uint32_t list_stride, uint32_t* counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= blocks) return;
  const uint8_t cell = cells[i];
  if (!(cell & 1)) return;
  const int f = StrategyFamily(cell >> 1);
  if (f < 0) return;
  const uint32_t slot = atomicAdd(&counts[f], 1u);
  lists[f * list_stride + slot] = make_int2(i % blocks_x, i / blocks_x);
}

// ---------------------------------------------------------------------------
// Forward coefficients of the selected transforms (footprint layout).

// K = 1024 / N transforms (3 channels each) per CTA of 384 threads, one
// 8-output chunk of one line per thread and pass (line_dct.cuh).
constexpr int kTransformThreads = 384;

template <int W, int H>
__global__ void __launch_bounds__(kTransformThreads)
ForwardCoefficientsKernel(const float* opsin, size_t stride, size_t pitch, const int2* anchors,
                          const uint32_t* count, uint32_t capacity, float* coef,
                          size_t coef_stride, size_t coef_pitch) {
  using S = TransformShape<W, H>;
  constexpr int N = W * H, K = 1024 / N, KC = 3 * K;
  using Batch = PlaneBatch<W, H, KC>;
  static_assert(Batch::Items == kTransformThreads, "one chunk per thread and pass");
  extern __shared__ __align__(16) unsigned char smem[];
  double* tmp = reinterpret_cast<double*>(smem);                  // [KC] padded planes
  float* px = reinterpret_cast<float*>(tmp + Batch::Elements);    // [KC] padded planes
  const uint32_t first = blockIdx.x * K;
  // The anchor loads do not wait for the count: the list index is clamped to
  // the list (capacity entries), and anchors past the count are never used.
  constexpr int kPerThread = KC * N / kTransformThreads;
  int2 item_anchor[kPerThread];
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const int k = (threadIdx.x + q * kTransformThreads) / (3 * N);
    item_anchor[q] = anchors[min(first + static_cast<uint32_t>(k), capacity - 1)];
  }
  const uint32_t n = *count;
  if (first >= n) return;
  const int active = min(K, static_cast<int>(n - first));
  // All of a thread's loads are issued before the first store.
  float value[kPerThread];
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const int i = threadIdx.x + q * kTransformThreads;
    const int r = i % (3 * N), c = r / N, yx = r % N;
    const bool live = i < active * 3 * N;
    const int2 a = item_anchor[q];
    value[q] = live ? opsin[c * pitch + static_cast<size_t>(a.y * 8 + yx / W) * stride + a.x * 8 +
                            yx % W]
                    : 0.0f;
  }
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const int i = threadIdx.x + q * kTransformThreads;
    if (i >= active * 3 * N) break;
    const int k = i / (3 * N), r = i % (3 * N), c = r / N, yx = r % N;
    px[Batch::At(k * 3 + c, yx / W, yx % W)] = value[q];
  }
  __syncthreads();
  const auto present = [&](int plane) { return plane < 3 * active; };
  BatchRowPass<W, H, KC, true>(px, tmp, threadIdx.x, kTransformThreads, present);
  __syncthreads();
  BatchColumnPass<W, H, KC, true>(tmp, px, threadIdx.x, kTransformThreads, present);
  __syncthreads();
  // Coefficient j = coefficient_index(v, u) goes to footprint (j % W, j / W).
  for (int i = threadIdx.x; i < active * 3 * N; i += kTransformThreads) {
    const int k = i / (3 * N), r = i % (3 * N), c = r / N, j = r % N;
    const int v = H < W ? j / W : j % H, u = H < W ? j % W : j / H;
    const int2 a = anchors[first + k];
    coef[c * coef_pitch + static_cast<size_t>(a.y * 8 + j / W) * coef_stride + a.x * 8 + j % W] =
      px[Batch::At(k * 3 + c, v, u)];
  }
  static_assert(S::N == N, "shape");
}

// ---------------------------------------------------------------------------
// Field adjustment, policy bounds, quantizer selection.

struct AnchorView {
  const uint8_t* cells;
  int blocks_x, blocks_y;
};

__device__ __forceinline__ bool AnchorAt(const AnchorView& v, int i, int* cw, int* ch, int* s) {
  const uint8_t cell = v.cells[i];
  if (!(cell & 1)) return false;
  *s = cell >> 1;
  const int f = StrategyFamily(*s);
  *cw = FamilyCoveredW(f);
  *ch = FamilyCoveredH(f);
  return true;
}

// AdjustQuantField (adaptive_quantization.cpp:776-812) for every anchor.
__global__ void AdjustFieldKernel(AnchorView v, const float* in, float* out, float mixer) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.blocks_x * v.blocks_y) return;
  int cw, ch, s;
  if (!AnchorAt(v, i, &cw, &ch, &s)) return;
  const int bx = i % v.blocks_x, by = i / v.blocks_x;
  float maximum = in[i];
  float mean = 0.0f;
  for (int dy = 0; dy < ch; ++dy) {
    for (int dx = 0; dx < cw; ++dx) {
      const float value = in[(by + dy) * v.blocks_x + bx + dx];
      maximum = fmaxf(maximum, value);
      mean += value;
    }
  }
  const int count = cw * ch;
  mean /= static_cast<float>(count);
  float result = maximum;
  if (count >= 4) result = maximum * mixer + mean * (1.0f - mixer);
  for (int dy = 0; dy < ch; ++dy)
    for (int dx = 0; dx < cw; ++dx) out[(by + dy) * v.blocks_x + bx + dx] = result;
}

// The field is positive, so its extremes reduce as unsigned bit patterns
// from {+inf, 0}.
__global__ void RangeInitKernel(float* range) {
  range[0] = __int_as_float(0x7f800000);
  range[1] = 0.0f;
}

__global__ void RangeKernel(const float* field, int n, float* range) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float lo = __int_as_float(0x7f800000), hi = 0.0f;
  if (i < n) lo = hi = field[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(reinterpret_cast<unsigned int*>(&range[0]), __float_as_uint(lo));
    atomicMax(reinterpret_cast<unsigned int*>(&range[1]), __float_as_uint(hi));
  }
}

// PrepareButteraugliPolicyFromRange (adaptive_quantization.cpp:1205-1240).
__global__ void PolicySetupKernel(const float* range, float quant_dc, AqPolicy* policy,
                                  uint32_t* error) {
  const float lo = range[0], hi = range[1];
  const float initial_ratio = hi / lo;
  const float maximum_deviation = sqrtf(250.0f / initial_ratio);
  const float asymmetry = fminf(2.0f, maximum_deviation);
  policy->lower_bound = lo / (asymmetry * maximum_deviation);
  policy->upper_bound = hi * (maximum_deviation / asymmetry);
  policy->quant_dc = quant_dc;
  if (!(IsFinite(policy->lower_bound) && IsFinite(policy->upper_bound) &&
        policy->lower_bound > 0.0f && policy->upper_bound >= policy->lower_bound &&
        policy->upper_bound / policy->lower_bound < 253.0f)) {
    RaiseError(error, kErrorRange);
  }
}

// k-th smallest of n positive floats (or of |field - center|) by radix
// selection over the ordered bit patterns in three digit passes (bits 21-31,
// 10-20, 0-9). Each pass is a grid-wide histogram of the elements that match
// the prefix chosen so far (SelectHistogramKernel) and a one-CTA scan that
// picks the digit holding the k-th element (SelectDigitKernel). The median
// of the field is selected first, then the median absolute deviation.
constexpr int kSelectBins = 2048;
constexpr int kSelectPasses = 3;
__host__ __device__ constexpr int SelectShift(int pass) { return pass == 0 ? 21 : pass == 1 ? 10 : 0; }
__host__ __device__ constexpr int SelectBits(int pass) { return pass == 2 ? 10 : 11; }

struct SelectState {
  uint32_t prefix, mask, k;
  uint32_t median_bits, mad_bits;
  uint32_t pad[3];
  uint32_t histogram[kSelectBins];
};

__global__ void SelectInitKernel(SelectState* st, int n) {
  for (int b = threadIdx.x; b < kSelectBins; b += blockDim.x) st->histogram[b] = 0;
  if (threadIdx.x == 0) {
    st->prefix = 0;
    st->mask = 0;
    st->k = static_cast<uint32_t>(n / 2);
  }
}

__device__ __forceinline__ uint32_t SelectKey(const float* field, int i, bool use_center,
                                              float center) {
  return __float_as_uint(use_center ? fabsf(field[i] - center) : field[i]);
}

__global__ void __launch_bounds__(256)
SelectHistogramKernel(const float* field, int n, bool use_center, int pass, SelectState* st) {
  __shared__ uint32_t histogram[kSelectBins];
  for (int b = threadIdx.x; b < kSelectBins; b += blockDim.x) histogram[b] = 0;
  __syncthreads();
  const uint32_t prefix = st->prefix, mask = st->mask;
  const float center = __uint_as_float(st->median_bits);
  const int shift = SelectShift(pass);
  const uint32_t digit_mask = (1u << SelectBits(pass)) - 1u;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t bits = SelectKey(field, i, use_center, center);
    if ((bits & mask) == prefix) atomicAdd(&histogram[(bits >> shift) & digit_mask], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kSelectBins; b += blockDim.x) {
    if (histogram[b] != 0) atomicAdd(&st->histogram[b], histogram[b]);
  }
}

// One CTA of 1024 threads: inclusive scan of the histogram (two bins per
// thread), the digit whose range holds rank k, and the histogram cleared for
// the next pass. After the last pass the selected value is stored and the
// state rearmed for the next selection.
__global__ void __launch_bounds__(1024) SelectDigitKernel(int pass, int n, bool mad,
                                                          SelectState* st) {
  __shared__ uint32_t warp_sums[32];
  const int t = threadIdx.x, lane = t % 32, warp = t / 32;
  const uint32_t h0 = st->histogram[2 * t], h1 = st->histogram[2 * t + 1];
  uint32_t inclusive = h0 + h1;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, inclusive, o);
    if (lane >= o) inclusive += v;
  }
  if (lane == 31) warp_sums[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_sums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += v;
    }
    warp_sums[lane] = w;
  }
  __syncthreads();
  const uint32_t before = inclusive - (h0 + h1) + (warp ? warp_sums[warp - 1] : 0u);
  const uint32_t k = st->k;
  __syncthreads();
  const int shift = SelectShift(pass);
  const uint32_t digit_mask = (1u << SelectBits(pass)) - 1u;
  // Exactly one (thread, bin) has before_bin <= k < before_bin + count.
  if (k >= before && k < before + h0) {
    st->prefix |= static_cast<uint32_t>(2 * t) << shift;
    st->k = k - before;
  } else if (k >= before + h0 && k < before + h0 + h1) {
    st->prefix |= static_cast<uint32_t>(2 * t + 1) << shift;
    st->k = k - before - h0;
  }
  st->histogram[2 * t] = 0;
  st->histogram[2 * t + 1] = 0;
  __syncthreads();
  if (t == 0) {
    st->mask |= digit_mask << shift;
    if (pass == kSelectPasses - 1) {
      if (mad) {
        st->mad_bits = st->prefix;
      } else {
        st->median_bits = st->prefix;
      }
      st->prefix = 0;
      st->mask = 0;
      st->k = static_cast<uint32_t>(n / 2);
    }
  }
}

// CreateQuantizerFromField + ComputeQuantizerParams + Quantizer::Create.
__global__ void QuantizerKernel(const SelectState* st, const AqPolicy* policy, AqQuantizer* q,
                                uint32_t* error) {
  const float median = __uint_as_float(st->median_bits);
  const float mad = __uint_as_float(st->mad_bits);
  const float quant_dc = policy->quant_dc;
  float scale = 65536.0f * (median - mad) / 5.0f;
  scale = fminf(fmaxf(scale, 1.0f), 32768.0f);
  int global_scale = static_cast<int>(scale);
  const int scaled_quant_dc = static_cast<int>(static_cast<double>(quant_dc * 4096.0f) * 1.6);
  if (global_scale > scaled_quant_dc) global_scale = max(1, scaled_quant_dc);
  const float inverse_global_scale = 65536.0f / static_cast<float>(global_scale);
  const float quant_dc_value = fminf(65536.0f, quant_dc * inverse_global_scale + 0.5f);
  const uint32_t qdc = static_cast<uint32_t>(quant_dc_value);
  q->global_scale = static_cast<uint32_t>(global_scale);
  q->quant_dc = qdc;
  if (global_scale < 1 || global_scale > 32768 || qdc == 0 || qdc > 65536) {
    RaiseError(error, kErrorRange);
  }
  q->scale = static_cast<float>(global_scale) / 65536.0f;
  q->inverse_global_scale = 65536.0f / static_cast<float>(global_scale);
  const float inverse_quant_dc = q->inverse_global_scale / static_cast<float>(qdc);
  const float kInverseDcQuant[3] = {4096.0f, 512.0f, 256.0f};
  for (int c = 0; c < 3; ++c) {
    q->dc_steps[c] = inverse_quant_dc / kInverseDcQuant[c];
    q->inverse_dc_steps[c] = kInverseDcQuant[c] * q->scale * static_cast<float>(qdc);
  }
}

__global__ void RawQuantKernel(const float* field, int n, const AqQuantizer* q, int32_t* raw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = field[i] * q->inverse_global_scale + 0.5f;
  raw[i] = static_cast<int32_t>(fminf(fmaxf(v, 1.0f), 256.0f));
}

// ---------------------------------------------------------------------------
// Final CfL, fast regression (one CTA per 64x64 tile; lane i of the solving
// lanes owns elements i (mod 4) in the reference's order: anchors in raster
// order, coefficients in storage order).

struct CflFinalParams {
  AnchorView grid;
  int tiles_x, tiles_y;
  const float* coef;  // footprint layout, 3 planes
  size_t coef_stride, coef_pitch;
  const int32_t* raw;
  const AqQuantizer* q;
  const float* inverse_dequant;  // packed tables
  size_t table_offset[kTableCount];
  size_t table_count[kTableCount];
  int8_t* y_to_x;
  int8_t* y_to_b;
};

__device__ __forceinline__ int8_t QuantizeMultiplierF(float x) {
  if (x >= 2.6f) {
    x -= 2.6f;
  } else if (x <= -2.6f) {
    x += 2.6f;
  } else {
    x = 0.0f;
  }
  return static_cast<int8_t>(fminf(fmaxf(roundf(x), -128.0f), 127.0f));
}

// Per tile, all threads first write the regression terms a = luma / 84 and
// b = base * luma - chroma of both problems into shared memory in the
// reference's element order (anchors in raster order, coefficients in
// storage order); then lanes 0-3 (y_to_x) and 4-7 (y_to_b) of warp 0 run the
// four ordered fused multiply-add chains per problem from shared memory.
constexpr int kFinalCflThreads = 128;
constexpr int kFinalCflTerms = 64 * 64;  // coefficients of one 64x64 tile

__global__ void __launch_bounds__(kFinalCflThreads)
FinalCflKernel(const __grid_constant__ CflFinalParams p) {
  extern __shared__ __align__(16) float terms[];  // [a_x, b_x, a_b, b_b][kFinalCflTerms]
  __shared__ int block_terms[64], offsets[64], total_terms;
  __shared__ uint8_t group_block[64];  // anchor block of each 64-term group
  // Per anchor block: covered width and height, inverse-dequant table
  // offset, and the quantization scale of its raw quant.
  __shared__ uint8_t block_cw[64], block_ch[64];
  __shared__ uint8_t block_w_shift[64], block_sw_shift[64];  // log2 of 8 * cw, 8 * max(cw, ch)
  __shared__ int block_table[64];
  __shared__ float block_scale[64];
  const int tile = blockIdx.x;
  const int tx = tile % p.tiles_x, ty = tile / p.tiles_x;
  const int bx0 = tx * 8, by0 = ty * 8;
  const int tw = min(8, p.grid.blocks_x - bx0), th = min(8, p.grid.blocks_y - by0);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x < 64) {
    int n = 0, cw = 1, ch = 1, s = kStrategyDct8;
    const int b = threadIdx.x;
    if (b < tw * th) {
      const int block = (by0 + b / tw) * p.grid.blocks_x + bx0 + b % tw;
      if (AnchorAt(p.grid, block, &cw, &ch, &s)) {
        n = cw * ch * 64;
        const int table = s == kStrategyDct8 ? kTableDct8 : s == kStrategyDct16x16 ? kTableDct16
                        : s == kStrategyDct32x32 ? kTableDct32
                        : (s == kStrategyDct16x8 || s == kStrategyDct8x16) ? kTableDct8x16
                                                                             : kTableDct16x32;
        block_table[b] = static_cast<int>(p.table_offset[table]);
        block_scale[b] = p.q->scale * 128.0f * static_cast<float>(p.raw[block]);
      }
    }
    block_cw[b] = static_cast<uint8_t>(cw);
    block_ch[b] = static_cast<uint8_t>(ch);
    block_w_shift[b] = static_cast<uint8_t>(3 + __ffs(cw) - 1);  // cw, ch are 1, 2 or 4
    block_sw_shift[b] = static_cast<uint8_t>(3 + __ffs(cw >= ch ? cw : ch) - 1);
    block_terms[b] = n;
  }
  __syncthreads();
  // Exclusive prefix sum of the blocks' term counts (64 blocks, two warps:
  // a shuffle scan per warp, then warp 0's total added to warp 1), and the
  // anchor block of each 64-term group.
  __shared__ int warp_total[2];
  if (threadIdx.x < 64) {
    const int b = threadIdx.x;
    const int n = block_terms[b];
    int inclusive = n;
#pragma unroll
    for (int d = 1; d < 32; d *= 2) {
      const int v = __shfl_up_sync(0xffffffffu, inclusive, d);
      if (lane >= d) inclusive += v;
    }
    offsets[b] = inclusive - n;
    if (lane == 31) warp_total[warp] = inclusive;
  }
  __syncthreads();
  if (threadIdx.x < 64) {
    const int b = threadIdx.x;
    const int n = block_terms[b];
    const int offset = offsets[b] + (b >= 32 ? warp_total[0] : 0);
    offsets[b] = offset;
    for (int g = offset / 64; g < (offset + n) / 64; ++g) group_block[g] = static_cast<uint8_t>(b);
    if (b == 63) total_terms = offset + n;
  }
  __syncthreads();
  // Every thread takes terms e = tid, tid + 128, ... of the tile; every
  // anchor's term count is a multiple of 64, so term e belongs to the anchor
  // of group e / 64. Batches of kBatch terms: all their global loads are
  // issued before the first term is computed.
  constexpr int kBatch = 8;
  const int count = total_terms;
  for (int e0 = threadIdx.x; e0 < count; e0 += kBatch * kFinalCflThreads) {
    float luma_v[kBatch], x_v[kBatch], b_v[kBatch], inv_x[kBatch], inv_b[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      const int e = e0 + j * kFinalCflThreads;
      luma_v[j] = x_v[j] = b_v[j] = inv_x[j] = inv_b[j] = 0.0f;
      if (e >= count) continue;
      const int b = group_block[e / 64], i = e - offsets[b];
      const int cw = block_cw[b], ch = block_ch[b];
      const int w_shift = block_w_shift[b], sw_shift = block_sw_shift[b];
      // LLF extent: covered blocks with the longer side first; the
      // coefficient extent is 8 * max(cw, ch) wide.
      const int lfw = cw > ch ? cw : ch, lfh = cw > ch ? ch : cw;
      const int cy = i >> sw_shift, cx = i & ((1 << sw_shift) - 1);
      const bool llf = cy < lfh && cx < lfw;
      const float* inv = p.inverse_dequant + block_table[b];
      inv_x[j] = inv[i];
      inv_b[j] = inv[2 * cw * ch * 64 + i];
      if (!llf) {
        const size_t at =
          static_cast<size_t>((by0 + b / tw) * 8 + (i >> w_shift)) * p.coef_stride +
          (bx0 + b % tw) * 8 + (i & ((1 << w_shift) - 1));
        luma_v[j] = p.coef[p.coef_pitch + at];
        x_v[j] = p.coef[at];
        b_v[j] = p.coef[2 * p.coef_pitch + at];
      }
    }
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      const int e = e0 + j * kFinalCflThreads;
      if (e >= count) continue;
      const float quant_scale = block_scale[group_block[e / 64]];
      const float base_x = 0.0f, base_b = 1.0f;
      const float luma_x = luma_v[j] * inv_x[j] * quant_scale;
      const float chroma_x = x_v[j] * inv_x[j] * quant_scale;
      const float luma_b = luma_v[j] * inv_b[j] * quant_scale;
      const float chroma_b = b_v[j] * inv_b[j] * quant_scale;
      terms[e] = luma_x / 84.0f;
      terms[kFinalCflTerms + e] = base_x * luma_x - chroma_x;
      terms[2 * kFinalCflTerms + e] = luma_b / 84.0f;
      terms[3 * kFinalCflTerms + e] = base_b * luma_b - chroma_b;
    }
  }
  __syncthreads();
  if (warp != 0) return;
  const int problem = lane / 4, slot = lane % 4;  // problem 0: X, 1: B
  float quadratic = 0.0f, linear = 0.0f;
  if (problem < 2) {
    const float* A = terms + 2 * problem * kFinalCflTerms;
    const float* B = A + kFinalCflTerms;
    // count is a multiple of 64: batches of 8 elements per lane; the next
    // batch is loaded while the current one goes through the ordered
    // multiply-adds.
    float a[8], b[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      a[j] = count > 0 ? A[slot + 4 * j] : 0.0f;
      b[j] = count > 0 ? B[slot + 4 * j] : 0.0f;
    }
    for (int e0 = slot; e0 < count; e0 += 32) {
      float na[8], nb[8];
      const int next = e0 + 32 < count ? e0 + 32 : slot;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        na[j] = A[next + 4 * j];
        nb[j] = B[next + 4 * j];
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        quadratic = fmaf(a[j], a[j], quadratic);
        linear = fmaf(a[j], b[j], linear);
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        a[j] = na[j];
        b[j] = nb[j];
      }
    }
  }
  const int base_lane = 4 * (problem < 2 ? problem : 0);
  const float q0 = __shfl_sync(0xffffffffu, quadratic, base_lane + 0);
  const float q1 = __shfl_sync(0xffffffffu, quadratic, base_lane + 1);
  const float q2 = __shfl_sync(0xffffffffu, quadratic, base_lane + 2);
  const float q3 = __shfl_sync(0xffffffffu, quadratic, base_lane + 3);
  const float l0 = __shfl_sync(0xffffffffu, linear, base_lane + 0);
  const float l1 = __shfl_sync(0xffffffffu, linear, base_lane + 1);
  const float l2 = __shfl_sync(0xffffffffu, linear, base_lane + 2);
  const float l3 = __shfl_sync(0xffffffffu, linear, base_lane + 3);
  if (slot == 0 && problem < 2) {
    int8_t result = 0;
    if (count > 0) {
      const float x = -((l0 + l1) + (l2 + l3)) /
                      (((q0 + q1) + (q2 + q3)) +
                       static_cast<float>(count) * 1.0e-9f * 0.5f);
      result = QuantizeMultiplierF(x);
    }
    (problem == 0 ? p.y_to_x : p.y_to_b)[tile] = result;
  }
}

// ---------------------------------------------------------------------------
// Coefficient coding (one CTA per anchor).

struct DcTables {
  // Inverse / forward LLF bases for lengths 1, 2, 4: [len][freq][sample].
  double inverse[3][4][4];
  double forward[3][4][4];
  float downsample[3][4];
  float upsample[3][4];
};
__constant__ DcTables c_dc_tables;

__device__ __forceinline__ int LenIndex(int len) { return len == 1 ? 0 : len == 2 ? 1 : 2; }

// QuantizationThresholds for X/B (quantization.cpp:185-201).
__device__ __forceinline__ void ChromaThresholds(int covered, float t[4]) {
  t[0] = 0.58f;
  t[1] = t[2] = t[3] = 0.62f;
  if (covered >= 4) {
    for (int i = 0; i < 4; ++i) t[i] = fmaxf(0.5f, t[i] - 0.00744f * static_cast<float>(covered));
  }
}

// AdjustQuantForChannel (quantization.cpp:285-480) for one channel, in two
// parts: the sums over the coefficients, and the decisions taken from them.
struct AdjustSums {
  float border_sum, error_sum, value_sum;
  float nonzeros[4], max_error[4];
};

// Initial thresholds of a channel: the reference's defaults, lowered for
// multi-block transforms.
template <int W, int H>
__device__ __forceinline__ void AdjustThresholds(float thresholds[4]) {
  using S = TransformShape<W, H>;
  constexpr int xsize = S::SW / 8, ysize = S::SH / 8;
  thresholds[0] = 0.58f;
  thresholds[1] = thresholds[2] = thresholds[3] = 0.64f;
  if (xsize > 1 || ysize > 1) {
    const float reduction = fminf(fmaxf(0.003f * static_cast<float>(xsize * ysize), 0.0f), 0.08f);
    for (int i = 0; i < 4; ++i) thresholds[i] = fmaxf(0.54f, thresholds[i] - reduction);
  }
}

// The sums, on one thread over the coefficients in storage order.
template <int W, int H>
__device__ void AdjustSumsSerial(float qac, int channel, float mm, const float* coef,
                                 const float* inv, const float thresholds[4], AdjustSums* out) {
  using S = TransformShape<W, H>;
  const int xsize = S::SW / 8, ysize = S::SH / 8;
  float border_sum = 0.0f, error_sum = 0.0f, value_sum = 0.0f;
  float nonzeros[4] = {0, 0, 0, 0}, max_error[4] = {0, 0, 0, 0};
  for (int y = 0; y < S::SH; ++y) {
    for (int x = 0; x < S::SW; ++x) {
      const int index = y * S::SW + x;
      if (x < xsize && y < ysize) continue;
      const int quadrant = (y >= S::SH / 2) * 2 + (x >= S::SW / 2);
      const float value = coef[index] * (inv[index] * qac * mm);
      const float quantized = fabsf(value) < thresholds[quadrant] ? 0.0f : rintf(value);
      const float err = fabsf(value - quantized);
      error_sum += err;
      value_sum += fabsf(quantized);
      if (channel == 1 && quantized == 0.0f) max_error[quadrant] = fmaxf(max_error[quadrant], err);
      if (quantized != 0.0f) {
        nonzeros[quadrant] += fabsf(quantized);
        const bool in_corner = y >= 7 * ysize && x >= 7 * xsize;
        const bool on_border = y + 1 == S::SH || x + 1 == S::SW;
        const bool in_larger_corner = x >= 4 * xsize && y >= 4 * ysize;
        if (in_corner || (on_border && in_larger_corner)) border_sum += fabsf(value);
      }
    }
  }
  out->border_sum = border_sum;
  out->error_sum = error_sum;
  out->value_sum = value_sum;
  for (int i = 0; i < 4; ++i) {
    out->nonzeros[i] = nonzeros[i];
    out->max_error[i] = max_error[i];
  }
}

// The decisions: raw quant and thresholds from the sums.
template <int W, int H>
__device__ void AdjustFinish(int channel, int strategy, const AdjustSums& sums,
                             float thresholds[4], int* raw_quant) {
  using S = TransformShape<W, H>;
  const int xsize = S::SW / 8, ysize = S::SH / 8;
  float border_sum = sums.border_sum, error_sum = sums.error_sum, value_sum = sums.value_sum;
  float nonzeros[4], max_error[4];
  for (int i = 0; i < 4; ++i) {
    nonzeros[i] = sums.nonzeros[i];
    max_error[i] = sums.max_error[i];
  }
  if (channel == 1 && value_sum * 8.0f < static_cast<float>(xsize * ysize)) {
    const double kLimit = 0.46, kMultiplier = 0.9999;
    const int original = *raw_quant;
    int new_quant = *raw_quant;
    for (int quadrant = 1; quadrant < 4; ++quadrant) {
      if (nonzeros[quadrant] == 0.0f && max_error[quadrant] > kLimit) {
        new_quant = original + 1;
        break;
      }
    }
    *raw_quant = new_quant;
    if (nonzeros[3] == 0.0f && max_error[3] > kLimit) {
      thresholds[3] =
        static_cast<float>(kMultiplier * max_error[3] * new_quant / original);
    } else if ((nonzeros[1] == 0.0f && max_error[1] > kLimit) ||
               (nonzeros[2] == 0.0f && max_error[2] > kLimit)) {
      thresholds[1] = static_cast<float>(kMultiplier * fmaxf(max_error[1], max_error[2]) *
                                         new_quant / original);
      thresholds[2] = thresholds[1];
    } else if (nonzeros[0] == 0.0f && max_error[0] > kLimit) {
      thresholds[0] =
        static_cast<float>(kMultiplier * max_error[0] * new_quant / original);
    }
  }
  const float all_nonzeros = nonzeros[0] + nonzeros[1] + nonzeros[2] + nonzeros[3] + 1.0f;
  const float kBorderMultiplier = channel == 0 ? 70.0f : channel == 1 ? 30.0f : 60.0f;
  if (kBorderMultiplier * border_sum >= all_nonzeros) {
    *raw_quant = static_cast<int>(static_cast<float>(*raw_quant) +
                                  kBorderMultiplier * border_sum / all_nonzeros);
    if (*raw_quant >= 256) *raw_quant = 255;
  }
  if (strategy == kStrategyDct8 &&
      nonzeros[0] + nonzeros[1] + nonzeros[2] + nonzeros[3] < 11.0f) {
    ++*raw_quant;
    if (*raw_quant >= 256) *raw_quant = 255;
  }
  const double kFirst[4][3] = {
    {0.22080615753848404, 0.45797479824262011, 0.29859235095977965},
    {0.70109486510286834, 0.16185281305512639, 0.14387691730035473},
    {0.114985964456218638, 0.44656840441027695, 0.10587658215149048},
    {0.46849665264409396, 0.41239077937781954, 0.088667407767185444}};
  const double kSecond[4][3] = {
    {0.27450281941822197, 1.1255766549984996, 0.98950459134128388},
    {0.4652168675598285, 0.40945807983455818, 0.36581899811751367},
    {0.28034972424715715, 0.9182653201929738, 1.5581531543057416},
    {0.26873118114033728, 0.68863712390392484, 1.2082185408666786}};
  const double kQuantNormalizer = 2.2942708343284721;
  error_sum = static_cast<float>(static_cast<double>(error_sum) * kQuantNormalizer);
  value_sum = static_cast<float>(static_cast<double>(value_sum) * kQuantNormalizer);
  if (strategy >= kStrategyDct16x16) {
    int cls = 3;
    if (strategy == kStrategyDct32x16 || strategy == kStrategyDct16x32) {
      cls = 1;
    } else if (strategy == kStrategyDct16x16) {
      cls = 0;
    } else if (strategy == kStrategyDct32x32) {
      cls = 2;
    }
    const double threshold =
      kFirst[cls][channel] * static_cast<double>(xsize) * static_cast<double>(ysize) * 8.0 * 8.0 +
      kSecond[cls][channel] * static_cast<double>(value_sum);
    int step = static_cast<int>(static_cast<double>(error_sum) / threshold);
    step = min(max(step, 0), 2);
    if (static_cast<double>(error_sum) > threshold) {
      *raw_quant += step;
      if (*raw_quant >= 256) *raw_quant = 255;
    }
  }
  const int divisor = xsize * ysize;
  const float minimum = fminf(fminf(nonzeros[0], nonzeros[1]), fminf(nonzeros[2], nonzeros[3]));
  int activity = 15;
  if (minimum < 15.0f * static_cast<float>(divisor)) {
    activity = (static_cast<int>(minimum) + divisor / 2) / divisor;
  }
  int adjusted = *raw_quant - activity;
  if (channel == 1) {
    for (int quadrant = 1; quadrant < 4; ++quadrant)
      thresholds[quadrant] += 0.01f * static_cast<float>(activity);
  }
  const int limit = max(4, *raw_quant / 2);
  if (adjusted < limit) adjusted = limit;
  *raw_quant = adjusted;
}

// ConvertLowFrequenciesToDc (dc_conversion.cpp:174-236) of one channel.
template <int W, int H>
__device__ void LowFrequenciesToDc(const float* coef, float* out) {
  using S = TransformShape<W, H>;
  constexpr int CW = S::CW, CH = S::CH;
  const int lh = LenIndex(CH), lw = LenIndex(CW);
  double scaled[16];
  for (int v = 0; v < CH; ++v) {
    for (int u = 0; u < CW; ++u) {
      const int small = CH < CW ? v * CW + u : u * CH + v;
      scaled[small] = static_cast<double>(coef[S::Index(v, u)]) *
                      static_cast<double>(c_dc_tables.downsample[lh][v]) *
                      static_cast<double>(c_dc_tables.downsample[lw][u]);
    }
  }
  for (int y = 0; y < CH; ++y) {
    for (int x = 0; x < CW; ++x) {
      double value = 0.0;
      for (int v = 0; v < CH; ++v) {
        for (int u = 0; u < CW; ++u) {
          const int small = CH < CW ? v * CW + u : u * CH + v;
          value += scaled[small] * c_dc_tables.inverse[lh][v][y] * c_dc_tables.inverse[lw][u][x];
        }
      }
      out[y * CW + x] = static_cast<float>(value);
    }
  }
}

// AdjustQuantizationBias (quantization.cpp:203-218).
__device__ __forceinline__ float QuantBias(int32_t quantized, int channel) {
  const float kBias[4] = {1.0f - 0.05465007330715401f, 1.0f - 0.07005449891748593f,
                          1.0f - 0.049935103337343655f, 0.145f};
  const float value = static_cast<float>(quantized);
  const float absolute = fabsf(value);
  if (absolute < 0.125f) return 0.0f;
  if (absolute < 1.125f) return copysignf(kBias[channel], value);
  return value - kBias[3] / value;
}


struct CodingParams {
  const int2* anchors;
  const uint32_t* count;
  int blocks_x;
  size_t dc_pitch;    // blocks per DC plane
  const float* coef;  // forward coefficients, footprint layout
  size_t stride, pitch;
  int32_t* qac;       // quantized AC, footprint layout
  float* dc;          // 3 planes of blocks: extracted DC
  int32_t* raw;       // raw quant field (the anchor's entry is updated)
  const AqQuantizer* q;
  const int8_t* y_to_x;
  const int8_t* y_to_b;
  int tiles_x;
  const float* dequant;          // this family's table, [3][N]
  const float* inverse_dequant;  // this family's table, [3][N]
  const float* matrix_multiplier;  // device, X / Y / B
  uint32_t* error;
};

// ComputeQuantizedCoefficientsImpl's per-transform body
// (reconstruction.cpp:480-700), one CTA of 64 threads per anchor.
// Threads per anchor.
template <int W, int H>
__host__ __device__ constexpr int CodingThreads() {
  return 64;
}

template <int W, int H>
__global__ void __launch_bounds__(CodingThreads<W, H>()) CodingKernel(const __grid_constant__ CodingParams p) {
  using S = TransformShape<W, H>;
  constexpr int N = S::N;
  constexpr int strategy = W == 8 && H == 8     ? kStrategyDct8
                         : W == 16 && H == 16   ? kStrategyDct16x16
                         : W == 32 && H == 32   ? kStrategyDct32x32
                         : W == 8               ? kStrategyDct16x8
                         : H == 8               ? kStrategyDct8x16
                         : W == 16              ? kStrategyDct32x16
                                                : kStrategyDct16x32;
  constexpr int covered = S::CW * S::CH;
  constexpr int kT = CodingThreads<W, H>();
  __shared__ float coef[3][N];
  // The family's inverse-dequant weights, staged so that the serial
  // threshold passes below read shared memory instead of waiting on L2.
  __shared__ float inverse_dequant[3][N];
  __shared__ float thresholds[3][4];
  __shared__ int candidates[3];
  __shared__ float adjust_err[3][N];   // per coefficient |value - quantized|, 0 on the LLF
  __shared__ uint32_t adjust_sum[2][3][5];  // per warp and channel: sum |q|, per quadrant
  __shared__ uint32_t adjust_max[2][4];     // per warp: Y max error per quadrant (float bits)
  __shared__ int adjust_big[2];             // per warp: a |q| sum reached 2^24
  __shared__ float dequant_y[N];            // the family's Y dequant weights
  static_assert(kT == 64, "two warps");
  const uint32_t anchor_index = blockIdx.x;
  // The grid is the anchor list's capacity, so the anchor load is in bounds;
  // it is issued beside the count load instead of after it.
  const int2 a = p.anchors[anchor_index];
  if (anchor_index >= *p.count) return;
  const int tid = threadIdx.x;
  // Every global value the CTA reads is requested here, before the first
  // barrier (loads are not moved across barriers), so that one round trip
  // covers them all.
  const AqQuantizer q = *p.q;
  const int anchor_block = a.y * p.blocks_x + a.x;
  const int initial_raw = p.raw[anchor_block];
  const float mm0 = p.matrix_multiplier[0], mm1 = p.matrix_multiplier[1],
              mm2 = p.matrix_multiplier[2];
  const int tile = (a.y / 8) * p.tiles_x + (a.x / 8);
  const int8_t y_to_x = p.y_to_x[tile], y_to_b = p.y_to_b[tile];
  for (int i = tid; i < 3 * N; i += kT) {
    const int c = i / N, j = i % N;
    coef[c][j] = p.coef[c * p.pitch + static_cast<size_t>(a.y * 8 + j / W) * p.stride +
                        a.x * 8 + j % W];
    inverse_dequant[c][j] = p.inverse_dequant[i];
    if (c == 1) dequant_y[j] = p.dequant[N + j];
  }
  __syncthreads();
  // SelectAdjustedAcQuantization, the sums in parallel: every thread takes
  // coefficients of all three channels, storing each error term for the
  // ordered error sum and adding |quantized| into integer sums. Those sums are
  // the reference's float sums exactly while they stay below 2^24 (every
  // partial sum is then an integer the float holds exactly); past that, the
  // channel threads redo the sums serially.
  using Sh = TransformShape<W, H>;
  constexpr int xsize = Sh::SW / 8, ysize = Sh::SH / 8;
  const float qac = q.scale * static_cast<float>(initial_raw);
  float t0[4];
  AdjustThresholds<W, H>(t0);
  {
    uint32_t sums[3][5];
    uint32_t max_bits[4] = {0, 0, 0, 0};
    bool big = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float mm = c == 0 ? mm0 : c == 1 ? mm1 : mm2;
#pragma unroll
      for (int k = 0; k < 5; ++k) sums[c][k] = 0;
      for (int index = tid; index < N; index += kT) {
        const int y = index / Sh::SW, x = index % Sh::SW;
        if (x < xsize && y < ysize) {
          adjust_err[c][index] = 0.0f;
          continue;
        }
        const int quadrant = (y >= Sh::SH / 2) * 2 + (x >= Sh::SW / 2);
        const float value = coef[c][index] * (inverse_dequant[c][index] * qac * mm);
        const float quantized = fabsf(value) < t0[quadrant] ? 0.0f : rintf(value);
        const float err = fabsf(value - quantized);
        adjust_err[c][index] = err;
        const float magnitude = fabsf(quantized);
        if (magnitude < 16777216.0f) {
          const uint32_t m = static_cast<uint32_t>(magnitude);
          sums[c][0] += m;
          sums[c][1 + quadrant] += m;
        } else {
          big = true;
        }
        if (c == 1 && quantized == 0.0f) {
          // Non-negative floats order like their bit patterns; NaN errors are
          // skipped, as fmaxf skips them.
          if (err == err) max_bits[quadrant] = max(max_bits[quadrant], __float_as_uint(err));
        }
      }
      if (sums[c][0] >= (1u << 24)) big = true;
    }
    const int warp = tid / 32, lane = tid % 32;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const uint32_t total = __reduce_add_sync(0xffffffffu, big ? 0u : sums[c][k]);
        if (lane == 0) adjust_sum[warp][c][k] = total;
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t m = __reduce_max_sync(0xffffffffu, max_bits[k]);
      if (lane == 0) adjust_max[warp][k] = m;
    }
    const bool any_big = __any_sync(0xffffffffu, big);
    if (lane == 0) adjust_big[warp] = any_big ? 1 : 0;
  }
  __syncthreads();
  if (tid < 3) {
    const int c = tid;
    float t[4] = {t0[0], t0[1], t0[2], t0[3]};
    int candidate = initial_raw;
    AdjustSums sums;
    const uint32_t total = adjust_sum[0][c][0] + adjust_sum[1][c][0];
    if (adjust_big[0] | adjust_big[1] || total >= (1u << 24)) {
      AdjustSumsSerial<W, H>(qac, c, c == 0 ? mm0 : c == 1 ? mm1 : mm2, coef[c],
                             inverse_dequant[c], t, &sums);
    } else {
      // The ordered sums: error terms in storage order (+0.0 on the LLF
      // leaves the never -0.0 sum unchanged), and the border terms, which
      // all lie in the larger corner, in storage order.
      float error_sum = 0.0f;
#pragma unroll 8
      for (int index = 0; index < N; ++index) error_sum += adjust_err[c][index];
      float border_sum = 0.0f;
      const float mm = c == 0 ? mm0 : c == 1 ? mm1 : mm2;
      for (int y = 4 * ysize; y < Sh::SH; ++y) {
        for (int x = 4 * xsize; x < Sh::SW; ++x) {
          const bool in_corner = y >= 7 * ysize && x >= 7 * xsize;
          const bool on_border = y + 1 == Sh::SH || x + 1 == Sh::SW;
          if (!(in_corner || on_border)) continue;
          const int index = y * Sh::SW + x;
          const int quadrant = (y >= Sh::SH / 2) * 2 + (x >= Sh::SW / 2);
          const float value = coef[c][index] * (inverse_dequant[c][index] * qac * mm);
          const float quantized = fabsf(value) < t[quadrant] ? 0.0f : rintf(value);
          if (quantized != 0.0f) border_sum += fabsf(value);
        }
      }
      sums.error_sum = error_sum;
      sums.border_sum = border_sum;
      sums.value_sum = static_cast<float>(total);
      for (int k = 0; k < 4; ++k) {
        sums.nonzeros[k] = static_cast<float>(adjust_sum[0][c][1 + k] + adjust_sum[1][c][1 + k]);
        sums.max_error[k] =
          c == 1 ? __uint_as_float(max(adjust_max[0][k], adjust_max[1][k])) : 0.0f;
      }
    }
    AdjustFinish<W, H>(c, strategy, sums, t, &candidate);
    for (int i = 0; i < 4; ++i) thresholds[c][i] = t[i];
    candidates[c] = candidate;
  } else if (tid == 32) {
    // Y DC from the unquantized Y coefficients.
    float dc[16];
    LowFrequenciesToDc<W, H>(coef[1], dc);
    for (int dy = 0; dy < S::CH; ++dy)
      for (int dx = 0; dx < S::CW; ++dx)
        p.dc[1 * p.dc_pitch + static_cast<size_t>(a.y + dy) * p.blocks_x + a.x + dx] =
          dc[dy * S::CW + dx];
  }
  __syncthreads();
  const int raw = max(candidates[0], max(candidates[1], candidates[2]));
  if (raw < 1 || raw > 256) RaiseError(p.error, kErrorRange);
  if (tid == 0) p.raw[anchor_block] = raw;
  // Y: quantize with the adjusted thresholds, store, dequantize in place.
  const float y_scale = q.scale * static_cast<float>(raw) * 1.0f;
  const float y_dequant_scale = (q.inverse_global_scale / static_cast<float>(raw)) / 1.0f;
  for (int j = tid; j < N; j += kT) {
    const int x = j % S::SW, y = j / S::SW;
    const int ti = (y >= S::SH / 2) * 2 + (x >= S::SW / 2);
    const float value = inverse_dequant[1][j] * y_scale * coef[1][j];
    const int32_t quantized =
      fabsf(value) < thresholds[1][ti] ? 0 : static_cast<int32_t>(rintf(value));
    p.qac[p.pitch + static_cast<size_t>(a.y * 8 + j / W) * p.stride + a.x * 8 + j % W] = quantized;
    coef[1][j] = QuantBias(quantized, 1) * (dequant_y[j] * y_dequant_scale);
  }
  __syncthreads();
  // Remove the Y prediction from X and B.
  const float f0 = static_cast<float>(y_to_x) / 84.0f;
  const float f2 = 1.0f + static_cast<float>(y_to_b) / 84.0f;
  for (int j = tid; j < N; j += kT) {
    coef[0][j] -= f0 * coef[1][j];
    coef[2][j] -= f2 * coef[1][j];
  }
  __syncthreads();
  if (tid == 0 || tid == 32) {
    const int c = tid == 0 ? 0 : 2;
    float dc[16];
    LowFrequenciesToDc<W, H>(coef[c], dc);
    for (int dy = 0; dy < S::CH; ++dy)
      for (int dx = 0; dx < S::CW; ++dx)
        p.dc[c * p.dc_pitch + static_cast<size_t>(a.y + dy) * p.blocks_x + a.x + dx] =
          dc[dy * S::CW + dx];
  }
  float t[4];
  ChromaThresholds(covered, t);
  for (int i = tid; i < 2 * N; i += kT) {
    const int c = i < N ? 0 : 2, j = i % N;
    const int x = j % S::SW, y = j / S::SW;
    const int ti = (y >= S::SH / 2) * 2 + (x >= S::SW / 2);
    const float qs = q.scale * static_cast<float>(raw) * (c == 0 ? mm0 : mm2);
    const float value = inverse_dequant[c][j] * qs * coef[c][j];
    const int32_t quantized = fabsf(value) < t[ti] ? 0 : static_cast<int32_t>(rintf(value));
    p.qac[c * p.pitch + static_cast<size_t>(a.y * 8 + j / W) * p.stride + a.x * 8 + j % W] =
      quantized;
  }
}

// ---------------------------------------------------------------------------
// Prediction-aware DC quantization with the weighted predictor.
//
// The reference walks each 256x256-block DC group in raster order, channel
// by channel (Y, X, B), resetting the predictor per channel. A sample at
// (x, y) depends on row y at x-1 and on row y-1 at x-1..x+1 and row y-2 at x,
// through the quantized values and the predictor's error state. So all
// samples on a line x + 2y = t are independent, and the kernel sweeps those
// lines (waves). Rows y-1 and y-2 are then 2 and 4 samples ahead of row y, so
// every value a sample reads was written within the last 4 waves. Each row
// keeps its quantized values, signed errors and the four sub-predictor error
// sums in an 8-slot ring (slot x & 7) in shared memory; nothing goes to
// global memory but the quantized output.
//
// Two CTAs per DC group, one thread per (channel, row): one CTA runs X, the
// other Y (threads 0-255) and B (256-511). X and Y are independent. B's
// residual subtracts Y's quantized value at the same position, so B runs one
// wave behind Y and reads it from Y's ring. Slot x & 7 of a row is rewritten 8 waves later, and
// a reader needs it at most 4 waves (B: 1 wave) after it was written.

struct DcQuantParams {
  const float* dc;  // 3 planes of blocks
  int32_t* quantized;
  float* reconstructed;
  int width, height;
  size_t pitch;
  const AqQuantizer* q;
  float precision;  // 1 << extra_dc_precision
  // Replay: `replay` holds quantized DC already (3 planes of `pitch`) and the
  // kernel only runs the predictor over it, for its tokens.
  const int32_t* replay;
  // Optional DC tokens (context, packed residual) in the encoder's stream
  // order (DcTokenOffset), and the error word for a residual outside int32.
  uint2* tokens;
  uint32_t* error;
};

constexpr int kDcGroup = 256;
constexpr int kDcRing = 8;
// Two CTAs per DC group on different SMs: blockIdx.z == 0 runs X (threads
// 0-255; 256-511 idle), blockIdx.z == 1 runs Y (0-255) and B (256-511), which
// reads Y's ring.
constexpr int kDcThreads = 2 * kDcGroup;

struct DcRings {
  int32_t q[3][kDcRing][kDcGroup];        // quantized values
  int32_t e[3][kDcRing][kDcGroup];        // signed prediction errors (error_)
  uint32_t pe[3][4][kDcRing][kDcGroup];   // sub-predictor errors (prediction_errors_)
  uint32_t row0[3][4][kDcRing];           // row 0's own errors, before row 1 adds
  uint32_t reciprocal[64];                // (1 << 24) / (i + 1)
  uint8_t contexts[1024];                 // DC tree leaf of 512 + property
  int wide;  // set once a stored value leaves the 32-bit bounds below
};

__device__ __forceinline__ int BitWidth64(uint64_t v) { return v == 0 ? 0 : 64 - __clzll(v); }
__device__ __forceinline__ int BitWidth32(uint32_t v) { return v == 0 ? 0 : 32 - __clz(v); }

// Bounds under which every intermediate of one predictor step fits in 32
// bits: |quantized| <= 2^21 and |signed error| <= 2^23 for every stored
// value the step reads, and |value * inverse step| < 2^21 for its own
// sample. Then |8 q| <= 2^24, every sub-prediction is below 2^26 in
// magnitude, their weighted sum (weights adding up to at most 31) below
// 2^31, and the sub-predictor error sums below 2^28. The reference computes
// in 64 bits; within these bounds the 32-bit step gives the same values.
constexpr int32_t kDcNarrowQuantized = 1 << 21;
constexpr int32_t kDcNarrowError = 1 << 23;
constexpr float kDcNarrowScaled = 2097152.0f;  // 2^21

// One step of the weighted predictor (prediction.h:73-141) and the residual
// quantization (dc_quantization.cpp:178-199) in integer type Int: the
// neighbours' quantized values and signed errors, the four sub-predictor
// error sums and value * inverse step in; the quantized value, its signed
// error and the four sub-predictor errors out.
// In replay form (kReplay) the sample's quantized value comes in through
// *quantized_out and only the prediction and the update run.
template <typename Int, bool kWide, bool kReplay = false>
__device__ __forceinline__ void WeightedPredictorStep(Int w, Int n, Int nw, Int ne, Int nn, Int ew,
                                                      Int en, Int enw, Int ene,
                                                      const uint32_t (&errors)[4],
                                                      const uint32_t* reciprocal,
                                                      float scaled_value, int32_t* quantized_out,
                                                      int32_t* error_out,
                                                      uint32_t (&sub_errors)[4],
                                                      int64_t* predicted_out) {
  // WeightedPredictorParameters defaults (prediction.h:36-40).
  constexpr int kP0 = 16, kP1 = 10, kP2 = 7, kP3 = 7, kP4 = 7, kP5 = 0, kP6 = 0;
  const uint32_t max_weights[4] = {13, 12, 12, 12};
  uint32_t weights[4];
  uint32_t weight_sum = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int bits = kWide ? BitWidth64(static_cast<uint64_t>(errors[i]) + 1)
                           : BitWidth32(errors[i] + 1u);
    const int shift = max(0, bits - 6);
    weights[i] = 4 + ((max_weights[i] * reciprocal[errors[i] >> shift]) >> shift);
    weight_sum += weights[i];
  }
  const int log_weight = BitWidth32(weight_sum) - 1;
  weight_sum = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    weights[i] >>= log_weight - 4;
    weight_sum += weights[i];
  }
  const Int n8 = n * 8, w8 = w * 8, ne8 = ne * 8, nw8 = nw * 8, nn8 = nn * 8;
  Int predictions[4];
  predictions[0] = w8 + ne8 - n8;
  predictions[1] = n8 - (((en + ew + ene) * Int(kP0)) >> 5);
  predictions[2] = w8 - (((en + ew + enw) * Int(kP1)) >> 5);
  predictions[3] = n8 - ((enw * Int(kP2) + en * Int(kP3) + ene * Int(kP4) + (nn8 - n8) * Int(kP5) +
                          (nw8 - w8) * Int(kP6)) >> 5);
  Int sum = static_cast<Int>(weight_sum >> 1) - 1;
#pragma unroll
  for (int i = 0; i < 4; ++i) sum += predictions[i] * static_cast<Int>(weights[i]);
  Int prediction = static_cast<Int>(
    (static_cast<int64_t>(sum) * static_cast<int64_t>(reciprocal[weight_sum - 1])) >> 24);
  if (((en ^ ew) | (en ^ enw)) <= 0) {
    const Int lo = min(w8, min(ne8, n8)), hi = max(w8, max(ne8, n8));
    prediction = min(max(prediction, lo), hi);
  }
  const Int predicted = (prediction + 3) >> 3;
  *predicted_out = static_cast<int64_t>(predicted);
  Int quantized;
  if (kReplay) {
    quantized = static_cast<Int>(*quantized_out);
  } else {
    float residual = scaled_value;
    residual -= static_cast<float>(predicted);
    if (residual > -0.62f && residual < 0.62f) residual = 0.0f;
    float rounded = roundf(residual);
    if (rounded > 2.0f || rounded < -2.0f) rounded = roundf(residual * 0.5f) * 2.0f;
    quantized = predicted + static_cast<Int>(rounded);
    *quantized_out = static_cast<int32_t>(quantized);
  }
  // Update (prediction.h:121-141).
  const Int scaled = quantized * 8;
  *error_out = static_cast<int32_t>(prediction - scaled);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const Int d = predictions[i] - scaled;
    sub_errors[i] = static_cast<uint32_t>(((d < 0 ? -d : d) + 3) >> 3);
  }
}

template <bool kReplay>
__global__ void __launch_bounds__(kDcThreads, 1)
DcQuantKernel(const __grid_constant__ DcQuantParams p) {
  extern __shared__ __align__(16) unsigned char dc_smem[];
  DcRings& r = *reinterpret_cast<DcRings*>(dc_smem);
  const int gx0 = blockIdx.x * kDcGroup, gy0 = blockIdx.y * kDcGroup;
  const int gw = min(kDcGroup, p.width - gx0), gh = min(kDcGroup, p.height - gy0);
  const int stride = p.width;
  const bool idle = blockIdx.z == 0 && threadIdx.x >= kDcGroup;
  const int c = blockIdx.z == 0 ? 0 : 1 + static_cast<int>(threadIdx.x) / kDcGroup;  // X, Y, B
  const int y = idle ? kDcGroup : static_cast<int>(threadIdx.x) % kDcGroup;
  const int lag = c == 2 ? 1 : 0;
  for (int i = threadIdx.x; i < 64; i += blockDim.x) r.reciprocal[i] = (1u << 24) / (i + 1);
  if (p.tokens != nullptr) {
    for (int i = threadIdx.x; i < 1024; i += blockDim.x)
      r.contexts[i] = static_cast<uint8_t>(DcContextOfIndex(i));
  }
  if (threadIdx.x == 0) r.wide = 0;
  const AqQuantizer q = kReplay ? AqQuantizer{} : *p.q;
  const float inverse_step = kReplay ? 0.0f : q.inverse_dc_steps[c] * p.precision;
  const float step_y = kReplay ? 0.0f : q.dc_steps[1] / p.precision;
  int32_t* plane = kReplay ? nullptr : p.quantized + c * p.pitch;
  // The samples: DC values to quantize, or quantized values to replay, read
  // as raw 32-bit words.
  const uint32_t* source = kReplay ? reinterpret_cast<const uint32_t*>(p.replay + c * p.pitch)
                                   : reinterpret_cast<const uint32_t*>(p.dc + c * p.pitch);
  uint2* tokens = p.tokens == nullptr
                    ? nullptr
                    : p.tokens + DcTokenOffset(blockIdx.x, blockIdx.y, p.width, p.height) +
                        static_cast<size_t>(DcChannelRank(c)) * gw * gh;
  int32_t (*Q)[kDcGroup] = r.q[c];
  int32_t (*E)[kDcGroup] = r.e[c];
  __syncthreads();
  // The sample of the next position is loaded one wave ahead, so its
  // global-memory latency overlaps this wave's work and barrier.
  const size_t row_index = static_cast<size_t>(gy0 + min(y, gh - 1)) * stride + gx0;
  uint32_t pending = y < gh ? source[row_index] : 0u;  // idle threads have y >= gh
  // This row's previous quantized value and signed error (its west
  // neighbour), kept in registers.
  int32_t own_q = 0, own_e = 0;
  const int waves = (gw - 1) + 2 * (gh - 1) + 2;
  for (int t = 0; t < waves; ++t) {
    const int x = t - lag - 2 * y;
    const int wide = r.wide;
    if (y < gh && x >= 0 && x < gw) {
      const uint32_t sample = pending;
      if (x + 1 < gw) pending = source[row_index + x + 1];
      const int s = x & 7, sw = (x - 1) & 7, sne = (x + 1 < gw ? x + 1 : x) & 7;
      const int snw = (x ? x - 1 : x) & 7;
      const int up = y - 1, up2 = y - 2;
      const int32_t w = x ? own_q : y ? Q[s][up] : 0;
      const int32_t n = y ? Q[s][up] : w;
      const int32_t nw = x && y ? Q[sw][up] : w;
      const int32_t ne = y && x + 1 < gw ? Q[(x + 1) & 7][up] : n;
      const int32_t nn = y > 1 ? Q[s][up2] : n;
      const int32_t ew = x ? own_e : 0;
      const int32_t en = y ? E[s][up] : 0;
      const int32_t enw = y ? E[snw][up] : 0;
      const int32_t ene = y ? E[sne][up] : 0;
      // Sub-predictor error sums (prediction.h:73-90). The signed errors of
      // row -1 read as zeros. The error sums of row 0 read the predictor's
      // other rolling row, which by then holds only row 0's own "+="
      // updates: its entry j carries the error of (j - 1, 0) once that
      // sample is done, so north = err(x-1), northwest = err(x-2) and
      // northeast (not yet written) = 0, or north at the right edge.
      uint32_t errors[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (y) {
          errors[i] = r.pe[c][i][s][up] + r.pe[c][i][sne][up] + r.pe[c][i][snw][up];
        } else {
          const uint32_t north = x ? r.row0[c][i][sw] : 0u;
          const uint32_t northeast = x + 1 < gw ? 0u : north;
          const uint32_t northwest = x >= 2 ? r.row0[c][i][(x - 2) & 7] : 0u;
          errors[i] = north + northeast + northwest;
        }
      }
      float scaled_value = 0.0f;
      int32_t quantized = 0, error_value;
      bool narrow;
      if (kReplay) {
        quantized = static_cast<int32_t>(sample);
        narrow = quantized > -kDcNarrowQuantized && quantized < kDcNarrowQuantized;
      } else {
        float value = __uint_as_float(sample);
        if (c == 2) value = fmaf(-static_cast<float>(r.q[1][s][y]), step_y, value);
        scaled_value = value * inverse_step;
        narrow = fabsf(scaled_value) < kDcNarrowScaled;
      }
      uint32_t sub[4];
      int64_t predicted;
      if (!wide && narrow) {
        WeightedPredictorStep<int32_t, false, kReplay>(w, n, nw, ne, nn, ew, en, enw, ene,
                                                       errors, r.reciprocal, scaled_value,
                                                       &quantized, &error_value, sub,
                                                       &predicted);
      } else {
        WeightedPredictorStep<int64_t, true, kReplay>(w, n, nw, ne, nn, ew, en, enw, ene,
                                                      errors, r.reciprocal, scaled_value,
                                                      &quantized, &error_value, sub,
                                                      &predicted);
      }
      // Later steps read this value: past the 32-bit bounds, every later
      // step of the CTA takes the 64-bit form.
      if (static_cast<uint32_t>(quantized) + static_cast<uint32_t>(kDcNarrowQuantized) >
            static_cast<uint32_t>(2 * kDcNarrowQuantized) ||
          static_cast<uint32_t>(error_value) + static_cast<uint32_t>(kDcNarrowError) >
            static_cast<uint32_t>(2 * kDcNarrowError)) {
        r.wide = 1;
      }
      if (!kReplay) plane[row_index + x] = quantized;
      if (tokens != nullptr) {
        // The weighted predictor's context property: of ew, en, enw, ene the
        // first with the largest magnitude (prediction.h:95-99); the token is
        // the packed residual against the prediction (weighted_dc.cpp:67-80).
        int64_t property = ew;
        if (llabs(static_cast<int64_t>(en)) > llabs(property)) property = en;
        if (llabs(static_cast<int64_t>(enw)) > llabs(property)) property = enw;
        if (llabs(static_cast<int64_t>(ene)) > llabs(property)) property = ene;
        const int64_t index = property < -512 ? 0 : property > 511 ? 1023 : 512 + property;
        const int64_t residual = static_cast<int64_t>(quantized) - predicted;
        if (residual < INT32_MIN || residual > INT32_MAX) RaiseError(p.error, kErrorRange);
        tokens[y * gw + x] = make_uint2(r.contexts[index],
                                        PackSigned(static_cast<int32_t>(residual)));
      }
      Q[s][y] = quantized;
      E[s][y] = error_value;
      own_q = quantized;
      own_e = error_value;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        r.pe[c][i][s][y] = sub[i];
        if (y && x + 1 < gw) r.pe[c][i][(x + 1) & 7][up] += sub[i];
        if (!y) r.row0[c][i][s] = sub[i];
      }
    }
    __syncthreads();
  }
}

// Reconstructed DC (dc_quantization.cpp:209-222), once both channel CTAs of
// every group are done.
__global__ void DcDequantKernel(const int32_t* quantized, float* reconstructed, int n,
                                size_t pitch, const AqQuantizer* q, float precision) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float steps[3] = {q->dc_steps[0] / precision, q->dc_steps[1] / precision,
                          q->dc_steps[2] / precision};
  const float ry = static_cast<float>(quantized[pitch + i]) * steps[1];
  for (int ch = 0; ch < 3; ++ch) {
    float v = static_cast<float>(quantized[ch * pitch + i]) * steps[ch];
    if (ch == 2) v = fmaf(ry, 1.0f, v);
    reconstructed[ch * pitch + i] = v;
  }
}

// ComputeEpfInverseSigma (epf.cpp:207-270) with neutral sharpness 4.
__global__ void SigmaKernel(AnchorView v, const int32_t* raw, const AqQuantizer* q,
                            float* inverse_sigma) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.blocks_x * v.blocks_y) return;
  int cw, ch, s;
  if (!AnchorAt(v, i, &cw, &ch, &s)) return;
  const float kInvSigmaNumerator = -1.1715728752538099024f;
  const float sigma_quant = 0.46f / (q->scale * static_cast<float>(raw[i]) * kInvSigmaNumerator);
  float sigma = sigma_quant * (4.0f / 7.0f);
  sigma = fminf(-1.0e-4f, sigma);
  const float value = 1.0f / sigma;
  const int bx = i % v.blocks_x, by = i / v.blocks_x;
  for (int dy = 0; dy < ch; ++dy)
    for (int dx = 0; dx < cw; ++dx) inverse_sigma[(by + dy) * v.blocks_x + bx + dx] = value;
}

// SelectQuantizationMatrixScales (src/codestream/workflow.cpp:1435-1483) and
// QuantizationMatrixMultiplier (src/codec/codestream.cpp:92-96) on the device,
// so the stage chain needs no host round trip. `table[s]` = float(1.25^(s-2)).
struct MatrixScaleTable {
  float multiplier[16];
};

__global__ void MatrixScalesKernel(const float* stats, int have_stats, float target,
                                   MatrixScaleTable table, float* multipliers, int* scales) {
  const float x_edge = have_stats ? stats[0] : 0.0f;
  const float b_edge = have_stats ? stats[1] : 0.0f;
  const float exposed = have_stats ? stats[2] : 0.0f;
  int x = 3, b = 2;
  if (target > 2.5f) ++x;
  if (target > 5.5f) ++x;
  if (target > 9.5f) ++x;
  const int xa = x_edge >= 0.026f ? 3 : x_edge >= 0.022f ? 2 : x_edge >= 0.015f ? 1 : 0;
  x = max(x, 2 + xa);
  const int eb = exposed >= 0.13f ? 1 : 0;
  const int ba = b_edge > 0.38f ? 2 + eb : b_edge > 0.33f ? 1 + eb : b_edge > 0.28f ? eb : 0;
  b += ba;
  multipliers[0] = table.multiplier[x];
  multipliers[1] = 1.0f;
  multipliers[2] = table.multiplier[b];
  scales[0] = x;
  scales[1] = b;
}

unsigned Blocks(size_t n, unsigned threads = kThreads) {
  return static_cast<unsigned>((n + threads - 1) / threads);
}

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers.

void UploadDcTables() {
  DcTables t;
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
        t.inverse[li][f][s] = sqrt2 * alpha * std::cos(angle);
        t.forward[li][f][s] = sqrt2 * alpha * std::cos(angle) / static_cast<double>(len);
      }
    }
  }
  // DCTTotalResampleScale tables (dc_conversion.cpp:95-158).
  const float down[3][4] = {{1.0f, 0, 0, 0},
                            {1.0f, 0.901764195028874394f, 0, 0},
                            {1.0f, 0.974886821136879522f, 0.901764195028874394f,
                             0.787054918159101335f}};
  const float up[3][4] = {{1.0f, 0, 0, 0},
                          {1.0f, 1.108937353592731823f, 0, 0},
                          {1.0f, 1.025760096781116015f, 1.108937353592731823f,
                           1.270559368765487251f}};
  std::memcpy(t.downsample, down, sizeof(down));
  std::memcpy(t.upsample, up, sizeof(up));
  cudaMemcpyToSymbol(c_dc_tables, &t, sizeof(t));
}

int AqMatrixScales(const float* stats, bool have_stats, float target, float* multipliers,
                   int* scales, cudaStream_t stream) {
  MatrixScaleTable table;
  for (int s = 0; s < 16; ++s) table.multiplier[s] = static_cast<float>(std::pow(1.25, s - 2));
  MatrixScalesKernel<<<1, 1, 0, stream>>>(stats, have_stats ? 1 : 0, target, table, multipliers,
                                          scales);
  return CheckLaunch("aq matrix scales");
}

int AqBuildAnchors(const uint8_t* cells, size_t bx, size_t by, int2* lists, uint32_t* counts,
                   cudaStream_t stream) {
  const size_t blocks = bx * by;
  cudaMemsetAsync(counts, 0, kFamilyCountT * sizeof(uint32_t), stream);
  AnchorListKernel<<<Blocks(blocks), kThreads, 0, stream>>>(
    cells, static_cast<uint32_t>(bx), static_cast<uint32_t>(blocks), lists,
    static_cast<uint32_t>(blocks), counts);
  return CheckLaunch("aq anchors");
}

template <int W, int H>
int LaunchForward(const float* opsin, size_t stride, size_t pitch, const int2* list,
                  const uint32_t* count, size_t max_count, float* coef, cudaStream_t stream) {
  constexpr int N = W * H, K = 1024 / N;
  const size_t smem = static_cast<size_t>(PlaneBatch<W, H, 3 * K>::Elements) * 12;
  int status = CheckCuda(cudaFuncSetAttribute(ForwardCoefficientsKernel<W, H>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(smem)),
                         "aq forward attribute");
  if (status != GJXL_B200_OK) return status;
  const unsigned grid = static_cast<unsigned>((max_count + K - 1) / K);
  if (grid == 0) return GJXL_B200_OK;
  ForwardCoefficientsKernel<W, H><<<grid, kTransformThreads, smem, stream>>>(
    opsin, stride, pitch, list, count, static_cast<uint32_t>(max_count), coef, stride, pitch);
  return CheckLaunch("aq forward coefficients");
}

int AqForwardCoefficients(const float* opsin, size_t stride, size_t pitch, size_t bx, size_t by,
                          const int2* lists, const uint32_t* counts, float* coef,
                          cudaStream_t stream, const StreamFan* fan) {
  int status = GJXL_B200_OK;
  const size_t blocks = bx * by;
  // The families are independent: with a fan they run side by side.
  if (status == GJXL_B200_OK) status = CheckCuda(FanFork(fan), "fork");
  for (int f = 0; f < kFamilyCountT && status == GJXL_B200_OK; ++f) {
    const cudaStream_t fs = fan != nullptr ? fan->For(f) : stream;
    const int2* list = lists + f * blocks;
    const size_t max_count = blocks / (FamilyCoveredW(f) * FamilyCoveredH(f));
    switch (f) {
      case 0: status = LaunchForward<8, 8>(opsin, stride, pitch, list, counts + f, max_count, coef, fs); break;
      case 1: status = LaunchForward<8, 16>(opsin, stride, pitch, list, counts + f, max_count, coef, fs); break;
      case 2: status = LaunchForward<16, 8>(opsin, stride, pitch, list, counts + f, max_count, coef, fs); break;
      case 3: status = LaunchForward<16, 16>(opsin, stride, pitch, list, counts + f, max_count, coef, fs); break;
      case 4: status = LaunchForward<16, 32>(opsin, stride, pitch, list, counts + f, max_count, coef, fs); break;
      case 5: status = LaunchForward<32, 16>(opsin, stride, pitch, list, counts + f, max_count, coef, fs); break;
      case 6: status = LaunchForward<32, 32>(opsin, stride, pitch, list, counts + f, max_count, coef, fs); break;
    }
  }
  const cudaError_t joined = FanJoin(fan);
  if (status == GJXL_B200_OK) status = CheckCuda(joined, "join");
  return status;
}

int AqAdjustField(const uint8_t* cells, size_t bx, size_t by, const float* in, float* out,
                  float target, cudaStream_t stream) {
  const size_t blocks = bx * by;
  float mixer = 1.0f;
  const float kMixerLimit = 1.54138f, kMixerSlope = 0.56391f;
  if (target > kMixerLimit) mixer = std::max(0.0f, mixer - (target - kMixerLimit) * kMixerSlope);
  if (in != out) cudaMemcpyAsync(out, in, blocks * sizeof(float), cudaMemcpyDeviceToDevice, stream);
  AnchorView v{cells, static_cast<int>(bx), static_cast<int>(by)};
  AdjustFieldKernel<<<Blocks(blocks), kThreads, 0, stream>>>(v, in, out, mixer);
  return CheckLaunch("aq adjust field");
}

int AqPolicySetup(const float* field, size_t blocks, float target, float* range,
                  AqPolicy* policy, uint32_t* error, cudaStream_t stream) {
  RangeInitKernel<<<1, 1, 0, stream>>>(range);
  RangeKernel<<<Blocks(blocks), kThreads, 0, stream>>>(field, static_cast<int>(blocks), range);
  // ComputeInitialQuantDc (adaptive_quantization.cpp:536-560), host powf.
  const float kDcMul = 0.3f;
  const float nonlinear = kDcMul * std::pow(target / kDcMul, 0.83f);
  const float target_dc = std::max(0.5f * target, std::min(target, nonlinear));
  const float quant_dc = std::min(1.095924047623553f / target_dc, 50.0f);
  PolicySetupKernel<<<1, 1, 0, stream>>>(range, quant_dc, policy, error);
  return CheckLaunch("aq policy setup");
}

size_t AqSelectStateBytes() { return sizeof(SelectState); }

int AqQuantizer_(const float* field, size_t blocks, const AqPolicy* policy, AqQuantizer* q,
                 int32_t* raw, void* select_state, uint32_t* error, cudaStream_t stream) {
  SelectState* st = static_cast<SelectState*>(select_state);
  const int n = static_cast<int>(blocks);
  const unsigned grid = static_cast<unsigned>(std::min<size_t>(Blocks(blocks), 4 * 148));
  SelectInitKernel<<<1, 1024, 0, stream>>>(st, n);
  for (int selection = 0; selection < 2; ++selection) {
    for (int pass = 0; pass < kSelectPasses; ++pass) {
      SelectHistogramKernel<<<grid, kThreads, 0, stream>>>(field, n, selection == 1, pass, st);
      SelectDigitKernel<<<1, 1024, 0, stream>>>(pass, n, selection == 1, st);
    }
  }
  QuantizerKernel<<<1, 1, 0, stream>>>(st, policy, q, error);
  RawQuantKernel<<<Blocks(blocks), kThreads, 0, stream>>>(field, n, q, raw);
  return CheckLaunch("aq quantizer");
}

int AqFinalCfl(const uint8_t* cells, size_t bx, size_t by, const float* coef, size_t stride,
               size_t pitch, const int32_t* raw, const AqQuantizer* q, int8_t* y_to_x,
               int8_t* y_to_b, cudaStream_t stream) {
  DeviceTables d;
  int status = GetDeviceTables(&d);
  if (status != GJXL_B200_OK) return status;
  const HostTables& h = GetHostTables();
  CflFinalParams p;
  std::memset(&p, 0, sizeof(p));
  p.grid = {cells, static_cast<int>(bx), static_cast<int>(by)};
  p.tiles_x = static_cast<int>((bx + 7) / 8);
  p.tiles_y = static_cast<int>((by + 7) / 8);
  p.coef = coef;
  p.coef_stride = stride;
  p.coef_pitch = pitch;
  p.raw = raw;
  p.q = q;
  p.inverse_dequant = d.inverse_dequant;
  for (int t = 0; t < kTableCount; ++t) {
    p.table_offset[t] = h.layout.offset[t];
    p.table_count[t] = h.layout.count[t];
  }
  p.y_to_x = y_to_x;
  p.y_to_b = y_to_b;
  const size_t smem = 4 * kFinalCflTerms * sizeof(float);
  status = CheckCuda(cudaFuncSetAttribute(FinalCflKernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)),
                     "final cfl smem attribute");
  if (status != GJXL_B200_OK) return status;
  FinalCflKernel<<<p.tiles_x * p.tiles_y, kFinalCflThreads, smem, stream>>>(p);
  return CheckLaunch("aq final cfl");
}

template <int W, int H>
int LaunchCoding(CodingParams p, const DeviceTables& d, int family, size_t max_count,
                 cudaStream_t stream) {
  const HostTables& h = GetHostTables();
  const int table = StrategyTableFamily(FamilyStrategy(family));
  p.dequant = d.dequant + h.layout.offset[table];
  p.inverse_dequant = d.inverse_dequant + h.layout.offset[table];
  if (max_count == 0) return GJXL_B200_OK;
  CodingKernel<W, H><<<static_cast<unsigned>(max_count), CodingThreads<W, H>(), 0, stream>>>(p);
  return CheckLaunch("aq coding");
}

int AqCoding(const int2* lists, const uint32_t* counts, size_t bx, size_t by, const float* coef,
             size_t stride, size_t pitch, int32_t* qac, float* dc, int32_t* raw,
             const AqQuantizer* q, const int8_t* y_to_x, const int8_t* y_to_b,
             const float* matrix_multiplier, uint32_t* error, cudaStream_t stream,
             const StreamFan* fan) {
  DeviceTables d;
  int status = GetDeviceTables(&d);
  if (status != GJXL_B200_OK) return status;
  const size_t blocks = bx * by;
  CodingParams p;
  std::memset(&p, 0, sizeof(p));
  p.blocks_x = static_cast<int>(bx);
  p.dc_pitch = blocks;
  p.coef = coef;
  p.stride = stride;
  p.pitch = pitch;
  p.qac = qac;
  p.dc = dc;
  p.raw = raw;
  p.q = q;
  p.y_to_x = y_to_x;
  p.y_to_b = y_to_b;
  p.tiles_x = static_cast<int>((bx + 7) / 8);
  p.matrix_multiplier = matrix_multiplier;
  p.error = error;
  // The families are independent: with a fan they run side by side.
  if (status == GJXL_B200_OK) status = CheckCuda(FanFork(fan), "fork");
  for (int f = 0; f < kFamilyCountT && status == GJXL_B200_OK; ++f) {
    const cudaStream_t fs = fan != nullptr ? fan->For(f) : stream;
    p.anchors = lists + f * blocks;
    p.count = counts + f;
    const size_t max_count = blocks / (FamilyCoveredW(f) * FamilyCoveredH(f));
    switch (f) {
      case 0: status = LaunchCoding<8, 8>(p, d, f, max_count, fs); break;
      case 1: status = LaunchCoding<8, 16>(p, d, f, max_count, fs); break;
      case 2: status = LaunchCoding<16, 8>(p, d, f, max_count, fs); break;
      case 3: status = LaunchCoding<16, 16>(p, d, f, max_count, fs); break;
      case 4: status = LaunchCoding<16, 32>(p, d, f, max_count, fs); break;
      case 5: status = LaunchCoding<32, 16>(p, d, f, max_count, fs); break;
      case 6: status = LaunchCoding<32, 32>(p, d, f, max_count, fs); break;
    }
  }
  const cudaError_t joined = FanJoin(fan);
  if (status == GJXL_B200_OK) status = CheckCuda(joined, "join");
  return status;
}

namespace {

template <bool kReplay>
int LaunchDcQuant(const DcQuantParams& p, size_t bx, size_t by, cudaStream_t stream) {
  const int smem = static_cast<int>(sizeof(DcRings));
  int status = CheckCuda(cudaFuncSetAttribute(DcQuantKernel<kReplay>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                         "dc predictor attribute");
  if (status != GJXL_B200_OK) return status;
  dim3 grid(static_cast<unsigned>((bx + kDcGroup - 1) / kDcGroup),
            static_cast<unsigned>((by + kDcGroup - 1) / kDcGroup), 2);
  DcQuantKernel<kReplay><<<grid, kDcThreads, smem, stream>>>(p);
  return CheckLaunch("dc predictor");
}

}  // namespace

int AqDcQuantize(const float* dc, size_t bx, size_t by, const AqQuantizer* q, int32_t* quantized,
                 float* reconstructed, int extra_precision, uint2* tokens, uint32_t* error,
                 cudaStream_t stream) {
  DcQuantParams p;
  std::memset(&p, 0, sizeof(p));
  p.dc = dc;
  p.quantized = quantized;
  p.reconstructed = reconstructed;
  p.width = static_cast<int>(bx);
  p.height = static_cast<int>(by);
  p.pitch = bx * by;
  p.q = q;
  p.precision = static_cast<float>(1u << extra_precision);
  p.tokens = tokens;
  p.error = error;
  int status = LaunchDcQuant<false>(p, bx, by, stream);
  if (status != GJXL_B200_OK) return status;
  DcDequantKernel<<<Blocks(bx * by), kThreads, 0, stream>>>(
    quantized, reconstructed, static_cast<int>(bx * by), bx * by, q, p.precision);
  return CheckLaunch("aq dc quantize");
}

int DcWeightedTokens(const int32_t* quantized, size_t pitch, size_t bx, size_t by, uint2* tokens,
                     uint32_t* error, cudaStream_t stream) {
  DcQuantParams p;
  std::memset(&p, 0, sizeof(p));
  p.width = static_cast<int>(bx);
  p.height = static_cast<int>(by);
  p.pitch = pitch;
  p.replay = quantized;
  p.tokens = tokens;
  p.error = error;
  return LaunchDcQuant<true>(p, bx, by, stream);
}

int AqInverseSigma(const uint8_t* cells, size_t bx, size_t by, const int32_t* raw,
                   const AqQuantizer* q, float* inverse_sigma, cudaStream_t stream) {
  AnchorView v{cells, static_cast<int>(bx), static_cast<int>(by)};
  SigmaKernel<<<Blocks(bx * by), kThreads, 0, stream>>>(v, raw, q, inverse_sigma);
  return CheckLaunch("aq inverse sigma");
}

}  // namespace gjxl_b200
