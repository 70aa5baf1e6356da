// Row f1: the DC-group token streams of a frame and their entropy-model
// histograms, on the device.
//
// Restates, with the reference's integer semantics:
//   TokenizeSimpleDcGroupsForEncoder (group slicing)  src/codestream/vardct/dc_group.cpp:469-546
//   TokenizeSimpleDcGroup (clamped gradient)          src/codestream/vardct/dc_group.cpp:291-347
//   TokenizeWeightedDcGroup (weighted predictor)      src/codestream/vardct/weighted_dc.cpp:47-89
//   TokenizeSimpleAcMetadata                          src/codestream/vardct/dc_group.cpp:349-427
//   AppendCflTokens / ClampedGradient                 src/codestream/vardct/dc_group.cpp:79-90,240-258
//   EncodeHybridUint {4, 2, 0} symbols                src/codestream/entropy.h:90-106
//
// Stream layout. DC tokens: groups in row-major order, each 3 * area tokens,
// channels Y, X, B, raster order (DcTokenOffset, no scan needed). Metadata
// tokens: per group 2 * tiles + 2 * anchors + area tokens (y_to_x map, y_to_b
// map, anchor strategies, anchor quant fields, EPF sharpness), groups in
// row-major order at offsets from a scan over the groups' anchor counts.
// Tokens are (context, value) uint32 pairs, EntropyToken's layout. Per group
// the host gets {dc_offset, dc_count, meta_offset, meta_count, anchors}.
//
// Kernels. Gradient DC: one thread per sample (the predictor is stateless).
// Weighted DC: the wavefront predictor of the DC quantization
// (aq_coding.cu), replaying quantized DC; inside the analysis it runs fused
// with the last DC quantization. Metadata: one CTA per group lists the
// group's anchors in raster order with a block-wide scan, a single CTA scans
// the groups, and a grid over (group, token) emits every token. Histograms:
// per-CTA shared-memory counts of (context, hybrid-uint symbol), merged with
// global atomics.

#include <cstring>

#include "aq.h"
#include "common.cuh"
#include "dc_tokens.cuh"
#include "host_util.h"

namespace gjxl_b200 {
namespace {

constexpr int kMetaThreads = 1024;
constexpr int kGroupInfoWords = 5;

struct DcTokenGeometry {
  int blocks_x, blocks_y, groups_x, groups_y, tiles_x;
};

__host__ __device__ inline int GroupWidth(const DcTokenGeometry& g, int gx) {
  return min(kDcGroupBlocks, g.blocks_x - gx * kDcGroupBlocks);
}
__host__ __device__ inline int GroupHeight(const DcTokenGeometry& g, int gy) {
  return min(kDcGroupBlocks, g.blocks_y - gy * kDcGroupBlocks);
}

// ClampedGradient (dc_group.cpp:79-90).
__device__ __forceinline__ int64_t ClampedGradient(int32_t top, int32_t left, int32_t top_left) {
  const int32_t lo = min(top, left), hi = max(top, left);
  if (top_left < lo) return hi;
  if (top_left > hi) return lo;
  return static_cast<int64_t>(top) + left - top_left;
}

__device__ __forceinline__ bool IsSimpleStrategy(int s) {
  return s == 0 || s == 4 || s == 5 || s == 6 || s == 7 || s == 10 || s == 11;
}

__device__ __forceinline__ uint32_t ResidualToken(int64_t residual, uint32_t* error) {
  if (residual < INT32_MIN || residual > INT32_MAX) RaiseError(error, kErrorRange);
  return PackSigned(static_cast<int32_t>(residual));
}

// Gradient-predicted DC tokens, one thread per (channel, block).
__global__ void DcGradientTokensKernel(const int32_t* dc, size_t pitch, DcTokenGeometry g,
                                       uint2* tokens, uint32_t* error) {
  const size_t per_channel = static_cast<size_t>(g.blocks_x) * g.blocks_y;
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 3 * per_channel) return;
  const int c = static_cast<int>(i / per_channel);
  const size_t b = i % per_channel;
  const int bx = static_cast<int>(b % g.blocks_x), by = static_cast<int>(b / g.blocks_x);
  const int gx = bx / kDcGroupBlocks, gy = by / kDcGroupBlocks;
  const int x = bx - gx * kDcGroupBlocks, y = by - gy * kDcGroupBlocks;
  const int gw = GroupWidth(g, gx), gh = GroupHeight(g, gy);
  const int32_t* row = dc + c * pitch + static_cast<size_t>(by) * g.blocks_x;
  const int32_t* up = row - g.blocks_x;
  const int32_t left = x ? row[bx - 1] : y ? up[bx] : 0;
  const int32_t top = y ? up[bx] : left;
  const int32_t top_left = x && y ? up[bx - 1] : left;
  const int64_t prediction = ClampedGradient(top, left, top_left);
  const uint32_t context =
    DcContext(static_cast<int64_t>(top) + left - static_cast<int64_t>(top_left));
  const size_t at = DcTokenOffset(gx, gy, g.blocks_x, g.blocks_y) +
                    static_cast<size_t>(DcChannelRank(c)) * gw * gh +
                    static_cast<size_t>(y) * gw + x;
  tokens[at] = make_uint2(context, ResidualToken(row[bx] - prediction, error));
}

// Anchors of one group in raster order: anchors[group base + rank] =
// strategy | raw quant << 8, and the group's anchor count. Also checks the
// reference's metadata preconditions (quant in [1, 256], sharpness below 8,
// a simple strategy at every anchor).
__global__ void __launch_bounds__(kMetaThreads)
MetaAnchorsKernel(const uint8_t* cells, const int32_t* raw_quant, const uint8_t* sharpness,
                  DcTokenGeometry g, uint32_t* anchors, uint32_t* counts, uint32_t* error) {
  __shared__ uint32_t warp_totals[kMetaThreads / 32];
  const int gx = blockIdx.x % g.groups_x, gy = blockIdx.x / g.groups_x;
  const int gw = GroupWidth(g, gx), gh = GroupHeight(g, gy);
  const int area = gw * gh;
  const int per_thread = (area + kMetaThreads - 1) / kMetaThreads;
  const int begin = min(area, static_cast<int>(threadIdx.x) * per_thread);
  const int end = min(area, begin + per_thread);
  const size_t origin = static_cast<size_t>(gy) * kDcGroupBlocks * g.blocks_x +
                        static_cast<size_t>(gx) * kDcGroupBlocks;
  uint32_t local = 0;
  for (int k = begin; k < end; ++k) {
    const size_t at = origin + static_cast<size_t>(k / gw) * g.blocks_x + k % gw;
    const uint8_t cell = cells[at];
    const int32_t quant = raw_quant[at];
    if (quant < 1 || quant > 256 || (sharpness != nullptr && sharpness[at] >= 8) ||
        ((cell & 1) && !IsSimpleStrategy(cell >> 1))) {
      RaiseError(error, kErrorRange);
    }
    local += cell & 1;
  }
  // Exclusive scan of the per-thread counts (thread order = raster order).
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inclusive = local;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, inclusive, d);
    if (lane >= d) inclusive += v;
  }
  if (lane == 31) warp_totals[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = warp_totals[lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, t, d);
      if (lane >= d) t += v;
    }
    warp_totals[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  uint32_t rank = inclusive - local + (warp ? warp_totals[warp - 1] : 0u);
  uint32_t* group_anchors = anchors + DcTokenOffset(gx, gy, g.blocks_x, g.blocks_y) / 3;
  for (int k = begin; k < end; ++k) {
    const size_t at = origin + static_cast<size_t>(k / gw) * g.blocks_x + k % gw;
    const uint8_t cell = cells[at];
    if (cell & 1) {
      group_anchors[rank++] =
        static_cast<uint32_t>(cell >> 1) | (static_cast<uint32_t>(raw_quant[at]) << 8);
    }
  }
  if (threadIdx.x == kMetaThreads - 1) counts[blockIdx.x] = warp_totals[31];
}

// Group table: {dc_offset, dc_count, meta_offset, meta_count, anchors}.
__global__ void MetaOffsetsKernel(const uint32_t* counts, DcTokenGeometry g, uint32_t* info) {
  if (threadIdx.x != 0) return;
  const int groups = g.groups_x * g.groups_y;
  uint32_t meta = 0;
  for (int i = 0; i < groups; ++i) {
    const int gx = i % g.groups_x, gy = i / g.groups_x;
    const int gw = GroupWidth(g, gx), gh = GroupHeight(g, gy);
    const uint32_t tiles = static_cast<uint32_t>(((gw + 7) / 8) * ((gh + 7) / 8));
    const uint32_t area = static_cast<uint32_t>(gw * gh);
    const uint32_t count = 2 * tiles + 2 * counts[i] + area;
    uint32_t* out = info + kGroupInfoWords * i;
    out[0] = static_cast<uint32_t>(DcTokenOffset(gx, gy, g.blocks_x, g.blocks_y));
    out[1] = 3 * area;
    out[2] = meta;
    out[3] = count;
    out[4] = counts[i];
    meta += count;
  }
}

__device__ __forceinline__ uint32_t StrategyContext(int32_t previous) {
  return previous > 11 ? 7 : previous > 5 ? 8 : previous > 3 ? 9 : 10;
}
__device__ __forceinline__ uint32_t QuantContext(int32_t previous) {
  return previous > 11 ? 3 : previous > 5 ? 4 : previous > 3 ? 5 : 6;
}

// Every metadata token of group blockIdx.y, thread-strided over its count.
__global__ void MetaEmitKernel(const uint8_t* cells, const uint8_t* sharpness, int sharpness_default,
                               const int8_t* y_to_x, const int8_t* y_to_b, DcTokenGeometry g,
                               const uint32_t* anchors, const uint32_t* info, uint2* tokens,
                               uint32_t* error) {
  const int group = blockIdx.y;
  const int gx = group % g.groups_x, gy = group / g.groups_x;
  const int gw = GroupWidth(g, gx), gh = GroupHeight(g, gy);
  const int tw = (gw + 7) / 8, th = (gh + 7) / 8, tiles = tw * th;
  const uint32_t* gi = info + kGroupInfoWords * group;
  const int count = static_cast<int>(gi[3]), anchor_count = static_cast<int>(gi[4]);
  uint2* out = tokens + gi[2];
  const uint32_t* group_anchors = anchors + gi[0] / 3;
  const size_t origin = static_cast<size_t>(gy) * kDcGroupBlocks * g.blocks_x +
                        static_cast<size_t>(gx) * kDcGroupBlocks;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    if (i < 2 * tiles) {
      // CfL maps (AppendCflTokens): y_to_x with context 2, then y_to_b with 1.
      const bool b_map = i >= tiles;
      const int t = b_map ? i - tiles : i;
      const int x = t % tw, y = t / tw;
      const int8_t* map = (b_map ? y_to_b : y_to_x) +
                          static_cast<size_t>(gy * 32 + y) * g.tiles_x + gx * 32 + x;
      const int32_t left = x ? map[-1] : y ? map[-g.tiles_x] : 0;
      const int32_t top = y ? map[-g.tiles_x] : left;
      const int32_t top_left = x && y ? map[-g.tiles_x - 1] : left;
      const int64_t residual = static_cast<int64_t>(*map) - ClampedGradient(top, left, top_left);
      out[i] = make_uint2(b_map ? 1u : 2u, ResidualToken(residual, error));
    } else if (i < 2 * tiles + anchor_count) {
      const int r = i - 2 * tiles;
      const int32_t code = static_cast<int32_t>(group_anchors[r] & 0xffu);
      const int32_t previous = r ? static_cast<int32_t>(group_anchors[r - 1] & 0xffu) : 0;
      out[i] = make_uint2(StrategyContext(previous), PackSigned(code));
    } else if (i < 2 * tiles + 2 * anchor_count) {
      // Quant field: the first anchor's predecessor is the strategy code of
      // the group's origin block (dc_group.cpp:398-412).
      const int r = i - 2 * tiles - anchor_count;
      const int32_t current = static_cast<int32_t>(group_anchors[r] >> 8) - 1;
      const int32_t previous = r ? static_cast<int32_t>(group_anchors[r - 1] >> 8) - 1
                                 : static_cast<int32_t>(cells[origin] >> 1);
      out[i] = make_uint2(QuantContext(previous),
                          ResidualToken(static_cast<int64_t>(current) - previous, error));
    } else {
      const int k = i - 2 * tiles - 2 * anchor_count;
      const size_t at = origin + static_cast<size_t>(k / gw) * g.blocks_x + k % gw;
      const int value = sharpness != nullptr ? sharpness[at] : sharpness_default;
      out[i] = make_uint2(0u, PackSigned(value));
    }
  }
}

// Hybrid-uint symbol of the default configuration {4, 2, 0}.
__device__ __forceinline__ uint32_t HybridSymbol(uint32_t v) {
  if (v < 16) return v;
  const int n = 31 - __clz(v);
  return 16 + (static_cast<uint32_t>(n) - 4) * 4 + ((v >> (n - 2)) & 3u);
}

__global__ void __launch_bounds__(256)
DcHistogramKernel(const uint2* dc_tokens, size_t dc_count, const uint2* meta_tokens,
                  const uint32_t* info, int groups, uint32_t* histogram) {
  __shared__ uint32_t counts[kDcContextCount * kHybridSymbols];
  for (int i = threadIdx.x; i < kDcContextCount * kHybridSymbols; i += blockDim.x) counts[i] = 0;
  __syncthreads();
  const uint32_t* last = info + kGroupInfoWords * (groups - 1);
  const size_t meta_count = static_cast<size_t>(last[2]) + last[3];
  const size_t total = dc_count + meta_count;
  for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint2 t = i < dc_count ? dc_tokens[i] : meta_tokens[i - dc_count];
    if (t.x < kDcContextCount) atomicAdd(&counts[t.x * kHybridSymbols + HybridSymbol(t.y)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kDcContextCount * kHybridSymbols; i += blockDim.x)
    if (counts[i] != 0) atomicAdd(&histogram[i], counts[i]);
}

DcTokenGeometry Geometry(size_t bx, size_t by) {
  DcTokenGeometry g;
  g.blocks_x = static_cast<int>(bx);
  g.blocks_y = static_cast<int>(by);
  g.groups_x = static_cast<int>((bx + kDcGroupBlocks - 1) / kDcGroupBlocks);
  g.groups_y = static_cast<int>((by + kDcGroupBlocks - 1) / kDcGroupBlocks);
  g.tiles_x = static_cast<int>((bx + 7) / 8);
  return g;
}

}  // namespace

size_t DcTokenScratchBytes(size_t bx, size_t by) {
  const DcTokenGeometry g = Geometry(bx, by);
  const size_t groups = static_cast<size_t>(g.groups_x) * g.groups_y;
  return (bx * by + groups) * sizeof(uint32_t);
}

size_t MetaTokenCapacity(size_t bx, size_t by) {
  return 2 * ((bx + 7) / 8) * ((by + 7) / 8) + 3 * bx * by;
}

int LaunchMetaTokens(const uint8_t* cells, const int32_t* raw_quant, const uint8_t* sharpness,
                     const int8_t* y_to_x, const int8_t* y_to_b, size_t bx, size_t by,
                     const uint2* dc_tokens, uint2* meta_tokens, uint32_t* info,
                     uint32_t* histogram, void* scratch, uint32_t* error, cudaStream_t stream) {
  const DcTokenGeometry g = Geometry(bx, by);
  const int groups = g.groups_x * g.groups_y;
  uint32_t* anchors = static_cast<uint32_t*>(scratch);
  uint32_t* counts = anchors + bx * by;
  MetaAnchorsKernel<<<groups, kMetaThreads, 0, stream>>>(cells, raw_quant, sharpness, g, anchors,
                                                         counts, error);
  MetaOffsetsKernel<<<1, 32, 0, stream>>>(counts, g, info);
  // Up to 2 * 1024 + 3 * 65536 tokens per group.
  MetaEmitKernel<<<dim3(64, groups), 256, 0, stream>>>(cells, sharpness, 4, y_to_x, y_to_b, g,
                                                       anchors, info, meta_tokens, error);
  if (histogram != nullptr) {
    cudaMemsetAsync(histogram, 0, kDcContextCount * kHybridSymbols * sizeof(uint32_t), stream);
    DcHistogramKernel<<<148, 256, 0, stream>>>(dc_tokens, 3 * bx * by, meta_tokens, info, groups,
                                               histogram);
  }
  return CheckLaunch("dc group tokens");
}

}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" int gjxl_b200_dc_token_sizes(size_t blocks_x, size_t blocks_y, size_t* dc_tokens,
                                        size_t* meta_tokens, size_t* groups,
                                        size_t* scratch_bytes) {
  ClearLastError();
  if (blocks_x == 0 || blocks_y == 0 || blocks_x > (1u << 17) || blocks_y > (1u << 17)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "dc_token_sizes: invalid extent");
  }
  if (dc_tokens != nullptr) *dc_tokens = 3 * blocks_x * blocks_y;
  if (meta_tokens != nullptr) *meta_tokens = MetaTokenCapacity(blocks_x, blocks_y);
  if (groups != nullptr) {
    *groups = ((blocks_x + kDcGroupBlocks - 1) / kDcGroupBlocks) *
              ((blocks_y + kDcGroupBlocks - 1) / kDcGroupBlocks);
  }
  if (scratch_bytes != nullptr) *scratch_bytes = DcTokenScratchBytes(blocks_x, blocks_y);
  return GJXL_B200_OK;
}

extern "C" int gjxl_b200_dc_tokenize(const int32_t* quantized_dc, size_t dc_plane_pitch,
                                     const uint8_t* cells, const int32_t* raw_quant,
                                     const uint8_t* epf_sharpness, const int8_t* y_to_x,
                                     const int8_t* y_to_b, size_t blocks_x, size_t blocks_y,
                                     int prediction, uint32_t* dc_tokens, uint32_t* meta_tokens,
                                     uint32_t* group_info, uint32_t* histogram, void* scratch,
                                     size_t scratch_bytes, uint32_t* device_error,
                                     void* stream) {
  ClearLastError();
  if (quantized_dc == nullptr || cells == nullptr || raw_quant == nullptr || y_to_x == nullptr ||
      y_to_b == nullptr || dc_tokens == nullptr || meta_tokens == nullptr ||
      group_info == nullptr || scratch == nullptr || blocks_x == 0 || blocks_y == 0 ||
      blocks_x > (1u << 17) || blocks_y > (1u << 17) ||
      dc_plane_pitch < blocks_x * blocks_y || (prediction != 0 && prediction != 1) ||
      scratch_bytes < DcTokenScratchBytes(blocks_x, blocks_y) ||
      reinterpret_cast<uintptr_t>(dc_tokens) % 8 || reinterpret_cast<uintptr_t>(meta_tokens) % 8 ||
      reinterpret_cast<uintptr_t>(scratch) % 4) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "dc_tokenize: invalid arguments");
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint2* dc = reinterpret_cast<uint2*>(dc_tokens);
  int status;
  if (prediction == 1) {
    status = DcWeightedTokens(quantized_dc, dc_plane_pitch, blocks_x, blocks_y, dc, device_error,
                              s);
  } else {
    const DcTokenGeometry g = Geometry(blocks_x, blocks_y);
    const size_t n = 3 * blocks_x * blocks_y;
    DcGradientTokensKernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
      quantized_dc, dc_plane_pitch, g, dc, device_error);
    status = CheckLaunch("dc gradient tokens");
  }
  if (status != GJXL_B200_OK) return status;
  return LaunchMetaTokens(cells, raw_quant, epf_sharpness, y_to_x, y_to_b, blocks_x, blocks_y, dc,
                          reinterpret_cast<uint2*>(meta_tokens), group_info, histogram, scratch,
                          device_error, s);
}
