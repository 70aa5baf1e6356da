// Rows a17 and a18: AC group packing, coefficient-order populations and
// custom orders, and AC tokenization on the device.
//
// Restates, with the reference's exact integer semantics:
//   ComputeSimpleNaturalCoefficientOrder       src/codestream/ac_group.cpp:381-488
//   CountGroupZeros / ComputeCoefficientOrdersWithCounts
//                                              src/codestream/coefficient_order.cpp:205-315,568-823
//   CoefficientOrderPopulation layout          src/codec/coefficient_order_population_internal.h
//   UseCoefficientOrderSample (xorshift128+)   src/codestream/coefficient_order.cpp:115-126
//   TokenizeSimpleAcGroupDirectValidated       src/codestream/ac_group.cpp:740-932
//   NonzeroBucket / ZeroDensityContext / PredictNonzeros / BlockContextValidated
//                                              src/codestream/ac_group.cpp:82-126
//   AppendDirectAcToken (hybrid-uint symbols)  src/codestream/ac_group.cpp:688-738
//   AC group coefficient order                 src/codec/vardct_frame.cpp:880-921
//
// Inputs are the analysis outputs in their device layout: the strategy grid
// ((strategy << 1) | anchor per block), the raw quant field, and quantized
// AC in footprint layout (coefficient i of the transform anchored at block
// (bx, by) with pixel footprint W x H at (bx*8 + i % W, by*8 + i / W)).
//
// Work decomposition. A task is one (anchor, channel) pair, indexed by block
// position and channel slot (Y, X, B in that order, as the reference emits
// them); non-anchor positions are empty tasks. One warp per task counts
// nonzeros and finds the last nonzero in scan order, one CTA per 256x256
// group scans the task token counts in the reference's order (anchors in
// raster order within the group), a single CTA scans the groups, and one
// warp per task emits its tokens with warp prefix sums over the scan.

#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "host_util.h"
#include "transform.cuh"

namespace gjxl_b200 {
namespace {

constexpr int kGroupBlocks = 32;           // kVarDctAcGroupBlockDimension
constexpr int kOrderFamilies = 13;         // kSimpleCoefficientOrderCount
constexpr int kNonzeroBuckets = 37;        // kSimpleNonzeroBucketCount
constexpr int kZeroDensityContexts = 458;  // kSimpleZeroDensityContextCount
constexpr int kSymbols = 128;              // kPrefixAlphabetSize
constexpr int kPopulationStride = 1984;    // per channel
constexpr int kPopulationFull = 3 * kPopulationStride;
constexpr int kPopulationCount = kPopulationFull + 3 * 64;
constexpr int kOrderStride = 1024;         // orders table: [13][3][1024]

// Order family of a strategy id (kSimpleStrategyOrder for the mixed-search
// strategies), its population offset and size, and a representative shape.
__host__ __device__ constexpr int OrderFamily(int strategy) {
  return strategy == kStrategyDct8 ? 0 : strategy == kStrategyDct16x16 ? 2
       : strategy == kStrategyDct32x32 ? 3
       : (strategy == kStrategyDct16x8 || strategy == kStrategyDct8x16) ? 4 : 6;
}
__host__ __device__ constexpr int PopulationOffset(int family) {
  return family == 0 ? 0 : family == 2 ? 64 : family == 3 ? 320 : family == 4 ? 1344 : 1472;
}
__host__ __device__ constexpr int FamilySize(int family) {
  return family == 0 ? 64 : family == 2 ? 256 : family == 3 ? 1024 : family == 4 ? 128
       : family == 6 ? 512 : 0;
}
// Covered blocks (longer side, shorter side) of a family's transforms.
__host__ __device__ constexpr int FamilyBlocksLong(int family) {
  return family == 0 ? 1 : family == 2 ? 2 : family == 3 ? 4 : family == 4 ? 2 : 4;
}
__host__ __device__ constexpr int FamilyBlocksShort(int family) {
  return family == 0 ? 1 : family == 2 ? 2 : family == 3 ? 4 : family == 4 ? 1 : 2;
}
constexpr int kFamilies[5] = {0, 2, 3, 4, 6};
__host__ __device__ constexpr int FamilyOfIndex(int i) {
  return i == 0 ? 0 : i == 1 ? 2 : i == 2 ? 3 : i == 3 ? 4 : 6;
}

__constant__ uint16_t c_frequency_context[64] = {
  0,  0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14,
  15, 15, 16, 16, 17, 17, 18, 18, 19, 19, 20, 20, 21, 21, 22, 22,
  23, 23, 23, 23, 24, 24, 24, 24, 25, 25, 25, 25, 26, 26, 26, 26,
  27, 27, 27, 27, 28, 28, 28, 28, 29, 29, 29, 29, 30, 30, 30, 30};
__constant__ uint16_t c_nonzero_context[64] = {
  0,   0,   31,  62,  62,  93,  93,  93,  93,  123, 123, 123, 123, 152, 152, 152,
  152, 152, 152, 152, 152, 180, 180, 180, 180, 180, 180, 180, 180, 180, 180, 180,
  180, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206,
  206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206, 206};

// The scan order of the JPEG XL natural coefficient order for a transform
// covering `blocks_long` x `blocks_short` blocks (longer side first): the LLF
// rectangle first, then the remaining coefficients along anti-diagonals of
// the square (8 * blocks_long)^2 grid, alternating direction, keeping only
// rows that are multiples of the anisotropy and scaling them down. Returns
// physical indices y * width + x of the coefficient layout.
std::vector<uint32_t> NaturalOrder(int blocks_long, int blocks_short) {
  const int width = blocks_long * 8;
  const int anisotropy = blocks_long / blocks_short;
  const int count = width * blocks_short * 8;
  std::vector<uint32_t> order(static_cast<size_t>(count), 0);
  int next = blocks_long * blocks_short;
  auto visit = [&](int x, int y, bool llf_slot) {
    if (y % anisotropy != 0) return;
    y /= anisotropy;
    if (llf_slot && x < blocks_long && y < blocks_short) {
      order[static_cast<size_t>(y * blocks_long + x)] = static_cast<uint32_t>(y * width + x);
    } else {
      order[static_cast<size_t>(next++)] = static_cast<uint32_t>(y * width + x);
    }
  };
  for (int diagonal = 0; diagonal < width; ++diagonal) {
    for (int position = 0; position <= diagonal; ++position) {
      int x = position, y = diagonal - position;
      if (diagonal & 1) std::swap(x, y);
      visit(x, y, true);
    }
  }
  for (int reverse = width - 1; reverse > 0; --reverse) {
    const int diagonal = reverse - 1;
    for (int position = 0; position <= diagonal; ++position) {
      int x = width - 1 - (diagonal - position), y = width - 1 - position;
      if (diagonal & 1) std::swap(x, y);
      visit(x, y, false);
    }
  }
  return order;
}

// Per-block decisions of the effort-7 DCT8 population sample: one draw of the
// xorshift128+ generator per block, groups in row-major order and blocks in
// raster order within each group, seeded as the reference seeds it.
std::vector<uint8_t> SampleDecisions(int bx, int by) {
  std::vector<uint8_t> decisions(static_cast<size_t>(bx) * by, 0);
  uint64_t s0 = 0x94D049BB133111EBull, s1 = 0xBF58476D1CE4E5B9ull;
  const int gx = (bx + kGroupBlocks - 1) / kGroupBlocks;
  const int gy = (by + kGroupBlocks - 1) / kGroupBlocks;
  for (int g = 0; g < gx * gy; ++g) {
    const int x0 = (g % gx) * kGroupBlocks, y0 = (g / gx) * kGroupBlocks;
    const int w = std::min(kGroupBlocks, bx - x0), h = std::min(kGroupBlocks, by - y0);
    for (int y = 0; y < h; ++y) {
      for (int x = 0; x < w; ++x) {
        uint64_t a = s0;
        const uint64_t b = s1;
        const uint64_t bits = a + b;
        s0 = b;
        a ^= a << 23;
        a ^= b ^ (a >> 18) ^ (b >> 5);
        s1 = a;
        decisions[static_cast<size_t>(y0 + y) * bx + x0 + x] =
          (bits >> 32) <= ((~uint64_t{0} >> 32) / 2) ? 1 : 0;
      }
    }
  }
  return decisions;
}

struct TaskShape {
  int family = -1;   // order family, -1 for a non-anchor block
  int cw = 0, ch = 0, n = 0, covered = 0, log2_covered = 0, footprint_w = 0;
  int llf_w = 0, llf_h = 0, coef_w = 0;
  int footprint_shift = 0, coef_shift = 0;  // log2 of footprint_w and coef_w
};

__device__ __forceinline__ TaskShape ShapeAt(const uint8_t* cells, int index) {
  TaskShape t;
  const uint8_t cell = cells[index];
  if (!(cell & 1)) return t;
  const int strategy = cell >> 1;
  const int f = StrategyFamily(strategy);
  t.family = OrderFamily(strategy);
  t.cw = FamilyCoveredW(f);
  t.ch = FamilyCoveredH(f);
  t.covered = t.cw * t.ch;
  t.n = t.covered * 64;
  t.log2_covered = __ffs(t.covered) - 1;  // covered is a power of two
  t.footprint_w = t.cw * 8;
  t.llf_w = max(t.cw, t.ch);
  t.llf_h = min(t.cw, t.ch);
  t.coef_w = t.llf_w * 8;
  // Widths are 8, 16 or 32.
  t.footprint_shift = __ffs(t.footprint_w) - 1;
  t.coef_shift = __ffs(t.coef_w) - 1;
  return t;
}

__device__ __forceinline__ int Coefficient(const int32_t* qac, size_t stride, size_t pitch, int c,
                                           int bx, int by, int footprint_w, int i) {
  return qac[c * pitch + static_cast<size_t>(by * 8 + i / footprint_w) * stride + bx * 8 +
             i % footprint_w];
}

// Coefficient() with the footprint width given as its log2 (a shift and a
// mask instead of a division by a runtime width).
__device__ __forceinline__ int CoefficientShift(const int32_t* qac, size_t stride, size_t pitch,
                                                int c, int bx, int by, int footprint_shift,
                                                int i) {
  return qac[c * pitch + static_cast<size_t>(by * 8 + (i >> footprint_shift)) * stride + bx * 8 +
             (i & ((1 << footprint_shift) - 1))];
}

__device__ __forceinline__ uint32_t WarpSumU(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int WarpMaxI(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ uint32_t WarpExclusive(uint32_t v, int lane) {
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x - v;
}

// ---------------------------------------------------------------------------
// Order populations (zero counts per family, channel and physical index).

struct PopulationParams {
  const uint8_t* cells;
  const int32_t* qac;
  size_t stride, pitch;
  int blocks_x, blocks_y, groups_x;
  const uint8_t* sample;      // per block
  uint32_t* population;       // kPopulationCount
  uint32_t* present_mask;
};

// One CTA per group and channel (blockIdx.y). The group's anchors are first
// listed per family, with the log2 of their footprint width; then, family by
// family, each thread owns one physical index (and a share of the anchors
// when the family has fewer than 256 indices) and counts zeros in a
// register, four anchors' coefficients loaded at a time, so shared-memory
// atomics happen once per thread and index, not once per coefficient.
__global__ void __launch_bounds__(256) PopulationKernel(const __grid_constant__ PopulationParams p) {
  __shared__ uint32_t counts[kPopulationStride + 64];  // this channel; then the DCT8 sample
  __shared__ short2 anchors[5][kGroupBlocks * kGroupBlocks];
  __shared__ uint8_t anchor_shift[5][kGroupBlocks * kGroupBlocks];
  __shared__ uint8_t sampled[kGroupBlocks * kGroupBlocks];
  __shared__ int anchor_count[5];
  __shared__ uint32_t present;
  const int c = blockIdx.y;
  for (int i = threadIdx.x; i < kPopulationStride + 64; i += blockDim.x) counts[i] = 0;
  if (threadIdx.x < 5) anchor_count[threadIdx.x] = 0;
  if (threadIdx.x == 0) present = 0;
  __syncthreads();
  const int x0 = (blockIdx.x % p.groups_x) * kGroupBlocks;
  const int y0 = (blockIdx.x / p.groups_x) * kGroupBlocks;
  const int w = min(kGroupBlocks, p.blocks_x - x0), h = min(kGroupBlocks, p.blocks_y - y0);
  for (int b = threadIdx.x; b < w * h; b += blockDim.x) {
    const int bx = x0 + b % w, by = y0 + b / w;
    const TaskShape t = ShapeAt(p.cells, by * p.blocks_x + bx);
    if (t.family < 0) continue;
    const int fi = t.family == 0 ? 0 : t.family == 2 ? 1 : t.family == 3 ? 2 : t.family == 4 ? 3 : 4;
    const int slot = atomicAdd(&anchor_count[fi], 1);
    anchors[fi][slot] = make_short2(static_cast<short>(bx), static_cast<short>(by));
    // Footprint widths are 8, 16 or 32.
    anchor_shift[fi][slot] = static_cast<uint8_t>(__ffs(t.footprint_w) - 1);
    if (fi == 0) sampled[slot] = p.sample[by * p.blocks_x + bx];
    atomicOr(&present, 1u << t.family);
  }
  __syncthreads();
  const int32_t* plane = p.qac + c * p.pitch;
  for (int fi = 0; fi < 5; ++fi) {
    const int count = anchor_count[fi];
    if (count == 0) continue;
    const int family = FamilyOfIndex(fi), n = FamilySize(family);
    const int shares = n >= static_cast<int>(blockDim.x) ? 1 : static_cast<int>(blockDim.x) / n;
    const int share = static_cast<int>(threadIdx.x) / (n >= static_cast<int>(blockDim.x) ? static_cast<int>(blockDim.x) : n);
    if (share >= shares) continue;
    for (int i = static_cast<int>(threadIdx.x) % n; i < n; i += blockDim.x) {
      uint32_t zeros = 0, zeros_sampled = 0;
      for (int a0 = share; a0 < count; a0 += 4 * shares) {
        // Both orientations of a rectangular family share physical indices;
        // the footprint width of each anchor decides where index i lies.
        int32_t v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int a = a0 + k * shares;
          v[k] = 1;
          if (a < count) {
            const short2 anchor = anchors[fi][a];
            const int shift = anchor_shift[fi][a];
            v[k] = plane[static_cast<size_t>(anchor.y * 8 + (i >> shift)) * p.stride +
                         anchor.x * 8 + (i & ((1 << shift) - 1))];
          }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int a = a0 + k * shares;
          const bool zero = a < count && v[k] == 0;
          zeros += zero;
          if (fi == 0 && zero && sampled[a]) ++zeros_sampled;
        }
      }
      if (zeros) atomicAdd(counts + PopulationOffset(family) + i, zeros);
      if (zeros_sampled) atomicAdd(counts + kPopulationStride + i, zeros_sampled);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kPopulationStride; i += blockDim.x) {
    if (counts[i]) atomicAdd(p.population + c * kPopulationStride + i, counts[i]);
  }
  for (int i = threadIdx.x; i < 64; i += blockDim.x) {
    if (counts[kPopulationStride + i]) {
      atomicAdd(p.population + kPopulationFull + c * 64 + i, counts[kPopulationStride + i]);
    }
  }
  if (threadIdx.x == 0 && present) atomicOr(p.present_mask, present);
}

// ---------------------------------------------------------------------------
// Custom orders (ComputeCoefficientOrdersWithCounts): per present family and
// channel, the natural scan with its non-LLF part stably sorted by
// uint64(float(zeros) / sqrt(N) + 0.1f), ties by natural position.

struct OrderParams {
  const uint32_t* natural;     // [13][1024]
  const uint32_t* population;  // kPopulationCount
  const uint32_t* present_mask;
  uint32_t* custom;            // [13][3][1024]
  uint32_t* used_mask;
  int sampled_behavior;        // effort-7 DCT8 sampling
  int enabled;                 // frame large enough for custom orders
};

__global__ void __launch_bounds__(1024) OrderKernel(const __grid_constant__ OrderParams p) {
  const int family = FamilyOfIndex(blockIdx.x / 3), c = blockIdx.x % 3;
  const int n = FamilySize(family);
  const uint32_t present = *p.present_mask;
  if (!p.enabled || !(present & (1u << family))) return;
  __shared__ uint32_t keys[1024];
  __shared__ uint32_t natural[1024];
  __shared__ uint32_t rank_of[1024];
  __shared__ int differs;
  const int llf = FamilyBlocksLong(family) * FamilyBlocksShort(family);
  const bool sample = family == 0 && present == 1u && p.sampled_behavior;
  const uint32_t* counts = sample ? p.population + kPopulationFull + c * 64
                                  : p.population + c * kPopulationStride + PopulationOffset(family);
  const float inverse_sqrt = 1.0f / sqrtf(static_cast<float>(n));
  if (threadIdx.x == 0) differs = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t physical = p.natural[family * 1024 + i];
    natural[i] = physical;
    keys[i] = static_cast<uint32_t>(
      static_cast<uint64_t>(static_cast<float>(counts[physical]) * inverse_sqrt + 0.1f));
  }
  __syncthreads();
  // Rank of scan position i among the sortable positions [llf, n).
  for (int i = llf + static_cast<int>(threadIdx.x); i < n; i += blockDim.x) {
    const uint32_t key = keys[i];
    int rank = llf;
    for (int j = llf; j < n; ++j) rank += keys[j] < key || (keys[j] == key && j < i);
    rank_of[i] = static_cast<uint32_t>(rank);
  }
  __syncthreads();
  uint32_t* out = p.custom + (family * 3 + c) * kOrderStride;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int at = i < llf ? i : static_cast<int>(rank_of[i]);
    out[at] = natural[i];
    if (at != i) differs = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0 && differs) atomicOr(p.used_mask, 1u << family);
}

// The scan each (family, channel) uses: custom where the family's custom
// order is used, else natural. Also zeroes the sampled DCT8 population bins
// unless the frame holds DCT8 only (they are defined only for such frames).
__global__ void FinalizeOrdersKernel(const uint32_t* natural, const uint32_t* custom,
                                     const uint32_t* masks, uint32_t* population,
                                     uint32_t* orders) {
  const uint32_t* used_mask = masks + 1;
  if (blockIdx.x == 0 && masks[0] != 1u) {
    for (int i = threadIdx.x; i < 3 * 64; i += blockDim.x) population[kPopulationFull + i] = 0;
  }
  const int family = FamilyOfIndex(blockIdx.x / 3), c = blockIdx.x % 3;
  const int n = FamilySize(family);
  const bool used = (*used_mask >> family) & 1u;
  uint32_t* out = orders + (family * 3 + c) * kOrderStride;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    out[i] = used ? custom[(family * 3 + c) * kOrderStride + i] : natural[family * 1024 + i];
  }
}

// ---------------------------------------------------------------------------
// Tokenization.

struct BlockContextMap {
  uint32_t threshold_count;
  uint32_t thresholds[15];
  uint32_t num_contexts;
  uint8_t map[3 * 13 * 16];
};

struct TokenParams {
  const uint8_t* cells;
  const int32_t* raw;
  const int32_t* qac;
  size_t stride, pitch;
  int blocks_x, blocks_y, groups_x;
  const uint32_t* orders;    // [13][3][1024] scans in use
  uint32_t* task_tokens;     // 3 * blocks: token count (0 for non-anchors)
  uint32_t* task_nonzeros;   // 3 * blocks
  int32_t* task_last;        // 3 * blocks: last nonzero scan position, -1 if none
  uint32_t* task_offset;     // 3 * blocks: offset within the group
  uint32_t* coef_offset;     // blocks: packed coefficient offset within the group
  uint32_t* group_tokens;    // groups
  uint32_t* group_coefs;     // groups
  uint32_t* group_offsets;   // groups + 1: token offsets
  uint32_t* group_coef_offsets;  // groups + 1: packed coefficient offsets (per channel x3)
  uint8_t* nonzero_map;      // 3 * blocks
  uint32_t* values;
  uint16_t* contexts;
  uint32_t* histogram;       // may be null
  int32_t* packed;           // may be null
  uint32_t capacity;
  uint32_t* error;
  BlockContextMap map;
};

// Channels of a task's slots, in the reference's emission order Y, X, B.
__device__ __forceinline__ int ChannelOfSlot(int slot) { return slot == 0 ? 1 : slot == 1 ? 0 : 2; }

// One warp per (block, channel slot): nonzero count outside the LLF, the last
// nonzero scan position, the token count and the scaled nonzero map.
__global__ void __launch_bounds__(256) TaskMetaKernel(const __grid_constant__ TokenParams p) {
  const int lane = threadIdx.x % 32;
  const int task = blockIdx.x * 8 + threadIdx.x / 32;
  const int blocks = p.blocks_x * p.blocks_y;
  if (task >= 3 * blocks) return;
  const int block = task / 3, slot = task % 3, c = ChannelOfSlot(slot);
  const TaskShape t = ShapeAt(p.cells, block);
  if (t.family < 0) {
    if (lane == 0) p.task_tokens[task] = 0;
    return;
  }
  const int bx = block % p.blocks_x, by = block / p.blocks_x;
  const uint32_t* order = p.orders + (t.family * 3 + c) * kOrderStride;
  uint32_t nonzeros = 0;
  int last = -1;
  for (int j = lane; j < t.n; j += 32) {
    const int physical = static_cast<int>(order[j]);
    const int v =
      CoefficientShift(p.qac, p.stride, p.pitch, c, bx, by, t.footprint_shift, physical);
    const int px = physical & (t.coef_w - 1), py = physical >> t.coef_shift;
    const bool llf = px < t.llf_w && py < t.llf_h;
    if (v != 0 && !llf) nonzeros += 1;
    if (v != 0 && j >= t.covered) last = j;
  }
  nonzeros = WarpSumU(nonzeros);
  last = WarpMaxI(last);
  if (lane == 0) {
    p.task_nonzeros[task] = nonzeros;
    p.task_last[task] = last;
    p.task_tokens[task] = nonzeros == 0 ? 1u : static_cast<uint32_t>(last - t.covered + 2);
  }
  const uint8_t scaled = static_cast<uint8_t>((nonzeros + t.covered - 1) / t.covered);
  if (lane < t.covered) {
    const int dx = lane % t.cw, dy = lane / t.cw;
    p.nonzero_map[c * blocks + (by + dy) * p.blocks_x + bx + dx] = scaled;
  }
}

// One CTA per group: token and packed-coefficient offsets of every task in
// the reference's order (anchors in raster order, channels Y, X, B).
__global__ void __launch_bounds__(1024) GroupScanKernel(const __grid_constant__ TokenParams p) {
  __shared__ uint32_t warp_tokens[32], warp_coefs[32];
  const int x0 = (blockIdx.x % p.groups_x) * kGroupBlocks;
  const int y0 = (blockIdx.x / p.groups_x) * kGroupBlocks;
  const int w = min(kGroupBlocks, p.blocks_x - x0), h = min(kGroupBlocks, p.blocks_y - y0);
  const int i = threadIdx.x, lane = i % 32, warp = i / 32;
  const bool in = i < w * h;
  const int block = in ? (y0 + i / w) * p.blocks_x + x0 + i % w : 0;
  uint32_t tokens[3] = {0, 0, 0}, coefs = 0;
  if (in) {
    for (int s = 0; s < 3; ++s) tokens[s] = p.task_tokens[3 * block + s];
    const TaskShape t = ShapeAt(p.cells, block);
    coefs = t.family < 0 ? 0u : static_cast<uint32_t>(t.n);
  }
  const uint32_t my_tokens = tokens[0] + tokens[1] + tokens[2];
  const uint32_t tok_prefix = WarpExclusive(my_tokens, lane);
  const uint32_t coef_prefix = WarpExclusive(coefs, lane);
  if (lane == 31) {
    warp_tokens[warp] = tok_prefix + my_tokens;
    warp_coefs[warp] = coef_prefix + coefs;
  }
  __syncthreads();
  if (warp == 0) {
    const uint32_t a = warp_tokens[lane], b = warp_coefs[lane];
    const uint32_t ea = WarpExclusive(a, lane), eb = WarpExclusive(b, lane);
    warp_tokens[lane] = ea;
    warp_coefs[lane] = eb;
    if (lane == 31) {
      p.group_tokens[blockIdx.x] = ea + a;
      p.group_coefs[blockIdx.x] = eb + b;
    }
  }
  __syncthreads();
  if (in) {
    uint32_t offset = warp_tokens[warp] + tok_prefix;
    for (int s = 0; s < 3; ++s) {
      p.task_offset[3 * block + s] = offset;
      offset += tokens[s];
    }
    p.coef_offset[block] = warp_coefs[warp] + coef_prefix;
  }
}

// Exclusive scan over the groups (a single CTA, sequential chunks of 1024).
__global__ void __launch_bounds__(1024) GroupOffsetsKernel(const __grid_constant__ TokenParams p,
                                                          int groups) {
  __shared__ uint32_t warp_sums[2][32];
  __shared__ uint32_t carry[2];
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  if (threadIdx.x == 0) carry[0] = carry[1] = 0;
  __syncthreads();
  for (int base = 0; base < groups; base += 1024) {
    const int g = base + static_cast<int>(threadIdx.x);
    const uint32_t t = g < groups ? p.group_tokens[g] : 0u;
    const uint32_t k = g < groups ? p.group_coefs[g] : 0u;
    const uint32_t et = WarpExclusive(t, lane), ek = WarpExclusive(k, lane);
    if (lane == 31) {
      warp_sums[0][warp] = et + t;
      warp_sums[1][warp] = ek + k;
    }
    __syncthreads();
    if (warp == 0) {
      const uint32_t a = warp_sums[0][lane], b = warp_sums[1][lane];
      warp_sums[0][lane] = WarpExclusive(a, lane);
      warp_sums[1][lane] = WarpExclusive(b, lane);
    }
    __syncthreads();
    if (g < groups) {
      p.group_offsets[g] = carry[0] + warp_sums[0][warp] + et;
      p.group_coef_offsets[g] = 3 * (carry[1] + warp_sums[1][warp] + ek);
    }
    __syncthreads();
    if (threadIdx.x == 1023) {
      carry[0] += warp_sums[0][31] + et + t;
      carry[1] += warp_sums[1][31] + ek + k;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    p.group_offsets[groups] = carry[0];
    p.group_coef_offsets[groups] = 3 * carry[1];
    if (carry[0] > p.capacity) RaiseError(p.error, kErrorRange);
  }
}

__device__ __forceinline__ uint32_t HybridSymbol(uint32_t value) {
  if (value < 16) return value;
  const uint32_t exponent = 31u - __clz(value);
  return 16u + ((exponent - 4u) << 2) + ((value - (1u << exponent)) >> (exponent - 2u));
}

// Adds one token to the histogram; lanes with the same (context, symbol) add
// once together.
__device__ __forceinline__ void CountToken(uint32_t* histogram, bool active, uint32_t context,
                                           uint32_t value) {
  const uint32_t key = active ? context * kSymbols + HybridSymbol(value) : 0xffffffffu;
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const int leader = __ffs(peers) - 1;
  if (active && (threadIdx.x % 32) == leader) atomicAdd(histogram + key, __popc(peers));
}

// One warp per task: the nonzero-count token, then the coefficients in scan
// order up to the last nonzero.
__global__ void __launch_bounds__(256) EmitKernel(const __grid_constant__ TokenParams p) {
  const int lane = threadIdx.x % 32;
  const int task = blockIdx.x * 8 + threadIdx.x / 32;
  const int blocks = p.blocks_x * p.blocks_y;
  if (task >= 3 * blocks) return;
  if (p.group_offsets[(p.blocks_x + kGroupBlocks - 1) / kGroupBlocks *
                      ((p.blocks_y + kGroupBlocks - 1) / kGroupBlocks)] > p.capacity) {
    return;  // capacity exceeded: reported by GroupOffsetsKernel
  }
  const int block = task / 3, slot = task % 3, c = ChannelOfSlot(slot);
  const TaskShape t = ShapeAt(p.cells, block);
  if (t.family < 0) return;
  const int bx = block % p.blocks_x, by = block / p.blocks_x;
  const int gx = bx / kGroupBlocks, gy = by / kGroupBlocks;
  const int group = gy * p.groups_x + gx;
  const uint32_t out = p.group_offsets[group] + p.task_offset[task];
  const uint32_t nonzeros = p.task_nonzeros[task];
  const int last = p.task_last[task];
  // Block context (BlockContextValidated).
  const int raw = p.raw[block];
  uint32_t segment = 0;
  while (segment < p.map.threshold_count && static_cast<uint32_t>(raw) > p.map.thresholds[segment]) {
    ++segment;
  }
  const int channel_row = c < 2 ? (c ^ 1) : 2;
  const uint32_t block_context =
    p.map.map[(channel_row * kOrderFamilies + t.family) * (p.map.threshold_count + 1) + segment];
  const uint32_t num_contexts = p.map.num_contexts;
  if (lane == 0) {
    // PredictNonzeros on the group-local map.
    const uint8_t* map = p.nonzero_map + c * blocks;
    const int x = bx - gx * kGroupBlocks, y = by - gy * kGroupBlocks;
    uint32_t prediction;
    if (x == 0) {
      prediction = y == 0 ? 32u : map[(by - 1) * p.blocks_x + bx - x];
    } else if (y == 0) {
      prediction = map[by * p.blocks_x + bx - 1];
    } else {
      prediction = (static_cast<uint32_t>(map[(by - 1) * p.blocks_x + bx]) +
                    map[by * p.blocks_x + bx - 1] + 1) / 2;
    }
    const uint32_t bucket = prediction < 8 ? prediction : prediction >= 64 ? 36 : 4 + prediction / 2;
    const uint32_t context = bucket * num_contexts + block_context;
    p.values[out] = nonzeros;
    p.contexts[out] = static_cast<uint16_t>(context);
    if (p.histogram != nullptr) {
      atomicAdd(p.histogram + context * kSymbols + HybridSymbol(nonzeros), 1u);
    }
  }
  if (nonzeros == 0) return;
  const uint32_t* order = p.orders + (t.family * 3 + c) * kOrderStride;
  const uint32_t coefficient_base = num_contexts * kNonzeroBuckets + kZeroDensityContexts * block_context;
  uint32_t consumed = 0;
  uint32_t previous = nonzeros > static_cast<uint32_t>(t.n / 16) ? 0u : 1u;
  for (int first = t.covered; first <= last; first += 32) {
    const int j = first + lane;
    const bool active = j <= last;
    const int v = active ? CoefficientShift(p.qac, p.stride, p.pitch, c, bx, by, t.footprint_shift,
                                       static_cast<int>(order[j]))
                         : 0;
    const uint32_t nz = v != 0 ? 1u : 0u;
    const uint32_t before = WarpExclusive(nz, lane);
    const uint32_t remaining = nonzeros - consumed - before;
    const uint32_t up = __shfl_up_sync(0xffffffffu, nz, 1);
    const uint32_t prev = lane == 0 ? previous : up;
    uint32_t context = 0, value = 0;
    if (active) {
      const uint32_t local =
        (c_nonzero_context[(remaining + t.covered - 1) >> t.log2_covered] +
         c_frequency_context[j >> t.log2_covered]) * 2 + prev;
      context = coefficient_base + local;
      value = (static_cast<uint32_t>(v) << 1) ^ static_cast<uint32_t>(v >> 31);
      const uint32_t at = out + 1 + static_cast<uint32_t>(j - t.covered);
      p.values[at] = value;
      p.contexts[at] = static_cast<uint16_t>(context);
    }
    if (p.histogram != nullptr) CountToken(p.histogram, active, context, value);
    consumed += WarpSumU(nz);
    previous = __shfl_sync(0xffffffffu, nz, 31);
  }
}

// Packed AC in group order: per group, channel 0..2 each holding the anchors'
// coefficients 0..N-1 in raster anchor order.
__global__ void __launch_bounds__(256) PackKernel(const __grid_constant__ TokenParams p) {
  const int lane = threadIdx.x % 32;
  const int block = blockIdx.x * 8 + threadIdx.x / 32;
  if (block >= p.blocks_x * p.blocks_y) return;
  const TaskShape t = ShapeAt(p.cells, block);
  if (t.family < 0) return;
  const int bx = block % p.blocks_x, by = block / p.blocks_x;
  const int group = (by / kGroupBlocks) * p.groups_x + bx / kGroupBlocks;
  const uint32_t used = p.group_coef_offsets[group + 1] - p.group_coef_offsets[group];
  const uint32_t per_channel = used / 3;
  for (int c = 0; c < 3; ++c) {
    int32_t* dst = p.packed + p.group_coef_offsets[group] + c * per_channel + p.coef_offset[block];
    for (int i = lane; i < t.n; i += 32) {
      dst[i] = CoefficientShift(p.qac, p.stride, p.pitch, c, bx, by, t.footprint_shift, i);
    }
  }
}

unsigned Grid(size_t n, unsigned per) { return static_cast<unsigned>((n + per - 1) / per); }

}  // namespace
}  // namespace gjxl_b200

using namespace gjxl_b200;

struct gjxl_b200_ac_tokens {
  int bx = 0, by = 0, gx = 0, gy = 0;
  void* arena = nullptr;
  uint32_t* natural = nullptr;        // [13][1024]
  uint8_t* sample = nullptr;          // per block
  uint32_t* population = nullptr;     // kPopulationCount
  uint32_t* masks = nullptr;          // [0] present, [1] used
  uint32_t* custom = nullptr;         // [13][3][1024]
  uint32_t* orders = nullptr;         // [13][3][1024]
  uint32_t* task_tokens = nullptr;
  uint32_t* task_nonzeros = nullptr;
  int32_t* task_last = nullptr;
  uint32_t* task_offset = nullptr;
  uint32_t* coef_offset = nullptr;
  uint32_t* group_tokens = nullptr;
  uint32_t* group_coefs = nullptr;
  uint32_t* group_offsets = nullptr;
  uint32_t* group_coef_offsets = nullptr;
  uint8_t* nonzero_map = nullptr;
  ~gjxl_b200_ac_tokens() {
    if (arena) cudaFree(arena);
  }
};

extern "C" size_t gjxl_b200_ac_token_capacity(size_t blocks_x, size_t blocks_y) {
  // Each (anchor, channel) task emits at most 1 + N - covered tokens.
  return 3 * blocks_x * blocks_y * 64 + 3 * blocks_x * blocks_y;
}

extern "C" int gjxl_b200_ac_tokens_create(size_t blocks_x, size_t blocks_y,
                                          gjxl_b200_ac_tokens** out) {
  ClearLastError();
  if (out == nullptr || blocks_x == 0 || blocks_y == 0 || blocks_x > (1u << 17) ||
      blocks_y > (1u << 17) || blocks_x * blocks_y > (1u << 26)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "ac_tokens_create: invalid extent");
  }
  *out = nullptr;
  auto* s = new (std::nothrow) gjxl_b200_ac_tokens();
  if (s == nullptr) return SetError(GJXL_B200_OUT_OF_MEMORY, "ac_tokens_create: host allocation");
  s->bx = static_cast<int>(blocks_x);
  s->by = static_cast<int>(blocks_y);
  s->gx = (s->bx + kGroupBlocks - 1) / kGroupBlocks;
  s->gy = (s->by + kGroupBlocks - 1) / kGroupBlocks;
  const size_t blocks = blocks_x * blocks_y, groups = static_cast<size_t>(s->gx) * s->gy;
  struct Item {
    void** ptr;
    size_t bytes;
  };
  const Item items[] = {
    {reinterpret_cast<void**>(&s->natural), 13 * 1024 * 4},
    {reinterpret_cast<void**>(&s->sample), blocks},
    {reinterpret_cast<void**>(&s->population), kPopulationCount * 4},
    {reinterpret_cast<void**>(&s->masks), 16},
    {reinterpret_cast<void**>(&s->custom), 13 * 3 * 1024 * 4},
    {reinterpret_cast<void**>(&s->orders), 13 * 3 * 1024 * 4},
    {reinterpret_cast<void**>(&s->task_tokens), 3 * blocks * 4},
    {reinterpret_cast<void**>(&s->task_nonzeros), 3 * blocks * 4},
    {reinterpret_cast<void**>(&s->task_last), 3 * blocks * 4},
    {reinterpret_cast<void**>(&s->task_offset), 3 * blocks * 4},
    {reinterpret_cast<void**>(&s->coef_offset), blocks * 4},
    {reinterpret_cast<void**>(&s->group_tokens), groups * 4},
    {reinterpret_cast<void**>(&s->group_coefs), groups * 4},
    {reinterpret_cast<void**>(&s->group_offsets), (groups + 1) * 4},
    {reinterpret_cast<void**>(&s->group_coef_offsets), (groups + 1) * 4},
    {reinterpret_cast<void**>(&s->nonzero_map), 3 * blocks},
  };
  size_t total = 0;
  for (const Item& item : items) total = (total + 255) / 256 * 256 + item.bytes;
  int status = CheckCuda(DeviceMalloc(&s->arena, total), "ac_tokens_create: cudaMalloc");
  if (status != GJXL_B200_OK) {
    delete s;
    return status;
  }
  size_t offset = 0;
  for (const Item& item : items) {
    offset = (offset + 255) / 256 * 256;
    *item.ptr = static_cast<unsigned char*>(s->arena) + offset;
    offset += item.bytes;
  }
  std::vector<uint32_t> natural(13 * 1024, 0);
  for (int family : kFamilies) {
    const std::vector<uint32_t> order = NaturalOrder(FamilyBlocksLong(family),
                                                     FamilyBlocksShort(family));
    std::copy(order.begin(), order.end(), natural.begin() + family * 1024);
  }
  const std::vector<uint8_t> decisions = SampleDecisions(s->bx, s->by);
  status = CheckCuda(cudaMemcpy(s->natural, natural.data(), natural.size() * 4,
                                cudaMemcpyHostToDevice), "ac_tokens_create: natural orders");
  if (status == GJXL_B200_OK) {
    status = CheckCuda(cudaMemcpy(s->sample, decisions.data(), decisions.size(),
                                  cudaMemcpyHostToDevice), "ac_tokens_create: sample");
  }
  if (status != GJXL_B200_OK) {
    delete s;
    return status;
  }
  *out = s;
  return GJXL_B200_OK;
}

extern "C" void gjxl_b200_ac_tokens_destroy(gjxl_b200_ac_tokens* s) { delete s; }

extern "C" int gjxl_b200_ac_tokenize(gjxl_b200_ac_tokens* s, const uint8_t* strategy_cells,
                                     const int32_t* raw_quant_field, const int32_t* quantized_ac,
                                     size_t stride, size_t plane_pitch,
                                     const gjxl_b200_block_context_map* map, int order_mode,
                                     const gjxl_b200_ac_token_outputs* out, void* stream_ptr) {
  ClearLastError();
  if (s == nullptr || strategy_cells == nullptr || raw_quant_field == nullptr ||
      quantized_ac == nullptr || map == nullptr || out == nullptr ||
      out->token_values == nullptr || out->token_contexts == nullptr ||
      out->group_offsets == nullptr || order_mode < 0 || order_mode > 2 ||
      stride < static_cast<size_t>(s->bx) * 8 ||
      plane_pitch < stride * static_cast<size_t>(s->by) * 8 || map->threshold_count > 15 ||
      map->num_contexts == 0 || map->num_contexts > 16) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "ac_tokenize: invalid arguments");
  }
  const int segments = static_cast<int>(map->threshold_count) + 1;
  for (int i = 0; i < 3 * 13 * segments; ++i) {
    if (map->context_map[i] >= map->num_contexts) {
      return SetError(GJXL_B200_INVALID_ARGUMENT, "ac_tokenize: context map entry out of range");
    }
  }
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const size_t blocks = static_cast<size_t>(s->bx) * s->by;
  const int groups = s->gx * s->gy;
  const size_t capacity = gjxl_b200_ac_token_capacity(s->bx, s->by);
  if (out->token_capacity < capacity || capacity > 0xffffffffu) {
    return SetError(GJXL_B200_INVALID_ARGUMENT,
                    "ac_tokenize: token_capacity below gjxl_b200_ac_token_capacity()");
  }
  int status = CheckCuda(cudaMemsetAsync(s->population, 0, kPopulationCount * 4, stream),
                         "ac_tokenize: clear population");
  if (status != GJXL_B200_OK) return status;
  status = CheckCuda(cudaMemsetAsync(s->masks, 0, 16, stream), "ac_tokenize: clear masks");
  if (status != GJXL_B200_OK) return status;
  if (out->histogram != nullptr) {
    status = CheckCuda(cudaMemsetAsync(out->histogram, 0,
                                       static_cast<size_t>(map->num_contexts) * 495 * kSymbols * 4,
                                       stream),
                       "ac_tokenize: clear histogram");
    if (status != GJXL_B200_OK) return status;
  }
  // a17: order populations and the scans in use.
  if (order_mode != 0 || out->order_population != nullptr) {
    PopulationParams pp;
    pp.cells = strategy_cells;
    pp.qac = quantized_ac;
    pp.stride = stride;
    pp.pitch = plane_pitch;
    pp.blocks_x = s->bx;
    pp.blocks_y = s->by;
    pp.groups_x = s->gx;
    pp.sample = s->sample;
    pp.population = s->population;
    pp.present_mask = s->masks;
    PopulationKernel<<<dim3(groups, 3), 256, 0, stream>>>(pp);
  }
  if (order_mode != 0) {
    OrderParams op;
    op.natural = s->natural;
    op.population = s->population;
    op.present_mask = s->masks;
    op.custom = s->custom;
    op.used_mask = s->masks + 1;
    op.sampled_behavior = order_mode == 2 ? 1 : 0;
    op.enabled = (s->bx >= 5 || s->by >= 5) ? 1 : 0;
    OrderKernel<<<15, 1024, 0, stream>>>(op);
  }
  FinalizeOrdersKernel<<<15, 256, 0, stream>>>(s->natural, s->custom, s->masks, s->population,
                                               s->orders);
  status = CheckLaunch("ac_tokenize: orders");
  if (status != GJXL_B200_OK) return status;
  // a18: tokens.
  TokenParams p;
  std::memset(&p, 0, sizeof(p));
  p.cells = strategy_cells;
  p.raw = raw_quant_field;
  p.qac = quantized_ac;
  p.stride = stride;
  p.pitch = plane_pitch;
  p.blocks_x = s->bx;
  p.blocks_y = s->by;
  p.groups_x = s->gx;
  p.orders = s->orders;
  p.task_tokens = s->task_tokens;
  p.task_nonzeros = s->task_nonzeros;
  p.task_last = s->task_last;
  p.task_offset = s->task_offset;
  p.coef_offset = s->coef_offset;
  p.group_tokens = s->group_tokens;
  p.group_coefs = s->group_coefs;
  p.group_offsets = out->group_offsets;
  p.group_coef_offsets = s->group_coef_offsets;
  p.nonzero_map = s->nonzero_map;
  p.values = out->token_values;
  p.contexts = out->token_contexts;
  p.histogram = out->histogram;
  p.packed = out->packed_ac;
  p.capacity = static_cast<uint32_t>(capacity);
  p.error = out->device_error;
  p.map.threshold_count = map->threshold_count;
  for (uint32_t i = 0; i < map->threshold_count; ++i) p.map.thresholds[i] = map->qf_thresholds[i];
  p.map.num_contexts = map->num_contexts;
  std::memcpy(p.map.map, map->context_map, 3 * 13 * segments);
  TaskMetaKernel<<<Grid(3 * blocks, 8), 256, 0, stream>>>(p);
  GroupScanKernel<<<groups, 1024, 0, stream>>>(p);
  GroupOffsetsKernel<<<1, 1024, 0, stream>>>(p, groups);
  EmitKernel<<<Grid(3 * blocks, 8), 256, 0, stream>>>(p);
  if (out->packed_ac != nullptr) PackKernel<<<Grid(blocks, 8), 256, 0, stream>>>(p);
  status = CheckLaunch("ac_tokenize: tokens");
  if (status != GJXL_B200_OK) return status;
  // Published side outputs.
  const struct {
    void* dst;
    const void* src;
    size_t bytes;
  } copies[] = {
    {out->order_population, s->population, kPopulationCount * 4},
    {out->present_mask, s->masks, 4},
    {out->used_order_mask, s->masks + 1, 4},
    {out->orders, s->orders, 13 * 3 * 1024 * 4},
    {out->group_coef_offsets, s->group_coef_offsets, (static_cast<size_t>(groups) + 1) * 4},
  };
  for (const auto& copy : copies) {
    if (copy.dst == nullptr) continue;
    status = CheckCuda(cudaMemcpyAsync(copy.dst, copy.src, copy.bytes, cudaMemcpyDeviceToDevice,
                                       stream),
                       "ac_tokenize: output copy");
    if (status != GJXL_B200_OK) return status;
  }
  return GJXL_B200_OK;
}
