// Shared pieces of the DC-group token streams (row f1): the fixed DC context
// tree's leaves, signed packing and the stream layout.
#pragma once

#include <cstdint>

namespace gjxl_b200 {

constexpr int kDcGroupBlocks = 256;  // blocks per side of a DC group
constexpr int kDcContextCount = 45;  // leaves of the fixed 45-context DC tree
constexpr int kHybridSymbols = 128;  // hybrid-uint {4, 2, 0} symbols of a uint32

// The leaves of the encoder's fixed DC context tree as runs over the clamped
// property index 512 + p in [0, 1023]: run k covers (end[k-1], end[k]] and
// maps to context ctx[k]. The same table serves the gradient property
// (dc_group.cpp:41-48) and the weighted predictor's error property
// (weighted_dc.cpp:22-29); it is part of the format's predefined tree, so the
// values must be these.
__host__ __device__ inline uint32_t DcContextOfIndex(int index) {
  constexpr uint16_t kEnd[34] = {12,  120, 257, 321, 385, 417, 449, 465, 481, 489, 497, 501,
                                 505, 508, 509, 511, 512, 513, 515, 517, 519, 523, 527, 535,
                                 543, 559, 575, 607, 639, 703, 767, 904, 1012, 1023};
  constexpr uint8_t kContext[34] = {44, 43, 40, 39, 38, 37, 36, 35, 34, 33, 32, 31,
                                    30, 29, 28, 27, 26, 42, 41, 25, 24, 23, 22, 21,
                                    20, 19, 18, 17, 16, 15, 14, 13, 12, 11};
  for (int k = 0; k < 34; ++k)
    if (index <= kEnd[k]) return kContext[k];
  return kContext[33];
}

// Context of a property value p: the leaf of clamp(512 + p, 0, 1023).
__host__ __device__ inline uint32_t DcContext(int64_t property) {
  const int64_t index = property < -512 ? 0 : property > 511 ? 1023 : 512 + property;
  return DcContextOfIndex(static_cast<int>(index));
}

// 0, -1, 1, -2, ... -> 0, 1, 2, 3, ... (entropy.h PackSigned).
__host__ __device__ inline uint32_t PackSigned(int32_t value) {
  return (static_cast<uint32_t>(value) << 1) ^ ((static_cast<uint32_t>(~value) >> 31) - 1u);
}

// First DC token of group (gx, gy): groups in row-major order, each holding
// 3 * area tokens (channels Y, X, B, raster order within each). Every group
// row above is 256 blocks high and every group to the left 256 blocks wide.
__host__ __device__ inline size_t DcTokenOffset(int gx, int gy, int blocks_x, int blocks_y) {
  const int row_height = blocks_y - gy * kDcGroupBlocks < kDcGroupBlocks
                           ? blocks_y - gy * kDcGroupBlocks
                           : kDcGroupBlocks;
  return 3 * (static_cast<size_t>(gy) * kDcGroupBlocks * blocks_x +
              static_cast<size_t>(gx) * kDcGroupBlocks * row_height);
}

// Rank of channel c (0 X, 1 Y, 2 B) in the stream order Y, X, B.
__host__ __device__ inline int DcChannelRank(int c) { return c == 1 ? 0 : c == 0 ? 1 : 2; }

}  // namespace gjxl_b200
