// Rows a6/a7/a8: AC-strategy candidate costs and the greedy hierarchical merge.
//
// Candidate cost: src/codec/ac_strategy.cpp:823-994 (EstimateAcStrategyCost)
// with ComputeQuantNormUnchecked (:103-130) and the CPU DCT
// (src/codec/dct.cpp:135-230). The reference transforms in double precision
// with sequential sums and rounds to float at the end of each pass; the
// kernel does the same (FP64 SIMT, same summation order, no FMA contraction),
// so every cost is bit-identical to the reference's.
//
// Merge: src/codec/ac_strategy.cpp:340-773 (TryMerge,
// FindBestFirstLevelDivision, SearchTile) over all 64x64 tiles. The
// reference's CUDA path evaluates the candidates on the GPU, copies the cost
// table to the host and merges there (src/gpu/ops/ac_strategy_search.cpp:
// 626-740); here the merge runs on the device, one thread per tile, so the
// strategy grid never leaves HBM.
//
// Work layout: one kernel instantiation per transform family <W, H>; each CTA
// of 384 threads evaluates K = 1024 / (W*H) candidates (all three channels)
// entirely in shared memory: pixels -> FP64 row pass -> FP64 column pass ->
// quantize -> FP64 inverse row/column passes -> weighted loss. Each FP64
// pass gives every thread one 8-output chunk of one line, with the length-8
// and length-16 bases in constant memory and the length-32 basis staged in
// shared memory (line_dct.cuh). The reference's
// order-dependent float sums (magnitude cost, pixel loss) are done by one
// thread per (candidate, channel) in the reference's order.

#include <algorithm>
#include <cmath>
#include <cstring>

#include <cuda_bf16.h>

#include "common.cuh"
#include "host_util.h"
#include "fan.h"
#include "line_dct.cuh"
#include "tables.h"
#include "umma.cuh"

namespace gjxl_b200 {
namespace {

// Strategy ids (reference src/core/ac_strategy.h:25-53).
constexpr int kDct8 = 0, kDct16x16 = 4, kDct32x32 = 5, kDct16x8 = 6, kDct8x16 = 7,
              kDct32x16 = 10, kDct16x32 = 11;

// The seven searched families in the reference's candidate-stage order
// (src/codec/ac_strategy_search_policy.h:21-29).
constexpr int kFamilyCount = 7;
constexpr int kFamilyStrategy[kFamilyCount] = {kDct8,     kDct16x8,  kDct8x16, kDct16x16,
                                               kDct32x16, kDct16x32, kDct32x32};
constexpr float kFamilyEntropy[kFamilyCount] = {1.0f, 1.21f, 1.21f, 1.34f, 1.49f, 1.49f, 1.48f};
// Covered blocks (width, height) and anchor steps (normal search).
constexpr int kFamilyCoveredW[kFamilyCount] = {1, 1, 2, 2, 2, 4, 4};
constexpr int kFamilyCoveredH[kFamilyCount] = {1, 2, 1, 2, 4, 2, 4};
constexpr int kFamilyStep[kFamilyCount] = {1, 1, 1, 1, 2, 2, 2};

__host__ __device__ constexpr int FamilyOfStrategy(int s) {
  return s == kDct8 ? 0 : s == kDct16x8 ? 1 : s == kDct8x16 ? 2 : s == kDct16x16 ? 3
       : s == kDct32x16 ? 4 : s == kDct16x32 ? 5 : s == kDct32x32 ? 6 : -1;
}

// One candidate of a same-strategy batch, AcStrategyCandidate's layout
// (src/gpu/ops/ac_strategy.h:27-42).
struct CandidateDesc {
  uint32_t block_x, block_y;
  float quant_norm, entropy_multiplier, cfl_x, cfl_b;
};

struct CostParams {
  const float* opsin;  // Gaborish-inverted padded XYB
  size_t stride, pitch;
  const float* quant_field;  // blocks_x x blocks_y, dense
  const float* pixel_mask;
  size_t mask_stride;
  const int8_t* y_to_x;  // color tiles, dense
  const int8_t* y_to_b;
  uint32_t blocks_x, blocks_y, tiles_x, tiles_y;
  float info_loss_multiplier, zeros_multiplier, cost_delta;
  float entropy_multiplier;
  int anchor_step;
  int local_x, local_y;  // local anchors per tile along x / y (full tile)
  const float* dequant;          // family table [3][N]
  const float* inverse_dequant;  // family table [3][N]
  float* costs;           // family plane, blocks_x x blocks_y (anchor positions)
  uint32_t* error;
  // Learned analysis mode: the tiles whose candidates of this family are
  // scored (raster indices) and their number. Null: every tile.
  const uint32_t* kept_tiles;
  const uint32_t* kept_count;
  // Candidate-batch form: candidate i is batch[i] and its cost goes to
  // batch_costs[i]. With batch_resident, the quant norm and CfL factors come
  // from quant_field / y_to_x / y_to_b as in the tile enumeration; otherwise
  // from the descriptor. A descriptor whose footprint leaves the image gets
  // a NaN cost.
  const CandidateDesc* batch;
  float* batch_costs;
  int batch_resident;
};

// Candidates scored: every tile's, or those of the kept tiles.
__device__ __forceinline__ uint32_t ScoredCandidates(const CostParams& p, uint32_t all) {
  return p.kept_count != nullptr ? *p.kept_count * (p.local_x * p.local_y) : all;
}
__device__ __forceinline__ uint32_t CandidateTile(const CostParams& p, uint32_t slot) {
  return p.kept_tiles != nullptr ? p.kept_tiles[slot] : slot;
}

template <int W, int H>
struct Shape {
  static constexpr int N = W * H;
  static constexpr int K = N >= 1024 ? 1 : 1024 / N;
  static constexpr int CW = W / 8, CH = H / 8;
  // AcStrategyInfo::coefficient_index (src/core/ac_strategy.h:103-113).
  __device__ static int Index(int v, int u) { return H < W ? v * W + u : u * H + v; }
};

// One CTA evaluates K = 1024 / N candidates, 3 channels each, with
// 3 * K * N / 8 = 384 threads: in each of the four transform passes every
// thread computes one 8-output chunk of one line (line_dct.cuh). Shared
// planes are [candidate * 3 + channel][row][column] with rows padded to
// W + 1 elements, so that threads on consecutive rows and threads on
// consecutive columns both hit distinct banks.
constexpr int kCostThreads = 384;

template <int W, int H, typename Acc = double>
struct CostLayout {
  static constexpr int N = W * H, K = 1024 / N, KC = 3 * K;
  using Batch = PlaneBatch<W, H, KC>;
  static constexpr int RowPitch = Batch::RowPitch;
  static constexpr int PlanePitch = Batch::PlanePitch;
  static constexpr int Planes = Batch::Elements;  // elements per padded buffer
  // Ordered-sum terms: one plane of N + 4 floats per (candidate, channel):
  // 16-byte aligned rows for 128-bit loads, and the summing threads (one per
  // plane, same index at the same time) of each quarter warp hit distinct
  // banks.
  static constexpr int TermPitch = N + 4;
  // Families with a length-32 side read that pass's basis from a shared copy
  // (the forward table through the forward passes, then the inverse table).
  static constexpr bool kStagedBasis = (W == 32 || H == 32) && sizeof(Acc) == 8;
  static constexpr int BasisDoubles = kStagedBasis ? 32 * 32 : 0;
  static constexpr size_t SharedBytes = static_cast<size_t>(BasisDoubles) * 8 +
                                        static_cast<size_t>(Planes) * (4 + 4 + sizeof(Acc)) +
                                        static_cast<size_t>(KC) * TermPitch * 4;
  static_assert(K * N <= Planes, "the pixel mask fits the residual buffer");
  static_assert(Batch::Items == kCostThreads, "one chunk per thread and pass");
};

// Sequential float sum t[0] + t[1] + ... + t[n-1] (the reference's loop
// order), read four terms at a time.
template <int kCount>
__device__ __forceinline__ float OrderedSum(const float* t) {
  float sum = 0.0f;
#pragma unroll 4
  for (int j = 0; j < kCount; j += 4) {
    const float4 v = *reinterpret_cast<const float4*>(t + j);
    sum += v.x;
    sum += v.y;
    sum += v.z;
    sum += v.w;
  }
  return sum;
}

// Sum of each plane's N terms by kThreads / KC threads per plane (a fixed
// pairwise order, not the reference's sequential one): the fast mode's
// magnitude and loss sums. Writes the sum of plane `tid / T` through `out`
// from its first thread.
template <int N, int KC, int kThreads, int kPitch, typename Out>
__device__ __forceinline__ void ParallelPlaneSums(const float* terms, int tid, Out out) {
  constexpr int T = kThreads / KC;
  static_assert(T * KC == kThreads && (T & (T - 1)) == 0 && T <= 32 && N % T == 0,
                "threads per plane: a power of two within a warp");
  const int plane = tid / T, part = tid % T;
  const float* t = terms + plane * kPitch + part * (N / T);
  float sum = 0.0f;
#pragma unroll 8
  for (int j = 0; j < N / T; ++j) sum += t[j];
#pragma unroll
  for (int o = T / 2; o >= 1; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (part == 0) out(plane, sum);
}

__device__ __forceinline__ int CeilLog2Nonzero(uint32_t v) {
  return v <= 1 ? 0 : 32 - __clz(v - 1);
}

// ComputeQuantNormUnchecked (ac_strategy.cpp:103-130) over the covered
// blocks of the transform anchored at (ax, ay).
template <int CW, int CH>
__device__ __forceinline__ float QuantNorm(const CostParams& p, int ax, int ay) {
  const float* q = p.quant_field;
  if (CW * CH == 1) return q[ay * p.blocks_x + ax];
  if (CW * CH == 2) {
    return CH == 2 ? fmaxf(q[ay * p.blocks_x + ax], q[(ay + 1) * p.blocks_x + ax])
                   : fmaxf(q[ay * p.blocks_x + ax], q[ay * p.blocks_x + ax + 1]);
  }
  float sum = 0.0f;
  for (int dy = 0; dy < CH; ++dy) {
    for (int dx = 0; dx < CW; ++dx) {
      float v = q[(ay + dy) * p.blocks_x + ax + dx];
      v *= v;
      v *= v;
      v *= v;
      sum += v * v;
    }
  }
  sum /= static_cast<float>(CW * CH);
  return FastPow2(FastLog2(sum) * (1.0f / 16.0f));
}

// The quantities of one candidate that the transform stage needs, loaded
// ahead of use: anchor block, the quant field over its covered blocks and
// the tile's CfL bytes.
template <int CW, int CH>
struct CandidateInputs {
  int ax = -1, ay = -1;
  float q[CW * CH];
  int y_to_x = 0, y_to_b = 0;
};

// Anchor of candidate `cand` of a family (the same enumeration as the FP64
// kernel: tiles in raster order, local anchors on the family's step), or
// ax = -1 where the candidate does not fit its tile; then the loads.
template <int CW, int CH>
__device__ __forceinline__ CandidateInputs<CW, CH> FetchCandidate(const CostParams& p,
                                                                 uint32_t cand,
                                                                 uint32_t candidate_count) {
  CandidateInputs<CW, CH> in;
  if (p.batch != nullptr) {
    // Candidate-batch form (the anchor only; quant norm and CfL below).
    if (cand < candidate_count) {
      const CandidateDesc d = p.batch[cand];
      if (d.block_x + CW <= p.blocks_x && d.block_y + CH <= p.blocks_y) {
        in.ax = static_cast<int>(d.block_x);
        in.ay = static_cast<int>(d.block_y);
      }
    }
    if (in.ax >= 0 && p.batch_resident) {
#pragma unroll
      for (int dy = 0; dy < CH; ++dy) {
#pragma unroll
        for (int dx = 0; dx < CW; ++dx) {
          in.q[dy * CW + dx] = __ldg(p.quant_field + (in.ay + dy) * p.blocks_x + in.ax + dx);
        }
      }
      const int tile_index = (in.ay / 8) * p.tiles_x + (in.ax / 8);
      in.y_to_x = p.y_to_x[tile_index];
      in.y_to_b = p.y_to_b[tile_index];
    }
    return in;
  }
  if (cand < candidate_count) {
    const uint32_t per_tile = p.local_x * p.local_y;
    const uint32_t tile = CandidateTile(p, cand / per_tile), local = cand % per_tile;
    const int tx = tile % p.tiles_x, ty = tile / p.tiles_x;
    const int lx = (local % p.local_x) * p.anchor_step;
    const int ly = (local / p.local_x) * p.anchor_step;
    const int tile_w = min(8, static_cast<int>(p.blocks_x) - tx * 8);
    const int tile_h = min(8, static_cast<int>(p.blocks_y) - ty * 8);
    if (lx + CW <= tile_w && ly + CH <= tile_h) {
      in.ax = tx * 8 + lx;
      in.ay = ty * 8 + ly;
    }
  }
  if (in.ax >= 0) {
#pragma unroll
    for (int dy = 0; dy < CH; ++dy) {
#pragma unroll
      for (int dx = 0; dx < CW; ++dx) {
        in.q[dy * CW + dx] = __ldg(p.quant_field + (in.ay + dy) * p.blocks_x + in.ax + dx);
      }
    }
    const int tile_index = (in.ay / 8) * p.tiles_x + (in.ax / 8);
    in.y_to_x = p.y_to_x[tile_index];
    in.y_to_b = p.y_to_b[tile_index];
  }
  return in;
}

// QuantNorm of loaded quant-field values (same arithmetic).
template <int CW, int CH>
__device__ __forceinline__ float QuantNormOf(const float (&q)[CW * CH]) {
  if (CW * CH == 1) return q[0];
  if (CW * CH == 2) return fmaxf(q[0], q[1]);
  float sum = 0.0f;
  for (int i = 0; i < CW * CH; ++i) {
    float v = q[i];
    v *= v;
    v *= v;
    v *= v;
    sum += v * v;
  }
  sum /= static_cast<float>(CW * CH);
  return FastPow2(FastLog2(sum) * (1.0f / 16.0f));
}

// The candidate's cost from its per-channel magnitude sums, nonzero counts
// and weighted-loss sums (EstimateAcStrategyCost, ac_strategy.cpp:960-994).
// kExactRoot: the eighth root as the reference rounds it (double pow);
// otherwise exp2(log2(x) / 8) in single precision (within a few ulp), for the
// fast mode.
template <int N, int kBlocks, bool kExactRoot = true>
__device__ __forceinline__ float CandidateCost(const CostParams& p, const float (&magnitude)[3],
                                               const uint32_t (&nonzero)[3],
                                               const float (&loss_sum)[3], float quant_norm,
                                               float entropy_multiplier) {
  const float kChannelMultiplier[3] = {2.0441408586549744e7f, 1.0f, 1.266770081387616f};
  float entropy = 0.0f, loss = 0.0f;
  for (int c = 0; c < 3; ++c) {
    loss += loss_sum[c] * kChannelMultiplier[c];
    entropy += p.cost_delta * magnitude[c];
    const int nonzero_bits = CeilLog2Nonzero(nonzero[c] + 1) + 1;
    entropy += p.zeros_multiplier *
               static_cast<float>(CeilLog2Nonzero(nonzero_bits + 17) + nonzero_bits);
    if (c == 0 && kBlocks >= 2) {
      const float weight = 1.0f + fminf(3.0f, static_cast<float>(kBlocks) / 8.0f);
      entropy *= weight;
      loss *= weight;
    }
  }
  const float normalized_loss = loss / static_cast<float>(N);
  // std::pow(float, 1/8): evaluated in double and rounded to float.
  const float root =
    kExactRoot ? static_cast<float>(pow(static_cast<double>(normalized_loss), 0.125))
               : (normalized_loss > 0.0f ? exp2f(log2f(normalized_loss) * 0.125f) : 0.0f);
  const float loss_cost = root * static_cast<float>(N) / quant_norm;
  return entropy * entropy_multiplier + p.info_loss_multiplier * loss_cost;
}

// Acc = double: the bit-exact restatement (FP64 products, separately
// rounded, sequential sums). Acc = float: the fast mode's FP32 passes for the
// 8-pixel families (fused multiply-adds on the bases rounded to float).
template <int W, int H, typename Acc>
__global__ void __launch_bounds__(kCostThreads, 3)
CandidateCostKernel(const __grid_constant__ CostParams p, uint32_t candidate_count) {
  using S = Shape<W, H>;
  using Lay = CostLayout<W, H, Acc>;
  constexpr bool kExact = sizeof(Acc) == 8;
  constexpr int N = S::N, K = Lay::K, KC = Lay::KC;
  static_assert(K == S::K, "candidates per CTA");
  static_assert(kExact || (W <= 16 && H <= 16), "FP32 passes cover lengths 8 and 16");
  extern __shared__ __align__(16) unsigned char smem[];
  double* basis = reinterpret_cast<double*>(smem);         // [32][32] staged length-32 basis
  Acc* T = reinterpret_cast<Acc*>(basis + Lay::BasisDoubles);  // [KC][H][W+1] row-pass results
  float* A = reinterpret_cast<float*>(T + Lay::Planes);    // [KC][H][W+1] pixels, residuals
  float* B = A + Lay::Planes;                              // [KC][H][W+1] coefficients, pixels
  float* terms = B + Lay::Planes;                          // [KC][N + 4] ordered sum terms
  float* mask = A;  // [K][H][W] pixel mask, once the inverse row pass has read A
  __shared__ int anchor_x[K], anchor_y[K];
  __shared__ float quant_norm[K], cfl[K][3];
  __shared__ float magnitude[K][3], loss_sum[K][3];
  __shared__ uint32_t nonzero[K][3];

  const int tid = threadIdx.x;
  // Anchors first (integer arithmetic only), so that the pixel loads can
  // start before the quant norms and CfL factors arrive.
  __shared__ float entropy[K];
  __shared__ int invalid[K];
  candidate_count = ScoredCandidates(p, candidate_count);
  if (blockIdx.x * K >= candidate_count) return;  // past the kept tiles' candidates
  if (tid < K) {
    const uint32_t cand = blockIdx.x * K + tid;
    int ax = -1, ay = -1;
    entropy[tid] = p.entropy_multiplier;
    invalid[tid] = 0;
    if (p.batch != nullptr) {
      if (cand < candidate_count) {
        const CandidateDesc d = p.batch[cand];
        entropy[tid] = d.entropy_multiplier;
        if (d.block_x + S::CW <= p.blocks_x && d.block_y + S::CH <= p.blocks_y) {
          ax = static_cast<int>(d.block_x);
          ay = static_cast<int>(d.block_y);
        } else {
          invalid[tid] = 1;
        }
      }
    } else if (cand < candidate_count) {
      const uint32_t per_tile = p.local_x * p.local_y;
      const uint32_t tile = CandidateTile(p, cand / per_tile), local = cand % per_tile;
      const int tx = tile % p.tiles_x, ty = tile / p.tiles_x;
      const int lx = (local % p.local_x) * p.anchor_step;
      const int ly = (local / p.local_x) * p.anchor_step;
      const int tile_w = min(8, static_cast<int>(p.blocks_x) - tx * 8);
      const int tile_h = min(8, static_cast<int>(p.blocks_y) - ty * 8);
      if (lx + S::CW <= tile_w && ly + S::CH <= tile_h) {
        ax = tx * 8 + lx;
        ay = ty * 8 + ly;
      }
    }
    anchor_x[tid] = ax;
    anchor_y[tid] = ay;
    magnitude[tid][0] = magnitude[tid][1] = magnitude[tid][2] = 0.0f;
    nonzero[tid][0] = nonzero[tid][1] = nonzero[tid][2] = 0;
  }
  __syncthreads();

  // Pixels into A (one W-float run of the source per row) and the forward
  // length-32 basis into `basis`: every load of a thread is issued before the
  // first store, so their latencies overlap.
  constexpr int kBasisLoads = (Lay::BasisDoubles / 2 + kCostThreads - 1) / kCostThreads;
  const double2* staged_forward = reinterpret_cast<const double2*>(kDctStagedForwardT32);
  const double2* staged_inverse = reinterpret_cast<const double2*>(kDctStagedInverse32);
  double2* basis2 = reinterpret_cast<double2*>(basis);
  {
    constexpr int kPixelLoads = KC * N / kCostThreads;
    float pixel[kPixelLoads];
    double2 table[kBasisLoads > 0 ? kBasisLoads : 1];
#pragma unroll
    for (int q = 0; q < kBasisLoads; ++q) {
      const int i = tid + q * kCostThreads;
      if (i < Lay::BasisDoubles / 2) table[q] = __ldg(staged_forward + i);
    }
#pragma unroll
    for (int q = 0; q < kPixelLoads; ++q) {
      const int i = tid + q * kCostThreads;
      const int kc = i / N, r = i % N, y = r / W, x = r % W, k = kc / 3, c = kc % 3;
      pixel[q] = anchor_x[k] < 0 ? 0.0f
               : p.opsin[c * p.pitch + static_cast<size_t>(anchor_y[k] * 8 + y) * p.stride +
                         anchor_x[k] * 8 + x];
    }
    // ComputeQuantNormUnchecked (ac_strategy.cpp:103-130) and the CfL
    // factors, while the loads above are in flight.
    if (tid < K && anchor_x[tid] >= 0 && p.batch != nullptr && !p.batch_resident) {
      const CandidateDesc d = p.batch[blockIdx.x * K + tid];
      quant_norm[tid] = d.quant_norm;
      cfl[tid][0] = d.cfl_x;
      cfl[tid][1] = 0.0f;
      cfl[tid][2] = d.cfl_b;
    } else if (tid < K && anchor_x[tid] >= 0) {
      const int ax = anchor_x[tid], ay = anchor_y[tid];
      const float qn = QuantNorm<S::CW, S::CH>(p, ax, ay);
      if (!(IsFinite(qn) && qn > 0.0f)) RaiseError(p.error, kErrorNonFiniteInput);
      quant_norm[tid] = qn;
      const int tile_index = (ay / 8) * p.tiles_x + (ax / 8);
      // ColorCorrelationMap::AcFactors (chroma_from_luma.cpp:412-432).
      cfl[tid][0] = static_cast<float>(p.y_to_x[tile_index]) / 84.0f;
      cfl[tid][1] = 0.0f;
      cfl[tid][2] = 1.0f + static_cast<float>(p.y_to_b[tile_index]) / 84.0f;
    }
#pragma unroll
    for (int q = 0; q < kPixelLoads; ++q) {
      const int i = tid + q * kCostThreads;
      const int kc = i / N, r = i % N, y = r / W, x = r % W;
      if (anchor_x[kc / 3] >= 0) A[kc * Lay::PlanePitch + y * Lay::RowPitch + x] = pixel[q];
    }
#pragma unroll
    for (int q = 0; q < kBasisLoads; ++q) {
      const int i = tid + q * kCostThreads;
      if (i < Lay::BasisDoubles / 2) basis2[i] = table[q];
    }
  }
  __syncthreads();

  // Forward DCT (ForwardDctCpu): rows into T, then columns into B.
  const auto present = [&](int plane) { return anchor_x[plane / 3] >= 0; };
  const double* staged = Lay::kStagedBasis ? basis : nullptr;
  if constexpr (kExact) {
    BatchRowPass<W, H, KC, true>(A, T, tid, kCostThreads, present, staged);
    __syncthreads();
    BatchColumnPass<W, H, KC, true>(T, B, tid, kCostThreads, present, staged);
  } else {
    BatchRowPassF<W, H, KC, true>(A, T, tid, kCostThreads, present);
    __syncthreads();
    BatchColumnPassF<W, H, KC, true>(T, B, tid, kCostThreads, present);
  }
  __syncthreads();

  // Quantize, coefficient j = coefficient_index(v, u) by coefficient:
  // residual coefficients into A at (v, u), sqrt terms into terms[j]. The
  // quantization weights of all of a thread's coefficients (and the inverse
  // length-32 basis, which replaces the forward one) are loaded first.
  {
    constexpr int kPerThread = KC * N / kCostThreads;
    float inv[kPerThread], dq[kPerThread];
    double2 table[kBasisLoads > 0 ? kBasisLoads : 1];
#pragma unroll
    for (int q = 0; q < kBasisLoads; ++q) {
      const int i = tid + q * kCostThreads;
      if (i < Lay::BasisDoubles / 2) table[q] = __ldg(staged_inverse + i);
    }
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
      const int i = tid + q * kCostThreads;
      const int c = (i / N) % 3, j = i % N;
      inv[q] = __ldg(p.inverse_dequant + c * N + j);
      dq[q] = __ldg(p.dequant + c * N + j);
    }
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
      const int i = tid + q * kCostThreads;
      const int kc = i / N, j = i % N, k = kc / 3, c = kc % 3;
      if (anchor_x[k] < 0) continue;
      const int v = H < W ? j / W : j % H, u = H < W ? j % W : j / H;
      const int at = v * Lay::RowPitch + u;
      const float decorrelated =
        B[kc * Lay::PlanePitch + at] - B[(k * 3 + 1) * Lay::PlanePitch + at] * cfl[k][c];
      const float scaled = decorrelated * inv[q] * quant_norm[k];
      const float rounded = roundf(scaled);
      const float difference = scaled - rounded;
      A[kc * Lay::PlanePitch + at] = dq[q] * difference;
      terms[kc * Lay::TermPitch + j] = sqrtf(fabsf(rounded));
      // A warp's 32 consecutive coefficients share (k, c) (N is a multiple
      // of 32 and every thread runs the same trip count): one count per warp.
      const unsigned nz = __ballot_sync(0xffffffffu, rounded != 0.0f);
      if ((tid & 31) == 0 && nz != 0u) {
        atomicAdd(&nonzero[k][c], static_cast<uint32_t>(__popc(nz)));
      }
    }
#pragma unroll
    for (int q = 0; q < kBasisLoads; ++q) {
      const int i = tid + q * kCostThreads;
      if (i < Lay::BasisDoubles / 2) basis2[i] = table[q];
    }
  }
  __syncthreads();

  // The pixel mask is loaded now and kept in registers until the inverse
  // row pass has read the residual out of A, where it then goes.
  constexpr int kMaskLoads = (K * N + kCostThreads - 1) / kCostThreads;
  float pmask[kMaskLoads];
#pragma unroll
  for (int q = 0; q < kMaskLoads; ++q) {
    const int i = tid + q * kCostThreads;
    const int k = i / N, r = i % N, y = r / W, x = r % W;
    pmask[q] = i >= K * N || anchor_x[k] < 0 ? 1.0f
             : p.pixel_mask[static_cast<size_t>(anchor_y[k] * 8 + y) * p.mask_stride +
                            anchor_x[k] * 8 + x];
  }

  // The exact mode's ordered magnitude sums (one thread per candidate and
  // channel) wait for the end, where they run beside the loss sums: summing
  // here would hold back those threads' share of the inverse passes. The
  // fast mode sums every plane with all threads now.
  if constexpr (!kExact) {
    ParallelPlaneSums<N, KC, kCostThreads, Lay::TermPitch>(
      terms, tid, [&](int plane, float sum) { magnitude[plane / 3][plane % 3] = sum; });
  }

  // Inverse DCT (InverseDctCpu): rows of the residual into T, columns into B.
  if constexpr (kExact) {
    BatchRowPass<W, H, KC, false>(A, T, tid, kCostThreads, present, staged);
  } else {
    BatchRowPassF<W, H, KC, false>(A, T, tid, kCostThreads, present);
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kMaskLoads; ++q) {
    const int i = tid + q * kCostThreads;
    if (i < K * N && anchor_x[i / N] >= 0) mask[i] = pmask[q];
  }
  if constexpr (kExact) {
    BatchColumnPass<W, H, KC, false>(T, B, tid, kCostThreads, present, staged);
  } else {
    BatchColumnPassF<W, H, KC, false>(T, B, tid, kCostThreads, present);
  }
  __syncthreads();

  // Weighted eighth powers in pixel order; the exact mode keeps them in the
  // row-pass buffer (free once the column pass has read it), as `terms`
  // still holds the magnitude terms.
  float* loss_terms = kExact ? reinterpret_cast<float*>(T) : terms;
  static_assert(!kExact || 2 * Lay::Planes >= KC * Lay::TermPitch, "loss terms fit T");
  for (int i = tid; i < KC * N; i += kCostThreads) {
    const int kc = i / N, r = i % N, y = r / W, x = r % W, k = kc / 3, c = kc % 3;
    if (anchor_x[k] < 0) continue;
    const float m = mask[k * N + r];
    if (!(IsFinite(m) && m > 0.0f)) RaiseError(p.error, kErrorNonFiniteInput);
    const float offset = c == 0 ? 12.0f : c == 1 ? 0.0f : 4.0f;
    float weighted = (m + offset) * B[kc * Lay::PlanePitch + y * Lay::RowPitch + x];
    weighted *= weighted;
    weighted *= weighted;
    weighted *= weighted;
    loss_terms[kc * Lay::TermPitch + r] = weighted;
  }
  __syncthreads();

  if constexpr (kExact) {
    // One code path for both kinds of sum, so that a warp holding threads
    // of both runs them side by side.
    static_assert(2 * KC <= kCostThreads, "one thread per ordered sum");
    const bool loss = tid >= KC;
    const int plane = loss ? tid - KC : tid;
    if (tid < 2 * KC && anchor_x[plane / 3] >= 0) {
      const float sum = OrderedSum<N>((loss ? loss_terms : terms) + plane * Lay::TermPitch);
      (loss ? &loss_sum[0][0] : &magnitude[0][0])[plane] = sum;
    }
  } else {
    ParallelPlaneSums<N, KC, kCostThreads, Lay::TermPitch>(
      terms, tid, [&](int plane, float sum) { loss_sum[plane / 3][plane % 3] = sum; });
  }
  __syncthreads();

  if (tid < K && anchor_x[tid] >= 0) {
    const float mag[3] = {magnitude[tid][0], magnitude[tid][1], magnitude[tid][2]};
    const uint32_t nz[3] = {nonzero[tid][0], nonzero[tid][1], nonzero[tid][2]};
    const float ls[3] = {loss_sum[tid][0], loss_sum[tid][1], loss_sum[tid][2]};
    const float result = CandidateCost<N, S::CW * S::CH, kExact>(p, mag, nz, ls, quant_norm[tid],
                                                                  entropy[tid]);
    if (p.batch != nullptr) {
      p.batch_costs[blockIdx.x * K + tid] = result;
    } else {
      if (!(IsFinite(result) && result >= 0.0f)) RaiseError(p.error, kErrorNonFiniteOutput);
      p.costs[anchor_y[tid] * p.blocks_x + anchor_x[tid]] = result;
    }
  } else if (tid < K && invalid[tid]) {
    p.batch_costs[blockIdx.x * K + tid] = __int_as_float(0x7fc00000);
  }
}

// ---------------------------------------------------------------------------
// Tensor-core candidate costs (the fast precision mode) for the families
// whose sides are 16 or 32 pixels.
//
// The same cost as CandidateCostKernel, with the four separable transform
// passes as tcgen05 MMAs (bf16 operands, f32 accumulation in tensor memory)
// instead of FP64 products. Every operand is split into three bf16 pieces
// (x = hi + mid + lo, each the bf16 rounding of what remains), and every
// product is the sum of the six piece products whose orders of magnitude
// reach 2^-24 of the leading one (hi*hi, hi*mid, mid*hi, hi*lo, mid*mid,
// lo*hi): the split-bf16 form of an FP32 product. The CfL subtraction is
// applied to the pixels before the forward transform (the transform is
// linear, so this equals the reference's subtraction of the luma
// coefficients up to rounding), and every channel is then independent.
//
// Work unit: G = 128 / min(W, H) candidates, one channel at a time, so that
// each pass is one or two M = 128 tiles. Rows and operand layouts per pass
// (P pixels, T row-pass result, C coefficients, R quantized residual, E
// pixel error; u/v horizontal/vertical frequency, x/y pixel):
//   1  rows (cand, y)  K = x   N = u   A K-major    from the staged pixels
//   2  rows (cand, u)  K = y   N = v   A MN-major   (written from pass 1)
//   3  rows (cand, v)  K = u   N = x   A MN-major   (written from pass 2)
//   4  rows (cand, x)  K = v   N = y   A MN-major   (written from pass 3)
// A thread owns one accumulator row (tensor-memory lane) per tile and writes
// its row's values as 16-byte runs of the next operand: the transposes
// between passes are absorbed by the MN-major operand mode.

constexpr int kTcThreads = 128;
constexpr int kTcSplits = 3;
constexpr int kTcProducts = 6;
__device__ constexpr int kTcProductA[kTcProducts] = {0, 0, 1, 0, 1, 2};
__device__ constexpr int kTcProductB[kTcProducts] = {0, 1, 0, 2, 1, 0};
constexpr uint32_t kTcWaitPolls = 1u << 22;

template <int W, int H>
struct TcLayout {
  static constexpr int N = W * H;
  static constexpr int G = 128 / (W < H ? W : H);  // candidates per unit
  static constexpr int R1 = G * H, R2 = G * W;      // rows of passes 1/3 and 2/4
  static constexpr int T1 = R1 / 128, T2 = R2 / 128;
  static constexpr int kOperandBytes = G * N * 2;   // one bf16 piece of one A operand
  static constexpr int kSquare = W == H;
  // Basis tables (B operands, K-major [n / 8][k / 8][8][8] bf16): forward and
  // inverse for the width, and for the height unless the family is square.
  static constexpr int kTableBytesW = W * W * 2, kTableBytesH = H * H * 2;
  static constexpr int kTablesBytes =
    kTcSplits * 2 * (kTableBytesW + (kSquare ? 0 : kTableBytesH));
  // Quantization weights {inverse, dequant} of the family, [channel][v][u].
  static constexpr int kWeightsBytes = 3 * N * 8;
  // One operand buffer serves all four passes: pass k's operand is dead once
  // its MMA completed, before the epilogue writes pass k + 1's operand.
  static constexpr size_t SharedBytes = static_cast<size_t>(kTcSplits) * kOperandBytes +
                                        kTablesBytes + kWeightsBytes;
  static constexpr uint32_t kTmemColumns = 32;
  static_assert(T1 * W <= 32 && T2 * H <= 32, "every pass accumulates within 32 columns");
  static_assert(R1 % 128 == 0 && R2 % 128 == 0, "whole M = 128 tiles");
};

// Square root of a nonnegative float by the hardware approximation (within
// 2 ulp); the fast mode's magnitude terms sqrt|q| of integer-valued q.
__device__ __forceinline__ float ApproxSqrt(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Splits 8 floats into three bf16 pieces and stores each piece's 16 bytes
// at piece_base[s] + offset.
__device__ __forceinline__ void StoreSplit8(const float (&v)[8], unsigned char* const (&base)[3],
                                            int offset) {
  uint32_t hi[4], mid[4], lo[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    const float r0 = v[2 * i] - __low2float(h), r1 = v[2 * i + 1] - __high2float(h);
    const __nv_bfloat162 m = __floats2bfloat162_rn(r0, r1);
    const __nv_bfloat162 l = __floats2bfloat162_rn(r0 - __low2float(m), r1 - __high2float(m));
    hi[i] = *reinterpret_cast<const uint32_t*>(&h);
    mid[i] = *reinterpret_cast<const uint32_t*>(&m);
    lo[i] = *reinterpret_cast<const uint32_t*>(&l);
  }
  *reinterpret_cast<uint4*>(base[0] + offset) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  *reinterpret_cast<uint4*>(base[1] + offset) = make_uint4(mid[0], mid[1], mid[2], mid[3]);
  *reinterpret_cast<uint4*>(base[2] + offset) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

// Byte offset of element (n, k) in a K-major [n / 8][k / 8][8][8] bf16 table.
template <int K>
__device__ __forceinline__ int KMajorOffset(int n, int k) {
  return (n >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
}

// One table of L x L basis values (from the exact double tables) in its three
// bf16 pieces: element (n, k) = forward[n * L + k] (frequency n, sample k) or
// inverse[k * L + n] (frequency k, sample n).
template <int L, bool kForward>
__device__ void StageBasis(unsigned char* table, int tid) {
  for (int i = tid; i < L * L; i += kTcThreads) {
    const int n = i / L, k = i % L;
    const double value = kForward ? DctBasis<L, true>(n * L + k) : DctBasis<L, false>(k * L + n);
    const __nv_bfloat16 hi = __double2bfloat16(value);
    const double r1 = value - static_cast<double>(__bfloat162float(hi));
    const __nv_bfloat16 mid = __double2bfloat16(r1);
    const double r2 = r1 - static_cast<double>(__bfloat162float(mid));
    const __nv_bfloat16 lo = __double2bfloat16(r2);
    const int at = KMajorOffset<L>(n, k);
    *reinterpret_cast<__nv_bfloat16*>(table + at) = hi;
    *reinterpret_cast<__nv_bfloat16*>(table + L * L * 2 + at) = mid;
    *reinterpret_cast<__nv_bfloat16*>(table + 2 * L * L * 2 + at) = lo;
  }
}

// Issues the six piece products of one pass over `tiles` M = 128 tiles and
// `kchunks` K = 16 chunks, then commits to `barrier` (one thread).
__device__ __forceinline__ void IssuePass(uint32_t tmem, int n_out, int tiles, int kchunks,
                                          uint32_t a_base, int a_piece_bytes, int a_tile_bytes,
                                          int a_kchunk_bytes, uint32_t a_lbo, uint32_t a_sbo,
                                          bool a_mn_major, uint32_t b_base, int b_piece_bytes,
                                          uint32_t b_sbo, uint64_t* barrier) {
  const uint32_t instr = umma::InstrBf16F32(128, n_out, a_mn_major, false);
  for (int tile = 0; tile < tiles; ++tile) {
    for (int kc = 0; kc < kchunks; ++kc) {
#pragma unroll
      for (int q = 0; q < kTcProducts; ++q) {
        const uint64_t a = umma::Descriptor(
          a_base + kTcProductA[q] * a_piece_bytes + tile * a_tile_bytes + kc * a_kchunk_bytes,
          a_lbo, a_sbo);
        const uint64_t b =
          umma::Descriptor(b_base + kTcProductB[q] * b_piece_bytes + kc * 256, 128, b_sbo);
        umma::Mma(tmem + tile * n_out, a, b, instr, kc > 0 || q > 0);
      }
    }
  }
  umma::Commit(barrier);
}

template <int W, int H>
__global__ void __launch_bounds__(kTcThreads)
CandidateCostTcKernel(const __grid_constant__ CostParams p, uint32_t candidate_count) {
  using S = Shape<W, H>;
  using L = TcLayout<W, H>;
  constexpr int N = S::N, G = L::G, R1 = L::R1, R2 = L::R2, T1 = L::T1, T2 = L::T2;
  extern __shared__ __align__(128) unsigned char tc_smem[];
  unsigned char* operand = tc_smem;                          // A1..A4, three pieces
  unsigned char* tables = tc_smem + kTcSplits * L::kOperandBytes;
  float2* weights = reinterpret_cast<float2*>(tables + L::kTablesBytes);
  unsigned char* fwdW = tables;
  unsigned char* invW = fwdW + kTcSplits * L::kTableBytesW;
  unsigned char* fwdH = L::kSquare ? fwdW : invW + kTcSplits * L::kTableBytesW;
  unsigned char* invH = L::kSquare ? invW : fwdH + kTcSplits * L::kTableBytesH;
  __shared__ __align__(8) uint64_t barrier;
  __shared__ uint32_t tmem_slot;
  __shared__ int anchor_x[G], anchor_y[G];
  __shared__ float quant_norm[G], cfl[G][3];
  __shared__ float magnitude[G][3], loss_sum[G][3];
  __shared__ uint32_t nonzero[G][3];
  __shared__ float entropy[G];
  __shared__ int invalid[G];
  __shared__ int aborted;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) umma::Allocate(&tmem_slot, L::kTmemColumns);
  if (tid == 0) {
    umma::InitBarrier(&barrier, 1);
    aborted = 0;
  }
  StageBasis<W, true>(fwdW, tid);
  StageBasis<W, false>(invW, tid);
  if constexpr (!L::kSquare) {
    StageBasis<H, true>(fwdH, tid);
    StageBasis<H, false>(invH, tid);
  }
  // The quantization weights, [c][v][u]: the threads of one epilogue row
  // group (consecutive u) read consecutive words.
  for (int i = tid; i < 3 * N; i += kTcThreads) {
    const int c = i / N, v = (i % N) / W, u = i % W;
    const int index = c * N + S::Index(v, u);
    weights[i] = make_float2(__ldg(p.inverse_dequant + index), __ldg(p.dequant + index));
  }
  umma::FenceBeforeSync();
  __syncthreads();
  umma::FenceAfterSync();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = tmem + (static_cast<uint32_t>(warp * 32) << 16);
  uint32_t phase = 0;
  unsigned char* const pieces[3] = {operand, operand + L::kOperandBytes,
                                     operand + 2 * L::kOperandBytes};
  const uint32_t address = umma::SmemAddress(operand);
  // Leading (K) byte offsets of the MN-major operands.
  constexpr uint32_t kLbo2 = (R2 / 8) * 128, kLbo3 = (R1 / 8) * 128, kLbo4 = (R2 / 8) * 128;

  // Waits for the pass just committed. A timeout in any thread stops the
  // whole CTA (the decision is CTA-uniform, so no thread is left at a
  // barrier the others skip).
  const auto wait_pass = [&]() -> bool {
    const bool ok = umma::WaitParity(&barrier, phase, kTcWaitPolls);
    phase ^= 1u;
    umma::FenceAfterSync();
    const bool all = __syncthreads_and(ok ? 1 : 0) != 0;
    if (!all && tid == 0) {
      aborted = 1;
      RaiseError(p.error, kErrorInternal);
    }
    return all;
  };
  // Makes this thread's operand writes visible to the tensor core and lines
  // the CTA up before one thread issues the next pass.
  const auto operands_ready = [&]() {
    umma::FenceAsyncShared();
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
  };

  candidate_count = ScoredCandidates(p, candidate_count);
  const uint32_t units = (candidate_count + G - 1) / G;
  for (uint32_t unit = blockIdx.x; unit < units && !aborted; unit += gridDim.x) {
    if (tid < G) {
      const CandidateInputs<S::CW, S::CH> in =
        FetchCandidate<S::CW, S::CH>(p, unit * G + tid, candidate_count);
      anchor_x[tid] = in.ax;
      anchor_y[tid] = in.ay;
      float qn = 1.0f;
      entropy[tid] = p.entropy_multiplier;
      invalid[tid] = 0;
      if (p.batch != nullptr && unit * G + tid < candidate_count) {
        const CandidateDesc d = p.batch[unit * G + tid];
        entropy[tid] = d.entropy_multiplier;
        invalid[tid] = in.ax < 0 ? 1 : 0;
        if (in.ax >= 0 && !p.batch_resident) {
          qn = d.quant_norm;
          cfl[tid][0] = d.cfl_x;
          cfl[tid][1] = 0.0f;
          cfl[tid][2] = d.cfl_b;
        }
      }
      if (in.ax >= 0 && !(p.batch != nullptr && !p.batch_resident)) {
        qn = QuantNormOf<S::CW, S::CH>(in.q);
        if (!(IsFinite(qn) && qn > 0.0f)) RaiseError(p.error, kErrorNonFiniteInput);
        // ColorCorrelationMap::AcFactors (chroma_from_luma.cpp:412-432).
        cfl[tid][0] = static_cast<float>(in.y_to_x) / 84.0f;
        cfl[tid][1] = 0.0f;
        cfl[tid][2] = 1.0f + static_cast<float>(in.y_to_b) / 84.0f;
      }
      quant_norm[tid] = qn;
      for (int c = 0; c < 3; ++c) {
        magnitude[tid][c] = 0.0f;
        loss_sum[tid][c] = 0.0f;
        nonzero[tid][c] = 0;
      }
    }
    __syncthreads();

    for (int c = 0; c < 3 && !aborted; ++c) {
      // Stage: rows (cand, y) of the decorrelated pixels, K-major.
#pragma unroll
      for (int i = 0; i < T1; ++i) {
        const int r = i * 128 + tid, cand = r / H, y = r % H;
        const int ax = anchor_x[cand], ay = anchor_y[cand];
        float row[W];
        if (ax >= 0) {
          const size_t at = static_cast<size_t>(ay * 8 + y) * p.stride + ax * 8;
          const float4* src = reinterpret_cast<const float4*>(p.opsin + c * p.pitch + at);
#pragma unroll
          for (int q = 0; q < W / 4; ++q) {
            const float4 v = src[q];
            row[4 * q] = v.x;
            row[4 * q + 1] = v.y;
            row[4 * q + 2] = v.z;
            row[4 * q + 3] = v.w;
          }
          if (c != 1) {
            const float4* luma = reinterpret_cast<const float4*>(p.opsin + p.pitch + at);
            const float f = cfl[cand][c];
#pragma unroll
            for (int q = 0; q < W / 4; ++q) {
              const float4 v = luma[q];
              row[4 * q] = fmaf(-f, v.x, row[4 * q]);
              row[4 * q + 1] = fmaf(-f, v.y, row[4 * q + 1]);
              row[4 * q + 2] = fmaf(-f, v.z, row[4 * q + 2]);
              row[4 * q + 3] = fmaf(-f, v.w, row[4 * q + 3]);
            }
          }
        } else {
#pragma unroll
          for (int x = 0; x < W; ++x) row[x] = 0.0f;
        }
#pragma unroll
        for (int g = 0; g < W / 8; ++g) {
          float v[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) v[j] = row[g * 8 + j];
          StoreSplit8(v, pieces, KMajorOffset<W>(r, g * 8));
        }
      }
      operands_ready();
      // Pass 1: forward row transform.
      if (tid == 0) {
        IssuePass(tmem, W, T1, W / 16, address, L::kOperandBytes, 16 * (W / 8) * 128, 256, 128,
                  (W / 8) * 128, false, umma::SmemAddress(fwdW), L::kTableBytesW,
                  (W / 8) * 128, &barrier);
      }
      if (!wait_pass()) break;
      // Epilogue 1: T[(cand, y)][u] -> A2 (rows (cand, u), K = y, MN-major).
#pragma unroll
      for (int i = 0; i < T1; ++i) {
        const int r = i * 128 + tid, cand = r / H, y = r % H;
        float t[W];
        umma::Load<W>(lane_base + i * W, t);
#pragma unroll
        for (int g = 0; g < W / 8; ++g) {
          float v[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) v[j] = t[g * 8 + j];
          const int m = cand * W + g * 8;
          StoreSplit8(v, pieces, (y >> 3) * kLbo2 + (m >> 3) * 128 + (y & 7) * 16);
        }
      }
      operands_ready();
      // Pass 2: forward column transform.
      if (tid == 0) {
        IssuePass(tmem, H, T2, H / 16, address, L::kOperandBytes, 2048, 2 * kLbo2, kLbo2, 128,
                  true, umma::SmemAddress(fwdH), L::kTableBytesH, (H / 8) * 128, &barrier);
      }
      if (!wait_pass()) break;
      // Epilogue 2: quantize C[(cand, u)][v]; residual -> A3 (rows (cand, v),
      // K = u, MN-major); magnitude and nonzero sums per candidate.
      const float2* channel_weights = weights + c * N;
#pragma unroll
      for (int i = 0; i < T2; ++i) {
        const int r = i * 128 + tid, cand = r / W, u = r % W;
        float coef[H];
        umma::Load<H>(lane_base + i * H, coef);
        const float qn = quant_norm[cand];
        // All of the row's weights first: the operand stores below could
        // alias them as far as the compiler knows.
        float2 weight[H];
#pragma unroll
        for (int v = 0; v < H; ++v) weight[v] = channel_weights[v * W + u];
        float mag = 0.0f;
        uint32_t nz = 0;
#pragma unroll
        for (int g = 0; g < H / 8; ++g) {
          float res[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int v = g * 8 + j;
            const float scaled = coef[v] * weight[v].x * qn;
            const float rounded = roundf(scaled);
            res[j] = weight[v].y * (scaled - rounded);
            mag += ApproxSqrt(fabsf(rounded));
            nz += rounded != 0.0f ? 1u : 0u;
          }
          const int m = cand * H + g * 8;
          StoreSplit8(res, pieces, (u >> 3) * kLbo3 + (m >> 3) * 128 + (u & 7) * 16);
        }
        // The W rows of one candidate are W consecutive lanes.
#pragma unroll
        for (int o = W / 2; o >= 1; o >>= 1) {
          mag += __shfl_xor_sync(0xffffffffu, mag, o);
          nz += __shfl_xor_sync(0xffffffffu, nz, o);
        }
        if ((lane & (W - 1)) == 0 && anchor_x[cand] >= 0) {
          magnitude[cand][c] += mag;
          nonzero[cand][c] += nz;
        }
      }
      operands_ready();
      // Pass 3: inverse transform along the rows of the residual.
      if (tid == 0) {
        IssuePass(tmem, W, T1, W / 16, address, L::kOperandBytes, 2048, 2 * kLbo3, kLbo3, 128,
                  true, umma::SmemAddress(invW), L::kTableBytesW, (W / 8) * 128, &barrier);
      }
      if (!wait_pass()) break;
      // Epilogue 3: Z[(cand, v)][x] -> A4 (rows (cand, x), K = v, MN-major).
#pragma unroll
      for (int i = 0; i < T1; ++i) {
        const int r = i * 128 + tid, cand = r / H, v = r % H;
        float z[W];
        umma::Load<W>(lane_base + i * W, z);
#pragma unroll
        for (int g = 0; g < W / 8; ++g) {
          float e[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) e[j] = z[g * 8 + j];
          const int m = cand * W + g * 8;
          StoreSplit8(e, pieces, (v >> 3) * kLbo4 + (m >> 3) * 128 + (v & 7) * 16);
        }
      }
      operands_ready();
      // Pass 4: inverse transform along the columns. The pixel mask of this
      // thread's rows is loaded while it runs.
      if (tid == 0) {
        IssuePass(tmem, H, T2, H / 16, address, L::kOperandBytes, 2048, 2 * kLbo4, kLbo4, 128,
                  true, umma::SmemAddress(invH), L::kTableBytesH, (H / 8) * 128, &barrier);
      }
      float mask[T2][H];
#pragma unroll
      for (int i = 0; i < T2; ++i) {
        const int r = i * 128 + tid, cand = r / W, x = r % W;
        const int ax = anchor_x[cand], ay = anchor_y[cand];
#pragma unroll
        for (int y = 0; y < H; ++y) {
          mask[i][y] = ax < 0 ? 1.0f
                     : __ldg(p.pixel_mask + static_cast<size_t>(ay * 8 + y) * p.mask_stride +
                             ax * 8 + x);
        }
      }
      if (!wait_pass()) break;
      // Epilogue 4: weighted eighth powers of E[(cand, x)][y].
      const float offset = c == 0 ? 12.0f : c == 1 ? 0.0f : 4.0f;
#pragma unroll
      for (int i = 0; i < T2; ++i) {
        const int r = i * 128 + tid, cand = r / W;
        float e[H];
        umma::Load<H>(lane_base + i * H, e);
        float loss = 0.0f;
        bool finite = true;
#pragma unroll
        for (int y = 0; y < H; ++y) {
          const float m = mask[i][y];
          finite &= IsFinite(m) && m > 0.0f;
          float weighted = (m + offset) * e[y];
          weighted *= weighted;
          weighted *= weighted;
          weighted *= weighted;
          loss += weighted;
        }
        if (!finite) RaiseError(p.error, kErrorNonFiniteInput);
#pragma unroll
        for (int o = W / 2; o >= 1; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
        if ((lane & (W - 1)) == 0 && anchor_x[cand] >= 0) loss_sum[cand][c] += loss;
      }
    }
    __syncthreads();
    if (!aborted && tid < G && anchor_x[tid] >= 0) {
      const float mag[3] = {magnitude[tid][0], magnitude[tid][1], magnitude[tid][2]};
      const uint32_t nz[3] = {nonzero[tid][0], nonzero[tid][1], nonzero[tid][2]};
      const float ls[3] = {loss_sum[tid][0], loss_sum[tid][1], loss_sum[tid][2]};
      const float result =
        CandidateCost<N, S::CW * S::CH, false>(p, mag, nz, ls, quant_norm[tid], entropy[tid]);
      if (p.batch != nullptr) {
        p.batch_costs[unit * G + tid] = result;
      } else {
        if (!(IsFinite(result) && result >= 0.0f)) RaiseError(p.error, kErrorNonFiniteOutput);
        p.costs[anchor_y[tid] * p.blocks_x + anchor_x[tid]] = result;
      }
    } else if (!aborted && tid < G && invalid[tid]) {
      p.batch_costs[unit * G + tid] = __int_as_float(0x7fc00000);
    }
    __syncthreads();
  }
  // A CTA that gave up on a pass waits once more (bounded) for the tensor
  // core to finish with its tensor memory before releasing it.
  if (aborted) umma::WaitParity(&barrier, phase ^ 1u, kTcWaitPolls);
  umma::FenceBeforeSync();
  __syncthreads();
  umma::FenceAfterSync();
  if (warp == 0) umma::Deallocate(tmem, L::kTmemColumns);
}

// ---------------------------------------------------------------------------
// Greedy merge (one thread per 64x64 tile).

struct SearchParams {
  const float* costs;  // [7][blocks] family planes
  uint32_t blocks_x, blocks_y, tiles_x, tiles_y;
  float baseline_multiplier;  // DCT8 cost multiplier
  int dct32_step;
  uint8_t* cells;  // blocks_x x blocks_y, (strategy << 1) | anchor
  uint32_t* error;
};

__device__ __forceinline__ int CoveredW(int s) {
  return s == kDct16x16 ? 2 : s == kDct32x32 ? 4 : s == kDct8x16 ? 2 : s == kDct32x16 ? 2
       : s == kDct16x32 ? 4 : 1;
}
__device__ __forceinline__ int CoveredH(int s) {
  return s == kDct16x16 ? 2 : s == kDct32x32 ? 4 : s == kDct16x8 ? 2 : s == kDct32x16 ? 4
       : s == kDct16x32 ? 2 : 1;
}

struct TileState {
  uint8_t cell[64];
  float cost[64];
  uint8_t priority[64];
  int tile_w, tile_h;
  int bx0, by0;
};

__device__ __forceinline__ uint8_t Encode(int s, bool anchor) {
  return static_cast<uint8_t>((s << 1) | (anchor ? 1 : 0));
}

__device__ void SetCells(TileState& t, int lx, int ly, int s) {
  const int cw = CoveredW(s), ch = CoveredH(s);
  for (int dy = 0; dy < ch; ++dy)
    for (int dx = 0; dx < cw; ++dx) t.cell[(ly + dy) * 8 + lx + dx] = Encode(s, dx == 0 && dy == 0);
}

// SearchGrid::CrossesHorizontalBoundary / CrossesVerticalBoundary
// (ac_strategy.cpp:155-200), restricted to the tile (which they never leave).
__device__ bool CrossesHorizontal(const TileState& t, int start_x, int y, int end_x) {
  if (start_x >= t.tile_w || y >= t.tile_h || y % 8 == 0) return false;
  end_x = min(end_x, t.tile_w);
  while (start_x != 0 && !(t.cell[y * 8 + start_x] & 1)) --start_x;
  for (int x = start_x; x < end_x;) {
    const uint8_t c = t.cell[y * 8 + x];
    if (!(c & 1)) return true;
    x += CoveredW(c >> 1);
  }
  return false;
}

__device__ bool CrossesVertical(const TileState& t, int x, int start_y, int end_y) {
  if (x >= t.tile_w || start_y >= t.tile_h || x % 8 == 0) return false;
  end_y = min(end_y, t.tile_h);
  while (start_y != 0 && !(t.cell[start_y * 8 + x] & 1)) --start_y;
  for (int y = start_y; y < end_y;) {
    const uint8_t c = t.cell[y * 8 + x];
    if (!(c & 1)) return true;
    y += CoveredH(c >> 1);
  }
  return false;
}

__device__ float Cost(const SearchParams& p, const TileState& t, int s, int lx, int ly) {
  const int f = FamilyOfStrategy(s);
  const size_t blocks = static_cast<size_t>(p.blocks_x) * p.blocks_y;
  const float v = p.costs[f * blocks + static_cast<size_t>(t.by0 + ly) * p.blocks_x + t.bx0 + lx];
  if (!(IsFinite(v) && v >= 0.0f)) RaiseError(p.error, kErrorInternal);
  return v;
}

__device__ void SetCost(TileState& t, int lx, int ly, int s, float cost) {
  const int cw = CoveredW(s), ch = CoveredH(s);
  for (int dy = 0; dy < ch; ++dy)
    for (int dx = 0; dx < cw; ++dx) t.cost[(ly + dy) * 8 + lx + dx] = 0.0f;
  t.cost[ly * 8 + lx] = cost;
}

// TryMerge (ac_strategy.cpp:340-386).
__device__ void TryMerge(const SearchParams& p, TileState& t, int s, int lx, int ly,
                         uint8_t priority) {
  const int cw = CoveredW(s), ch = CoveredH(s);
  float current = 0.0f;
  for (int dy = 0; dy < ch; ++dy) {
    for (int dx = 0; dx < cw; ++dx) {
      const int i = (ly + dy) * 8 + lx + dx;
      if (t.priority[i] >= priority) return;
      current += t.cost[i];
    }
  }
  const float candidate = Cost(p, t, s, lx, ly);
  if (!(candidate < current)) return;
  for (int dy = 0; dy < ch; ++dy) {
    for (int dx = 0; dx < cw; ++dx) {
      const int i = (ly + dy) * 8 + lx + dx;
      t.cost[i] = 0.0f;
      t.priority[i] = priority;
    }
  }
  SetCells(t, lx, ly, s);
  t.cost[ly * 8 + lx] = candidate;
}

// FindBestFirstLevelDivision (ac_strategy.cpp:406-589).
__device__ void FirstLevelDivision(const SearchParams& p, TileState& t, int blocks, int lx,
                                   int ly) {
  const int half = blocks / 2;
  if (CrossesHorizontal(t, lx, ly, lx + blocks) ||
      CrossesHorizontal(t, lx, ly + blocks, lx + blocks) ||
      CrossesVertical(t, lx, ly, ly + blocks) ||
      CrossesVertical(t, lx + blocks, ly, ly + blocks)) {
    return;
  }
  const bool allow_vertical = !CrossesVertical(t, lx + half, ly, ly + blocks);
  const bool allow_horizontal = !CrossesHorizontal(t, lx, ly + half, lx + blocks);
  float quadrant[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
  for (int dy = 0; dy < blocks; ++dy)
    for (int dx = 0; dx < blocks; ++dx)
      quadrant[dy / half][dx / half] += t.cost[(ly + dy) * 8 + lx + dx];
  const float kUnavailable = 3.40282347e+38f;
  float vl = kUnavailable, vr = kUnavailable, ht = kUnavailable, hb = kUnavailable;
  const int vs = blocks == 2 ? kDct16x8 : kDct32x16;
  const int hs = blocks == 2 ? kDct8x16 : kDct16x32;
  const int ss = blocks == 2 ? kDct16x16 : kDct32x32;
  if (allow_vertical) {
    if ((t.cell[ly * 8 + lx] >> 1) != vs) vl = Cost(p, t, vs, lx, ly);
    if ((t.cell[ly * 8 + lx + half] >> 1) != vs) vr = Cost(p, t, vs, lx + half, ly);
  }
  if (allow_horizontal) {
    if ((t.cell[ly * 8 + lx] >> 1) != hs) ht = Cost(p, t, hs, lx, ly);
    if ((t.cell[(ly + half) * 8 + lx] >> 1) != hs) hb = Cost(p, t, hs, lx, ly + half);
  }
  const float square = Cost(p, t, ss, lx, ly);
  const float vertical_cost = fminf(vl, quadrant[0][0] + quadrant[1][0]) +
                              fminf(vr, quadrant[0][1] + quadrant[1][1]);
  const float horizontal_cost = fminf(ht, quadrant[0][0] + quadrant[0][1]) +
                                fminf(hb, quadrant[1][0] + quadrant[1][1]);
  // ChooseFirstLevelDivision (ac_strategy_search_policy.h:69-83).
  if (square < vertical_cost && square < horizontal_cost) {
    SetCells(t, lx, ly, ss);
    SetCost(t, lx, ly, ss, square);
  } else if (vertical_cost < horizontal_cost) {
    if (vl < quadrant[0][0] + quadrant[1][0]) {
      SetCells(t, lx, ly, vs);
      SetCost(t, lx, ly, vs, vl);
    }
    if (vr < quadrant[0][1] + quadrant[1][1]) {
      SetCells(t, lx + half, ly, vs);
      SetCost(t, lx + half, ly, vs, vr);
    }
  } else {
    if (ht < quadrant[0][0] + quadrant[0][1]) {
      SetCells(t, lx, ly, hs);
      SetCost(t, lx, ly, hs, ht);
    }
    if (hb < quadrant[1][0] + quadrant[1][1]) {
      SetCells(t, lx, ly + half, hs);
      SetCost(t, lx, ly + half, hs, hb);
    }
  }
}

// SearchTile (ac_strategy.cpp:591-773).
__global__ void __launch_bounds__(64) SearchTileKernel(const __grid_constant__ SearchParams p) {
  const uint32_t tile = blockIdx.x * blockDim.x + threadIdx.x;
  if (tile >= p.tiles_x * p.tiles_y) return;
  TileState t;
  const int tx = tile % p.tiles_x, ty = tile / p.tiles_x;
  t.bx0 = tx * 8;
  t.by0 = ty * 8;
  t.tile_w = min(8, static_cast<int>(p.blocks_x) - t.bx0);
  t.tile_h = min(8, static_cast<int>(p.blocks_y) - t.by0);
  for (int i = 0; i < 64; ++i) {
    t.cell[i] = Encode(kDct8, true);
    t.cost[i] = 0.0f;
    t.priority[i] = 0;
  }
  const int w = t.tile_w, h = t.tile_h;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) t.cost[y * 8 + x] = Cost(p, t, kDct8, x, y) * p.baseline_multiplier;

  const int merge_strategy[4] = {kDct16x8, kDct8x16, kDct16x32, kDct32x16};
  const uint8_t merge_priority[4] = {2, 2, 4, 4};
  for (int m = 0; m < 4; ++m) {
    const int s = merge_strategy[m];
    const int cw = CoveredW(s), ch = CoveredH(s);
    for (int y = 0; y + ch <= h; y += ch) {
      for (int x = 0; x + cw <= w; x += cw) {
        if (y + 3 < h && x + 3 < w) {
          if (s == kDct16x32) {
            if ((y | x) % 4 == 0) FirstLevelDivision(p, t, 4, x, y);
            continue;
          }
          if (s == kDct32x16) continue;
        }
        if ((s == kDct16x32 && y % 4 != 0) || (s == kDct32x16 && x % 4 != 0)) continue;
        if (y + 1 < h && x + 1 < w) {
          if (s == kDct8x16) {
            if ((y | x) % 2 == 0) FirstLevelDivision(p, t, 2, x, y);
            continue;
          }
          if (s == kDct16x8) continue;
        }
        if ((s == kDct8x16 && y % 2 == 1) || (s == kDct16x8 && x % 2 == 1)) continue;
        TryMerge(p, t, s, x, y, merge_priority[m]);
      }
    }
  }
  for (int y = 0; y + 1 < h; ++y)
    for (int x = 0; x + 1 < w; ++x)
      if ((y | x) % 2 != 0) FirstLevelDivision(p, t, 2, x, y);
  for (int y = 0; y + 3 < h; y += p.dct32_step)
    for (int x = 0; x + 3 < w; x += p.dct32_step)
      if ((y | x) % 4 != 0) FirstLevelDivision(p, t, 4, x, y);

  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x)
      p.cells[static_cast<size_t>(t.by0 + y) * p.blocks_x + t.bx0 + x] = t.cell[y * 8 + x];
}

template <int W, int H, typename Acc = double>
int LaunchFamily(CostParams p, const DeviceTables& d, int family, cudaStream_t stream,
                 uint32_t batch_count = 0) {
  using S = Shape<W, H>;
  const int table = StrategyTableFamily(kFamilyStrategy[family]);
  const HostTables& h = GetHostTables();
  if (p.dequant == nullptr) {
    p.dequant = d.dequant + h.layout.offset[table];
    p.inverse_dequant = d.inverse_dequant + h.layout.offset[table];
  }
  p.entropy_multiplier = kFamilyEntropy[family];
  const int cw = kFamilyCoveredW[family], ch = kFamilyCoveredH[family];
  p.local_x = (8 - cw) / p.anchor_step + 1;
  p.local_y = (8 - ch) / p.anchor_step + 1;
  const uint32_t count = p.batch != nullptr
                           ? batch_count
                           : static_cast<uint32_t>(p.tiles_x * p.tiles_y * p.local_x * p.local_y);
  if (count == 0) return GJXL_B200_OK;
  const size_t smem = CostLayout<W, H, Acc>::SharedBytes;
  int status = CheckCuda(cudaFuncSetAttribute(CandidateCostKernel<W, H, Acc>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(smem)),
                         "ac_strategy smem attribute");
  if (status != GJXL_B200_OK) return status;
  const unsigned grid = (count + S::K - 1) / S::K;
  CandidateCostKernel<W, H, Acc><<<grid, kCostThreads, smem, stream>>>(p, count);
  return CheckLaunch("ac_strategy candidate costs");
}

// The tensor-core form of a 16/32-sided family: persistent CTAs (as many as
// fit on the device at once) walk the units of G candidates.
template <int W, int H>
int LaunchFamilyTc(CostParams p, const DeviceTables& d, int family, cudaStream_t stream,
                   uint32_t batch_count = 0) {
  using Lay = TcLayout<W, H>;
  const int table = StrategyTableFamily(kFamilyStrategy[family]);
  const HostTables& h = GetHostTables();
  if (p.dequant == nullptr) {
    p.dequant = d.dequant + h.layout.offset[table];
    p.inverse_dequant = d.inverse_dequant + h.layout.offset[table];
  }
  p.entropy_multiplier = kFamilyEntropy[family];
  const int cw = kFamilyCoveredW[family], ch = kFamilyCoveredH[family];
  p.local_x = (8 - cw) / p.anchor_step + 1;
  p.local_y = (8 - ch) / p.anchor_step + 1;
  const uint32_t count = p.batch != nullptr
                           ? batch_count
                           : static_cast<uint32_t>(p.tiles_x * p.tiles_y * p.local_x * p.local_y);
  if (count == 0) return GJXL_B200_OK;
  const size_t smem = Lay::SharedBytes;
  int status = CheckCuda(cudaFuncSetAttribute(CandidateCostTcKernel<W, H>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(smem)),
                         "ac_strategy tensor-core smem attribute");
  if (status != GJXL_B200_OK) return status;
  // All of the SM's unified memory for shared memory, so that the CTAs the
  // shared memory admits are all resident.
  status = CheckCuda(cudaFuncSetAttribute(CandidateCostTcKernel<W, H>,
                                          cudaFuncAttributePreferredSharedMemoryCarveout, 100),
                     "ac_strategy tensor-core carveout");
  if (status != GJXL_B200_OK) return status;
  int device = 0, sms = 0, smem_per_sm = 0;
  status = CheckCuda(cudaGetDevice(&device), "ac_strategy device");
  if (status == GJXL_B200_OK) {
    status = CheckCuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device),
                       "ac_strategy SM count");
  }
  if (status == GJXL_B200_OK) {
    status = CheckCuda(cudaDeviceGetAttribute(&smem_per_sm,
                                              cudaDevAttrMaxSharedMemoryPerMultiprocessor, device),
                       "ac_strategy shared memory per SM");
  }
  if (status != GJXL_B200_OK) return status;
  // Resident CTAs per SM, bounded by shared memory (with the static part and
  // the 1 KB the runtime reserves per CTA), registers (allocated in units of
  // 8 per thread), threads, and 16 CTAs of 32 tensor-memory columns in the
  // SM's 512, so that no CTA of this launch ever waits for tensor memory.
  // (The runtime's occupancy calculator reports one CTA per SM for kernels
  // that allocate tensor memory, which the hardware does not require.)
  cudaFuncAttributes attributes;
  status = CheckCuda(cudaFuncGetAttributes(&attributes, CandidateCostTcKernel<W, H>),
                     "ac_strategy attributes");
  if (status != GJXL_B200_OK) return status;
  const int per_cta = static_cast<int>(smem + attributes.sharedSizeBytes) + 1024;
  const int registers = ((attributes.numRegs + 7) / 8) * 8 * kTcThreads;
  const int per_sm = std::max(
    1, std::min({smem_per_sm / per_cta, 65536 / std::max(registers, 1), 2048 / kTcThreads, 16}));
  const uint32_t units = (count + Lay::G - 1) / Lay::G;
  const unsigned grid = std::max(1u, std::min<unsigned>(units, sms * per_sm));
  CandidateCostTcKernel<W, H><<<grid, kTcThreads, smem, stream>>>(p, count);
  return CheckLaunch("ac_strategy tensor-core candidate costs");
}

}  // namespace

size_t AcStrategyCostFloats(size_t blocks_x, size_t blocks_y) {
  return kFamilyCount * blocks_x * blocks_y;
}

int LaunchAcStrategyCosts(const float* opsin, size_t stride, size_t pitch, size_t pw, size_t ph,
                          const float* quant_field, const float* pixel_mask, size_t mask_stride,
                          const int8_t* y_to_x, const int8_t* y_to_b, float target, bool dense,
                          int precision, float* costs, uint32_t* error, cudaStream_t stream,
                          const StreamFan* fan, const uint32_t* kept_tiles,
                          const uint32_t* kept_counts) {
  DeviceTables d;
  int status = GetDeviceTables(&d);
  if (status != GJXL_B200_OK) return status;
  const size_t bx = pw / 8, by = ph / 8;
  // Reset the table so anchors that are never evaluated read as NaN.
  status = CheckCuda(cudaMemsetAsync(costs, 0xff, AcStrategyCostFloats(bx, by) * sizeof(float),
                                     stream), "ac_strategy memset");
  if (status != GJXL_B200_OK) return status;
  CostParams p;
  std::memset(&p, 0, sizeof(p));
  p.opsin = opsin;
  p.stride = stride;
  p.pitch = pitch;
  p.quant_field = quant_field;
  p.pixel_mask = pixel_mask;
  p.mask_stride = mask_stride;
  p.y_to_x = y_to_x;
  p.y_to_b = y_to_b;
  p.blocks_x = static_cast<uint32_t>(bx);
  p.blocks_y = static_cast<uint32_t>(by);
  p.tiles_x = static_cast<uint32_t>((bx + 7) / 8);
  p.tiles_y = static_cast<uint32_t>((by + 7) / 8);
  // Target-dependent constants (ac_strategy.cpp:880-888), with the host
  // C library's powf exactly as in the reference.
  const float kBias = 0.13731742964354549f;
  const float ratio = (target + kBias) / (1.0f + kBias);
  p.info_loss_multiplier = 1.2f * std::pow(ratio, 0.33677806662454718f);
  p.zeros_multiplier = 9.3089059022677905f * std::pow(ratio, 0.50990926717963703f);
  p.cost_delta = 10.833273317067883f * std::pow(ratio, 0.36702940662370243f);
  p.error = error;
  // The families are independent: with a fan they run side by side.
  if (status == GJXL_B200_OK) status = CheckCuda(FanFork(fan), "ac_strategy fork");
  for (int f = 0; f < kFamilyCount && status == GJXL_B200_OK; ++f) {
    const cudaStream_t fs = fan != nullptr ? fan->For(f) : stream;
    CostParams q = p;
    q.anchor_step = (dense && f >= 4) ? 1 : kFamilyStep[f];
    q.costs = costs + f * bx * by;
    if (kept_tiles != nullptr) {
      q.kept_tiles = kept_tiles + static_cast<size_t>(f) * p.tiles_x * p.tiles_y;
      q.kept_count = kept_counts + f;
    }
    const bool tensor = precision == GJXL_B200_PRECISION_FAST;
    switch (f) {
      case 0:
        status = tensor ? LaunchFamily<8, 8, float>(q, d, f, fs) : LaunchFamily<8, 8>(q, d, f, fs);
        break;
      case 1:
        status = tensor ? LaunchFamily<8, 16, float>(q, d, f, fs)
                        : LaunchFamily<8, 16>(q, d, f, fs);
        break;
      case 2:
        status = tensor ? LaunchFamily<16, 8, float>(q, d, f, fs)
                        : LaunchFamily<16, 8>(q, d, f, fs);
        break;
      case 3:
        status = tensor ? LaunchFamilyTc<16, 16>(q, d, f, fs) : LaunchFamily<16, 16>(q, d, f, fs);
        break;
      case 4:
        status = tensor ? LaunchFamilyTc<16, 32>(q, d, f, fs) : LaunchFamily<16, 32>(q, d, f, fs);
        break;
      case 5:
        status = tensor ? LaunchFamilyTc<32, 16>(q, d, f, fs) : LaunchFamily<32, 16>(q, d, f, fs);
        break;
      case 6:
        status = tensor ? LaunchFamilyTc<32, 32>(q, d, f, fs) : LaunchFamily<32, 32>(q, d, f, fs);
        break;
    }
  }
  const cudaError_t joined = FanJoin(fan);
  if (status == GJXL_B200_OK) status = CheckCuda(joined, "ac_strategy join");
  return status;
}

int LaunchAcStrategySearch(const float* costs, size_t pw, size_t ph, float target, bool dense,
                           uint8_t* cells, uint32_t* error, cudaStream_t stream) {
  SearchParams p;
  p.costs = costs;
  p.blocks_x = static_cast<uint32_t>(pw / 8);
  p.blocks_y = static_cast<uint32_t>(ph / 8);
  p.tiles_x = (p.blocks_x + 7) / 8;
  p.tiles_y = (p.blocks_y + 7) / 8;
  // SearchTile baseline multiplier (ac_strategy.cpp:612-617).
  p.baseline_multiplier = 1.0f + -0.4f / (target + 1.4f);
  p.dct32_step = dense ? 1 : 2;
  p.cells = cells;
  p.error = error;
  const unsigned tiles = p.tiles_x * p.tiles_y;
  SearchTileKernel<<<(tiles + 63) / 64, 64, 0, stream>>>(p);
  return CheckLaunch("ac_strategy search");
}

}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" size_t gjxl_b200_ac_strategy_cost_bytes(size_t padded_width, size_t padded_height) {
  return AcStrategyCostFloats(padded_width / 8, padded_height / 8) * sizeof(float);
}

extern "C" int gjxl_b200_ac_strategy_costs(
  const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch, size_t padded_width,
  size_t padded_height, const float* quant_field, const float* pixel_mask,
  size_t pixel_mask_stride, const int8_t* y_to_x, const int8_t* y_to_b,
  float butteraugli_target, int dense_dct32, int precision, float* costs,
  uint32_t* device_error, void* stream) {
  ClearLastError();
  if (opsin == nullptr || quant_field == nullptr || pixel_mask == nullptr || y_to_x == nullptr ||
      y_to_b == nullptr || costs == nullptr || padded_width % 8 || padded_height % 8 ||
      padded_width == 0 || padded_height == 0 || opsin_stride < padded_width ||
      opsin_plane_pitch < opsin_stride * padded_height || pixel_mask_stride < padded_width ||
      opsin_stride % 4 != 0 || opsin_plane_pitch % 4 != 0 || !Aligned16(opsin) ||
      !std::isfinite(butteraugli_target) || butteraugli_target <= 0.0f ||
      (precision != GJXL_B200_PRECISION_EXACT && precision != GJXL_B200_PRECISION_FAST) ||
      padded_width > (1u << 30) || padded_height > (1u << 30)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "ac_strategy_costs: invalid arguments");
  }
  return LaunchAcStrategyCosts(opsin, opsin_stride, opsin_plane_pitch, padded_width,
                               padded_height, quant_field, pixel_mask, pixel_mask_stride, y_to_x,
                               y_to_b, butteraugli_target, dense_dct32 != 0, precision, costs,
                               device_error, static_cast<cudaStream_t>(stream), nullptr,
                               nullptr, nullptr);
}

extern "C" int gjxl_b200_ac_strategy_search(
  const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch, size_t padded_width,
  size_t padded_height, const float* quant_field, const float* pixel_mask,
  size_t pixel_mask_stride, const int8_t* y_to_x, const int8_t* y_to_b,
  float butteraugli_target, int dense_dct32, int precision, float* costs, uint8_t* cells,
  uint32_t* device_error, void* stream) {
  int status = gjxl_b200_ac_strategy_costs(opsin, opsin_stride, opsin_plane_pitch, padded_width,
                                           padded_height, quant_field, pixel_mask,
                                           pixel_mask_stride, y_to_x, y_to_b,
                                           butteraugli_target, dense_dct32, precision, costs,
                                           device_error, stream);
  if (status != GJXL_B200_OK) return status;
  if (cells == nullptr) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "ac_strategy_search: cells is null");
  }
  return LaunchAcStrategySearch(costs, padded_width, padded_height, butteraugli_target,
                                dense_dct32 != 0, cells, device_error,
                                static_cast<cudaStream_t>(stream));
}

// Candidate-batch evaluation: GpuAcStrategyEvaluation::
// EvaluateAcStrategyCandidateBatches (src/gpu/ops/ac_strategy.h:118-170) for
// one same-strategy batch.
extern "C" int gjxl_b200_ac_strategy_candidate_costs(
  int strategy, const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch,
  const float* pixel_mask, size_t pixel_mask_stride, size_t padded_width, size_t padded_height,
  const void* candidates, size_t candidate_count, const float* matrices,
  const float* quant_field, const int8_t* y_to_x, const int8_t* y_to_b, float butteraugli_target,
  int precision, float* costs, uint32_t* device_error, void* stream) {
  ClearLastError();
  int family = -1;
  for (int f = 0; f < kFamilyCount; ++f)
    if (kFamilyStrategy[f] == strategy) family = f;
  if (opsin == nullptr || pixel_mask == nullptr || (candidate_count > 0 && candidates == nullptr) ||
      (candidate_count > 0 && costs == nullptr) || padded_width % 8 || padded_height % 8 ||
      padded_width == 0 || padded_height == 0 || opsin_stride < padded_width ||
      opsin_plane_pitch < opsin_stride * padded_height || pixel_mask_stride < padded_width ||
      candidate_count > (1u << 30) || !(butteraugli_target > 0.0f) ||
      (precision != GJXL_B200_PRECISION_EXACT && precision != GJXL_B200_PRECISION_FAST) ||
      ((quant_field == nullptr) != (y_to_x == nullptr) || (y_to_x == nullptr) != (y_to_b == nullptr)) ||
      !Aligned16(opsin)) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "ac_strategy_candidate_costs: invalid arguments");
  }
  if (family < 0) {
    return SetError(GJXL_B200_UNSUPPORTED,
                    "ac_strategy_candidate_costs: the 7 searched strategies are supported");
  }
  if (candidate_count == 0) return GJXL_B200_OK;
  DeviceTables d;
  int status = GetDeviceTables(&d);
  if (status != GJXL_B200_OK) return status;
  const size_t bx = padded_width / 8, by = padded_height / 8;
  CostParams p;
  std::memset(&p, 0, sizeof(p));
  p.opsin = opsin;
  p.stride = opsin_stride;
  p.pitch = opsin_plane_pitch;
  p.quant_field = quant_field;
  p.pixel_mask = pixel_mask;
  p.mask_stride = pixel_mask_stride;
  p.y_to_x = y_to_x;
  p.y_to_b = y_to_b;
  p.blocks_x = static_cast<uint32_t>(bx);
  p.blocks_y = static_cast<uint32_t>(by);
  p.tiles_x = static_cast<uint32_t>((bx + 7) / 8);
  p.tiles_y = static_cast<uint32_t>((by + 7) / 8);
  const float kBias = 0.13731742964354549f;
  const float ratio = (butteraugli_target + kBias) / (1.0f + kBias);
  p.info_loss_multiplier = 1.2f * std::pow(ratio, 0.33677806662454718f);
  p.zeros_multiplier = 9.3089059022677905f * std::pow(ratio, 0.50990926717963703f);
  p.cost_delta = 10.833273317067883f * std::pow(ratio, 0.36702940662370243f);
  p.error = device_error;
  p.anchor_step = 1;
  p.batch = static_cast<const CandidateDesc*>(candidates);
  p.batch_costs = costs;
  p.batch_resident = quant_field != nullptr ? 1 : 0;
  if (matrices != nullptr) {
    const size_t n = static_cast<size_t>(kFamilyCoveredW[family]) * kFamilyCoveredH[family] * 64;
    p.dequant = matrices;
    p.inverse_dequant = matrices + 3 * n;
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint32_t count = static_cast<uint32_t>(candidate_count);
  const bool tensor = precision == GJXL_B200_PRECISION_FAST;
  switch (family) {
    case 0: status = tensor ? LaunchFamily<8, 8, float>(p, d, 0, s, count) : LaunchFamily<8, 8>(p, d, 0, s, count); break;
    case 1: status = tensor ? LaunchFamily<8, 16, float>(p, d, 1, s, count) : LaunchFamily<8, 16>(p, d, 1, s, count); break;
    case 2: status = tensor ? LaunchFamily<16, 8, float>(p, d, 2, s, count) : LaunchFamily<16, 8>(p, d, 2, s, count); break;
    case 3: status = tensor ? LaunchFamilyTc<16, 16>(p, d, 3, s, count) : LaunchFamily<16, 16>(p, d, 3, s, count); break;
    case 4: status = tensor ? LaunchFamilyTc<16, 32>(p, d, 4, s, count) : LaunchFamily<16, 32>(p, d, 4, s, count); break;
    case 5: status = tensor ? LaunchFamilyTc<32, 16>(p, d, 5, s, count) : LaunchFamily<32, 16>(p, d, 5, s, count); break;
    default: status = tensor ? LaunchFamilyTc<32, 32>(p, d, 6, s, count) : LaunchFamily<32, 32>(p, d, 6, s, count); break;
  }
  return status;
}
