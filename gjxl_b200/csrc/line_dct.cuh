// Line passes of the reference CPU DCT (src/codec/dct.cpp:135-230) for the
// FP64 transform kernels.
//
// The reference transforms one W x H block as two 1-D passes of dense matrix
// products in double precision, each output one sequential sum
// `sum += sample[s] * basis[...]` over s = 0..L-1 (multiply and add rounded
// separately; the device code is built with --fmad=false). A *line* is the L
// samples one output depends on (a row of W for the row pass, a column of H
// for the column pass); a *chunk* is 8 consecutive outputs of one line.
//
// One thread computes one chunk: it streams the line's samples once from
// shared memory and keeps 8 independent double accumulators, so every sample
// load feeds 8 multiply-adds and the 8 chains give the FP64 pipe enough
// independent work. Callers map warps to chunks so that the chunk is
// warp-uniform. For lengths 8 and 16 the chunk is a template parameter and,
// fully unrolled, every basis value is a compile-time offset into constant
// memory that enters the multiply as a constant-bank operand. Length 32 keeps
// the sample loop rolled, because its fully unrolled code thrashes the
// instruction cache, and reads the basis with a runtime (warp-uniform) index:
// from a copy that the caller staged in shared memory, four 128-bit broadcast
// loads per sample, or else from constant memory.
#pragma once

#include "dct_basis.inc"

namespace gjxl_b200 {

// basis[frequency * L + sample] of the forward (DCT-II, 1/L scaled) or inverse
// (DCT-III) transform of length L.
template <int L, bool kForward>
__device__ __forceinline__ double DctBasis(int index) {
  if constexpr (kForward) {
    if constexpr (L == 8) return kDctForward8[index];
    if constexpr (L == 16) return kDctForward16[index];
    if constexpr (L == 32) return kDctForward32[index];
  } else {
    if constexpr (L == 8) return kDctInverse8[index];
    if constexpr (L == 16) return kDctInverse16[index];
    if constexpr (L == 32) return kDctInverse32[index];
  }
  return 0.0;
}

// Outputs k = C*8 .. C*8+7 of one line of length L:
//   forward: out[k] = sum_s in[s] * basis[k * L + s]   (k = frequency)
//   inverse: out[k] = sum_s in[s] * basis[s * L + k]   (k = sample, s = frequency)
// `in` advances by InStep elements per sample, `out` by OutStep per output.
template <int L, bool kForward, int C, int InStep, int OutStep, typename In, typename Out>
__device__ __forceinline__ void LineChunk(const In* __restrict__ in, Out* __restrict__ out) {
  double acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = 0.0;
#pragma unroll
  for (int s = 0; s < L; ++s) {
    const double v = static_cast<double>(in[s * InStep]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = C * 8 + j;
      acc[j] += v * DctBasis<L, kForward>(kForward ? k * L + s : s * L + k);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) out[j * OutStep] = static_cast<Out>(acc[j]);
}

// basis table laid out [s][k]: the transposed forward basis, or the inverse
// basis as stored.
template <int L, bool kForward>
__device__ __forceinline__ double DctTable(int index) {
  if constexpr (kForward) {
    if constexpr (L == 8) return kDctForwardT8[index];
    if constexpr (L == 16) return kDctForwardT16[index];
    if constexpr (L == 32) return kDctForwardT32[index];
  } else {
    if constexpr (L == 8) return kDctInverse8[index];
    if constexpr (L == 16) return kDctInverse16[index];
    if constexpr (L == 32) return kDctInverse32[index];
  }
  return 0.0;
}

// Outputs k = chunk*8 .. chunk*8+7 of one line of length L, reading the basis
// from constant memory with a runtime (warp-uniform) index:
// out[k] = sum_s in[s] * table[s * L + k]. The sample loop is only partly
// unrolled, so the code stays small.
template <int L, bool kForward, int InStep, int OutStep, typename In, typename Out>
__device__ __forceinline__ void LineChunkTable(int chunk, const In* __restrict__ in,
                                               Out* __restrict__ out) {
  double acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = 0.0;
#pragma unroll 4
  for (int s = 0; s < L; ++s) {
    const double v = static_cast<double>(in[s * InStep]);
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] += v * DctTable<L, kForward>(s * L + chunk * 8 + j);
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) out[j * OutStep] = static_cast<Out>(acc[j]);
}

// As LineChunkTable, with the basis table staged in shared memory by the
// caller (laid out [s][k], 16-byte aligned): every lane of the warp reads the
// same eight entries per sample, four 128-bit broadcast loads.
template <int L, int InStep, int OutStep, typename In, typename Out>
__device__ __forceinline__ void LineChunkShared(int chunk, const double* __restrict__ table,
                                                const In* __restrict__ in,
                                                Out* __restrict__ out) {
  double acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = 0.0;
  const double2* row = reinterpret_cast<const double2*>(table + chunk * 8);
#pragma unroll 4
  for (int s = 0; s < L; ++s) {
    const double v = static_cast<double>(in[s * InStep]);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double2 b = row[s * (L / 2) + q];
      acc[2 * q] += v * b.x;
      acc[2 * q + 1] += v * b.y;
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) out[j * OutStep] = static_cast<Out>(acc[j]);
}

// Runtime chunk index (warp-uniform). Lengths 8 and 16 use the unrolled form
// with compile-time basis offsets; length 32 reads its basis from a shared
// table when the caller staged one (`table`), else from constant memory,
// because the fully unrolled length-32 passes outgrow the instruction cache.
template <int L, bool kForward, int InStep, int OutStep, typename In, typename Out>
__device__ __forceinline__ void LineChunkAt(int chunk, const In* __restrict__ in,
                                            Out* __restrict__ out,
                                            const double* table = nullptr) {
  if constexpr (L == 32) {
    if (table != nullptr) {
      LineChunkShared<L, InStep, OutStep>(chunk, table, in, out);
    } else {
      LineChunkTable<L, kForward, InStep, OutStep>(chunk, in, out);
    }
  } else {
    (void)table;
    switch (chunk) {
      case 0:
        LineChunk<L, kForward, 0, InStep, OutStep>(in, out);
        break;
      case 1:
        if constexpr (L > 8) LineChunk<L, kForward, 1, InStep, OutStep>(in, out);
        break;
      default:
        break;
    }
  }
}

}  // namespace gjxl_b200

namespace gjxl_b200 {

// A batch of KC = transforms x channels W x H planes in shared memory,
// [plane][row][column] with rows padded to W + 1 elements: threads on
// consecutive rows (row passes) and threads on consecutive columns (column
// passes) then hit distinct banks. Items = one 8-output chunk of one line,
// KC * W * H / 8 per pass.
template <int W, int H, int KC>
struct PlaneBatch {
  static constexpr int N = W * H;
  static constexpr int RowPitch = W + 1;
  static constexpr int PlanePitch = H * RowPitch;
  static constexpr int Elements = KC * PlanePitch;
  static constexpr int Items = KC * N / 8;
  static_assert((KC * H) % 32 == 0 && (KC * W) % 32 == 0, "warp-uniform chunks");
  __device__ static int At(int plane, int row, int column) {
    return plane * PlanePitch + row * RowPitch + column;
  }
};

// Row pass over all KC * H rows of `in` into `out` (same layout): item
// `item` is chunk item / (KC * H) of row item % (KC * H). `valid(plane)`
// skips planes of absent transforms.
// `table`: a shared copy of the width-length basis laid out [s][k], or null.
template <int W, int H, int KC, bool kForward, typename In, typename Valid>
__device__ __forceinline__ void BatchRowPass(const In* in, double* out, int tid, int threads,
                                             Valid valid, const double* table = nullptr) {
  using B = PlaneBatch<W, H, KC>;
  constexpr int kLines = KC * H;
  for (int item = tid; item < B::Items; item += threads) {
    const int chunk = item / kLines, line = item % kLines;
    if (!valid(line / H)) continue;
    LineChunkAt<W, kForward, 1, 1>(chunk, in + line * B::RowPitch,
                                   out + line * B::RowPitch + chunk * 8, table);
  }
}

// Column pass over all KC * W columns: item `item` is chunk item / (KC * W)
// of column item % (KC * W). `table`: as for the row pass, height-length.
template <int W, int H, int KC, bool kForward, typename Out, typename Valid>
__device__ __forceinline__ void BatchColumnPass(const double* in, Out* out, int tid, int threads,
                                                Valid valid, const double* table = nullptr) {
  using B = PlaneBatch<W, H, KC>;
  constexpr int kLines = KC * W;
  for (int item = tid; item < B::Items; item += threads) {
    const int chunk = item / kLines, line = item % kLines;
    const int plane = line / W, u = line % W;
    if (!valid(plane)) continue;
    const int base = plane * B::PlanePitch + u;
    LineChunkAt<H, kForward, B::RowPitch, B::RowPitch>(chunk, in + base,
                                                       out + base + chunk * 8 * B::RowPitch,
                                                       table);
  }
}

}  // namespace gjxl_b200

namespace gjxl_b200 {

// FP32 line passes of lengths 8 and 16 for the fast cost mode: the same
// chunking as the FP64 passes, with the bases rounded to float and each
// multiply-add fused (one rounding per term).
template <int L, bool kForward>
__device__ __forceinline__ float DctBasisF(int index) {
  if constexpr (kForward) {
    if constexpr (L == 8) return kDctForward8F[index];
    if constexpr (L == 16) return kDctForward16F[index];
  } else {
    if constexpr (L == 8) return kDctInverse8F[index];
    if constexpr (L == 16) return kDctInverse16F[index];
  }
  return 0.0f;
}

template <int L, bool kForward, int C, int InStep, int OutStep, typename In, typename Out>
__device__ __forceinline__ void LineChunkF(const In* __restrict__ in, Out* __restrict__ out) {
  static_assert(L == 8 || L == 16, "FP32 passes cover lengths 8 and 16");
  float acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = 0.0f;
#pragma unroll
  for (int s = 0; s < L; ++s) {
    const float v = static_cast<float>(in[s * InStep]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = C * 8 + j;
      acc[j] = fmaf(v, DctBasisF<L, kForward>(kForward ? k * L + s : s * L + k), acc[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) out[j * OutStep] = static_cast<Out>(acc[j]);
}

template <int L, bool kForward, int InStep, int OutStep, typename In, typename Out>
__device__ __forceinline__ void LineChunkAtF(int chunk, const In* __restrict__ in,
                                             Out* __restrict__ out) {
  if (chunk == 0) {
    LineChunkF<L, kForward, 0, InStep, OutStep>(in, out);
  } else if constexpr (L > 8) {
    if (chunk == 1) LineChunkF<L, kForward, 1, InStep, OutStep>(in, out);
  }
}

// FP32 counterparts of BatchRowPass / BatchColumnPass (float intermediate).
template <int W, int H, int KC, bool kForward, typename In, typename Valid>
__device__ __forceinline__ void BatchRowPassF(const In* in, float* out, int tid, int threads,
                                              Valid valid) {
  using B = PlaneBatch<W, H, KC>;
  constexpr int kLines = KC * H;
  for (int item = tid; item < B::Items; item += threads) {
    const int chunk = item / kLines, line = item % kLines;
    if (!valid(line / H)) continue;
    LineChunkAtF<W, kForward, 1, 1>(chunk, in + line * B::RowPitch,
                                    out + line * B::RowPitch + chunk * 8);
  }
}

template <int W, int H, int KC, bool kForward, typename Out, typename Valid>
__device__ __forceinline__ void BatchColumnPassF(const float* in, Out* out, int tid, int threads,
                                                 Valid valid) {
  using B = PlaneBatch<W, H, KC>;
  constexpr int kLines = KC * W;
  for (int item = tid; item < B::Items; item += threads) {
    const int chunk = item / kLines, line = item % kLines;
    const int plane = line / W, u = line % W;
    if (!valid(plane)) continue;
    const int base = plane * B::PlanePitch + u;
    LineChunkAtF<H, kForward, B::RowPitch, B::RowPitch>(chunk, in + base,
                                                        out + base + chunk * 8 * B::RowPitch);
  }
}

}  // namespace gjxl_b200
