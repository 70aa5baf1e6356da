// Constant tables shared by the transform kernels: JPEG XL default AC
// quantization weights for the seven searched transform families and the
// double-precision DCT-II/DCT-III bases of lengths 8, 16 and 32.
#pragma once

#include <cstddef>
#include <cstdint>

namespace gjxl_b200 {

// Table families, indexed like the reference's quantization tables
// (src/codec/quantization.cpp:658-696).
enum QuantTableFamily : int {
  kTableDct8 = 0,      // 8 x 8,   LLF 1 x 1
  kTableDct16 = 1,     // 16 x 16, LLF 2 x 2
  kTableDct32 = 2,     // 32 x 32, LLF 4 x 4
  kTableDct8x16 = 3,   // 8 rows x 16 columns, LLF 1 x 2 (DCT16x8, DCT8x16)
  kTableDct16x32 = 4,  // 16 rows x 32 columns, LLF 2 x 4 (DCT32x16, DCT16x32)
  kTableCount = 5,
};

// Offsets (in floats) of each family's [channel][coefficient] block inside
// the packed dequant / inverse-dequant arrays.
struct QuantTableLayout {
  size_t offset[kTableCount];
  size_t count[kTableCount];  // coefficients per channel
  size_t total;               // floats per array
};

struct HostTables {
  QuantTableLayout layout;
  const float* dequant;          // [total]
  const float* inverse_dequant;  // [total] (zero over the LLF region)
  // DCT bases, basis[frequency * N + sample] (reference src/codec/dct.cpp:16-37).
  const double* forward[3];  // N = 8, 16, 32
  const double* inverse[3];
};

// Built once on first use (thread-safe), immutable afterwards.
const HostTables& GetHostTables();

// Device copy for the current device: {dequant, inverse_dequant, forward
// bases transposed [sample * N + frequency], forward bases natural, inverse
// bases natural}. Allocated once per device and kept until process exit.
struct DeviceTables {
  const float* dequant;
  const float* inverse_dequant;
  const double* forward_t[3];
  const double* forward[3];
  const double* inverse[3];
};
int GetDeviceTables(DeviceTables* out);

// Maps an AC strategy id (reference src/core/ac_strategy.h:25-53) to its
// table family; -1 when the reference has no table for it.
int StrategyTableFamily(int strategy);

}  // namespace gjxl_b200
