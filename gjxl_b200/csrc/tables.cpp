// Construction of the JPEG XL default AC quantization weights and the DCT
// bases used by the reference encoder.
//
// Quantization weights: the JPEG XL default "DCT" parameterisation (ISO/IEC
// 18181-1 default matrices, as pinned by the reference from libjxl
// e8ff0976, see the reference's scripts/generate_quantization_tables.py and
// src/codec/quantization_tables_generated.h). Each channel has a list of
// band weights; the weight at frequency (x, y) interpolates geometrically
// between the two bands bracketing its scaled radial distance, using libjxl's
// FastPow. All arithmetic is single precision with the same rounding steps.
//
// DCT bases: src/codec/dct.cpp:16-37, in double precision.

#include "tables.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "host_util.h"

namespace gjxl_b200 {
namespace {

float F32(double v) { return static_cast<float>(v); }

float HostFastLog2(float value) {
  uint32_t bits;
  std::memcpy(&bits, &value, 4);
  const int32_t e = static_cast<int32_t>(bits - 0x3f2aaaabu) >> 23;
  const uint32_t m = bits - (static_cast<uint32_t>(e) << 23);
  float mantissa;
  std::memcpy(&mantissa, &m, 4);
  const float x = mantissa - 1.0f;
  float num = std::fma(0.74245873327820566f, x, 1.4287160470083755f);
  num = std::fma(num, x, -1.8503833400518310e-06f);
  float den = std::fma(0.17409343003366853f, x, 1.0096718572241148f);
  den = std::fma(den, x, 0.99032814277590719f);
  return num / den + static_cast<float>(e);
}

float HostFastPow2(float value) {
  const float fl = std::floor(value);
  const uint32_t eb = static_cast<uint32_t>(static_cast<int32_t>(fl) + 127) << 23;
  float ev;
  std::memcpy(&ev, &eb, 4);
  const float f = value - fl;
  float num = f + 1.01749063e+01f;
  num = std::fma(num, f, 4.88687798e+01f);
  num = std::fma(num, f, 9.85506591e+01f);
  num *= ev;
  float den = std::fma(f, 2.10242958e-01f, -2.22328856e-02f);
  den = std::fma(den, f, -1.94414990e+01f);
  den = std::fma(den, f, 9.85506633e+01f);
  return num / den;
}

float BandMultiplier(float v) { return v > 0.0f ? 1.0f + v : 1.0f / (1.0f - v); }

struct FamilyParams {
  int rows, columns, lf_rows, lf_columns;
  int band_count;
  double bands[3][8];
};

// JPEG XL default DCT quantization parameters (first value: weight of the
// lowest band; following values: log-ish band ratios).
const FamilyParams kFamilies[kTableCount] = {
  {8, 8, 1, 1, 6,
   {{3150.0, 0.0, -0.4, -0.4, -0.4, -2.0},
    {560.0, 0.0, -0.3, -0.3, -0.3, -0.3},
    {512.0, -2.0, -1.0, 0.0, -1.0, -2.0}}},
  {16, 16, 2, 2, 7,
   {{8996.8725711814115328, -1.3000777393353804, -0.49424529824571225, -0.439093774457103443,
     -0.6350101832695744, -0.90177264050827612, -1.6162099239887414},
    {3191.48366296844234752, -0.67424582104194355, -0.80745813428471001,
     -0.44925837484843441, -0.35865440981033403, -0.31322389111877305,
     -0.37615025315725483},
    {1157.50408145487200256, -2.0531423165804414, -1.4, -0.50687130033378396,
     -0.42708730624733904, -1.4856834539296244, -4.9209142884401604}}},
  {32, 32, 4, 4, 8,
   {{15718.40830982518931456, -1.025, -0.98, -0.9012, -0.4, -0.48819395464, -0.421064, -0.27},
    {7305.7636810695983104, -0.8041958212306401, -0.7633036457487539, -0.55660379990111464,
     -0.49785304658857626, -0.43699592683512467, -0.40180866526242109,
     -0.27321683125358037},
    {3803.53173721215041536, -3.060733579805728, -2.0413270132490346, -2.0235650159727417,
     -0.5495389509954993, -0.4, -0.4, -0.3}}},
  {8, 16, 1, 2, 7,
   {{7240.7734393502, -0.7, -0.7, -0.2, -0.2, -0.2, -0.5},
    {1448.15468787004, -0.5, -0.5, -0.5, -0.2, -0.2, -0.2},
    {506.854140754517, -1.4, -0.2, -0.5, -0.5, -1.5, -3.6}}},
  {16, 32, 2, 4, 8,
   {{13844.97076442300573, -0.97113799999999995, -0.658, -0.42026, -0.22712, -0.2206, -0.226,
     -0.6},
    {4798.964084220744293, -0.61125308982767057, -0.83770786552491361, -0.79014862079498627,
     -0.2692727459704829, -0.38272769465388551, -0.22924222653091453,
     -0.20719098826199578},
    {1807.236946760964614, -1.2, -1.2, -0.7, -0.7, -0.7, -0.4, -0.5}}},
};

void ChannelWeights(const FamilyParams& f, int channel, float* out) {
  float bands[8];
  bands[0] = F32(f.bands[channel][0]);
  for (int i = 1; i < f.band_count; ++i) {
    bands[i] = bands[i - 1] * BandMultiplier(F32(f.bands[channel][i]));
  }
  const float sqrt_two = F32(1.41421356237);
  const float distance_scale =
    static_cast<float>(f.band_count - 1) / (sqrt_two + F32(1.0e-6));
  const float row_scale = distance_scale / static_cast<float>(f.rows - 1);
  const float column_scale = distance_scale / static_cast<float>(f.columns - 1);
  for (int y = 0; y < f.rows; ++y) {
    const float dy = static_cast<float>(y) * row_scale;
    const float dy2 = dy * dy;
    for (int x = 0; x < f.columns; ++x) {
      const float dx = static_cast<float>(x) * column_scale;
      const float position = std::sqrt(std::fma(dx, dx, dy2));
      int index = static_cast<int>(position);
      if (index > f.band_count - 2) index = f.band_count - 2;
      const float fraction = position - static_cast<float>(index);
      const float a = bands[index];
      const float b = bands[index + 1];
      const float ratio = b / a;
      const float power = HostFastPow2(HostFastLog2(ratio) * fraction);
      out[y * f.columns + x] = a * power;
    }
  }
}

void MakeBasis(int n, bool forward, double* out) {
  const double sqrt_two = 1.41421356237309504880;  // std::numbers::sqrt2_v<double>
  const double pi = 3.14159265358979323846;        // std::numbers::pi_v<double>
  const double scale = forward ? sqrt_two / static_cast<double>(n) : sqrt_two;
  for (int frequency = 0; frequency < n; ++frequency) {
    const double alpha = frequency == 0 ? 1.0 / sqrt_two : 1.0;
    for (int sample = 0; sample < n; ++sample) {
      const double angle = (static_cast<double>(sample) + 0.5) *
                           static_cast<double>(frequency) * pi / static_cast<double>(n);
      out[frequency * n + sample] = scale * alpha * std::cos(angle);
    }
  }
}

struct Storage {
  HostTables tables;
  std::vector<float> dequant, inverse_dequant;
  std::vector<double> forward[3], inverse[3];
};

Storage* BuildStorage() {
  auto* s = new Storage();
  size_t total = 0;
  for (int t = 0; t < kTableCount; ++t) {
    s->tables.layout.offset[t] = total;
    s->tables.layout.count[t] = static_cast<size_t>(kFamilies[t].rows) * kFamilies[t].columns;
    total += 3 * s->tables.layout.count[t];
  }
  s->tables.layout.total = total;
  s->dequant.resize(total);
  s->inverse_dequant.resize(total);
  for (int t = 0; t < kTableCount; ++t) {
    const FamilyParams& f = kFamilies[t];
    const size_t n = s->tables.layout.count[t];
    std::vector<float> weights(n);
    for (int c = 0; c < 3; ++c) {
      ChannelWeights(f, c, weights.data());
      float* dq = s->dequant.data() + s->tables.layout.offset[t] + c * n;
      float* inv = s->inverse_dequant.data() + s->tables.layout.offset[t] + c * n;
      for (int y = 0; y < f.rows; ++y) {
        for (int x = 0; x < f.columns; ++x) {
          const size_t i = static_cast<size_t>(y) * f.columns + x;
          dq[i] = 1.0f / weights[i];
          inv[i] = (y < f.lf_rows && x < f.lf_columns) ? 0.0f : weights[i];
        }
      }
    }
  }
  for (int i = 0; i < 3; ++i) {
    const int n = 8 << i;
    s->forward[i].resize(n * n);
    s->inverse[i].resize(n * n);
    MakeBasis(n, true, s->forward[i].data());
    MakeBasis(n, false, s->inverse[i].data());
    s->tables.forward[i] = s->forward[i].data();
    s->tables.inverse[i] = s->inverse[i].data();
  }
  s->tables.dequant = s->dequant.data();
  s->tables.inverse_dequant = s->inverse_dequant.data();
  return s;
}

std::mutex g_device_mutex;
constexpr int kMaxDevices = 64;
void* g_device_block[kMaxDevices] = {};
DeviceTables g_device_tables[kMaxDevices];

}  // namespace

const HostTables& GetHostTables() {
  static Storage* storage = BuildStorage();
  return storage->tables;
}

int StrategyTableFamily(int strategy) {
  switch (strategy) {
    case 0: return kTableDct8;       // DCT8
    case 4: return kTableDct16;      // DCT16x16
    case 5: return kTableDct32;      // DCT32x32
    case 6: case 7: return kTableDct8x16;    // DCT16x8, DCT8x16
    case 10: case 11: return kTableDct16x32; // DCT32x16, DCT16x32
    default: return -1;
  }
}

int GetDeviceTables(DeviceTables* out) {
  int device = 0;
  int status = CheckCuda(cudaGetDevice(&device), "tables: cudaGetDevice");
  if (status != 0) return status;
  if (device < 0 || device >= kMaxDevices) {
    return SetError(GJXL_B200_UNSUPPORTED, "tables: device ordinal out of range");
  }
  std::lock_guard<std::mutex> lock(g_device_mutex);
  if (g_device_block[device] == nullptr) {
    const HostTables& h = GetHostTables();
    const size_t floats = h.layout.total;
    size_t doubles = 0;
    for (int i = 0; i < 3; ++i) doubles += 3 * static_cast<size_t>(64) << (2 * i);
    const size_t bytes = 2 * floats * sizeof(float) + doubles * sizeof(double) + 256;
    std::vector<unsigned char> host(bytes, 0);
    size_t offset = 0;
    auto place = [&](const void* src, size_t n) {
      offset = (offset + 15) & ~size_t{15};
      std::memcpy(host.data() + offset, src, n);
      const size_t at = offset;
      offset += n;
      return at;
    };
    size_t off_dq = place(h.dequant, floats * sizeof(float));
    size_t off_inv = place(h.inverse_dequant, floats * sizeof(float));
    size_t off_ft[3], off_f[3], off_i[3];
    for (int i = 0; i < 3; ++i) {
      const int n = 8 << i;
      std::vector<double> t(n * n);
      for (int f = 0; f < n; ++f)
        for (int s = 0; s < n; ++s) t[s * n + f] = h.forward[i][f * n + s];
      off_ft[i] = place(t.data(), t.size() * sizeof(double));
      off_f[i] = place(h.forward[i], n * n * sizeof(double));
      off_i[i] = place(h.inverse[i], n * n * sizeof(double));
    }
    void* block = nullptr;
    status = CheckCuda(cudaMalloc(&block, bytes), "tables: cudaMalloc");
    if (status != 0) return status;
    status = CheckCuda(cudaMemcpy(block, host.data(), bytes, cudaMemcpyHostToDevice),
                       "tables: upload");
    if (status != 0) {
      cudaFree(block);
      return status;
    }
    auto* base = static_cast<unsigned char*>(block);
    DeviceTables d;
    d.dequant = reinterpret_cast<const float*>(base + off_dq);
    d.inverse_dequant = reinterpret_cast<const float*>(base + off_inv);
    for (int i = 0; i < 3; ++i) {
      d.forward_t[i] = reinterpret_cast<const double*>(base + off_ft[i]);
      d.forward[i] = reinterpret_cast<const double*>(base + off_f[i]);
      d.inverse[i] = reinterpret_cast<const double*>(base + off_i[i]);
    }
    g_device_tables[device] = d;
    g_device_block[device] = block;
  }
  *out = g_device_tables[device];
  return GJXL_B200_OK;
}

}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" int gjxl_b200_quant_matrix(int strategy, int channel, float* dequant,
                                      float* inverse_dequant, size_t capacity) {
  ClearLastError();
  const int family = StrategyTableFamily(strategy);
  if (family < 0 || channel < 0 || channel > 2) {
    return SetError(GJXL_B200_UNAVAILABLE, "quant_matrix: no default matrix for strategy");
  }
  const HostTables& h = GetHostTables();
  const size_t n = h.layout.count[family];
  if (capacity < n || dequant == nullptr || inverse_dequant == nullptr) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "quant_matrix: output too small");
  }
  std::memcpy(dequant, h.dequant + h.layout.offset[family] + channel * n, n * sizeof(float));
  std::memcpy(inverse_dequant, h.inverse_dequant + h.layout.offset[family] + channel * n,
              n * sizeof(float));
  return GJXL_B200_OK;
}
