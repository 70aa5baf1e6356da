/*
 * CPU restatement of the gjxl reference's analysis arithmetic, stage by stage.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle). Compiled by oracle/Makefile into
 * oracle/_build/librestate.so with gcc -O2 -ffp-contract=off, so every
 * multiply and add rounds separately and fmaf() is the only fused operation,
 * matching the reference's x86 build. Each function cites the reference code
 * it restates; the CPU tests pin each one against the compiled reference
 * (oracle/_ref) and the committed golden vectors.
 *
 * Images are planar float32: plane c at base + c * width * height.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define API __attribute__((visibility("default")))

static float bits_to_float(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }
static uint32_t float_to_bits(float f) { uint32_t b; memcpy(&b, &f, 4); return b; }

/* src/c_api/image_conversion.cpp:18-31 — sRGB decode, double then float. */
API void restate_srgb_table(float table[256]) {
  for (int i = 0; i < 256; ++i) {
    double e = (double)i / 255.0;
    double l = e <= 0.04045 ? e / 12.92 : pow((e + 0.055) / 1.055, 2.4);
    table[i] = (float)l;
  }
}

/* src/codec/color_transform.cpp:54-80 — libjxl CubeRootAndAdd. */
static float cube_root_and_add(float v, float add) {
  const float third = 1.0f / 3.0f, four_thirds = 4.0f / 3.0f;
  uint32_t bits = float_to_bits(v);
  float r = bits_to_float(bits == 0 ? 0u : 0x54800000u - (bits >> 23) * 0x002AAAAAu);
  float d = third * v;
  for (int i = 0; i < 3; ++i) {
    float sq = r * r;
    r = fmaf(-d, sq * sq, four_thirds * r);
  }
  float sq = r * r;
  r = fmaf(third, fmaf(-v, sq * sq, r), r);
  sq = r * r;
  return fmaf(sq, v, add);
}

/*
 * src/c_api/image_conversion.cpp:116-138 followed by
 * src/codec/color_transform.cpp:233-330 (scalar path) and :365-393 (padding).
 * pixels: packed RGB8/RGBA8 rows; linear: 3 x h x w; opsin: 3 x ph x pw.
 */
API void restate_prepare_input(const uint8_t* pixels, size_t w, size_t h, size_t stride,
                               int channels, float intensity, float* linear, float* opsin,
                               size_t pw, size_t ph) {
  static const float m[3][3] = {
    {0.30f, 0.622f, 0.078f},
    {0.23f, 0.692f, 0.078f},
    {0.24342268924547819f, 0.20476744424496821f, 0.55180986650955360f}};
  const float bias = 0.0037930732552754493f;
  float table[256];
  restate_srgb_table(table);
  const float scale = intensity / 255.0f;
  const float bias_cbrt = cube_root_and_add(bias, 0.0f);
  for (size_t y = 0; y < h; ++y) {
    const uint8_t* row = pixels + y * stride;
    for (size_t x = 0; x < w; ++x) {
      float rgb[3];
      for (int c = 0; c < 3; ++c) {
        rgb[c] = table[row[x * channels + c]];
        linear[c * w * h + y * w + x] = rgb[c];
      }
      float g[3];
      for (int r = 0; r < 3; ++r) {
        float v = fmaf(scale * m[r][2], rgb[2], bias);
        v = fmaf(scale * m[r][1], rgb[1], v);
        v = fmaf(scale * m[r][0], rgb[0], v);
        g[r] = cube_root_and_add(v > 0.0f ? v : 0.0f, -bias_cbrt);
      }
      opsin[0 * pw * ph + y * pw + x] = 0.5f * (g[0] - g[1]);
      opsin[1 * pw * ph + y * pw + x] = 0.5f * (g[0] + g[1]);
      opsin[2 * pw * ph + y * pw + x] = g[2];
    }
    for (int c = 0; c < 3; ++c) {
      float* o = opsin + c * pw * ph + y * pw;
      for (size_t x = w; x < pw; ++x) o[x] = o[w - 1];
    }
  }
  for (int c = 0; c < 3; ++c) {
    for (size_t y = h; y < ph; ++y) {
      memcpy(opsin + c * pw * ph + y * pw, opsin + c * pw * ph + (h - 1) * pw,
             pw * sizeof(float));
    }
  }
}

/* src/codestream/workflow.cpp:1318-1432 — max x-edge, b-edge, exposed blue
 * over the unpadded region of a padded opsin image (row stride pw). */
API void restate_matrix_scale_stats(const float* opsin, size_t pw, size_t ph, size_t w,
                                    size_t h, float stats[3]) {
  const float* X = opsin;
  const float* Y = opsin + pw * ph;
  const float* B = opsin + 2 * pw * ph;
  float xe = 0.0f, be = 0.0f, eb = 0.0f;
  for (size_t y = 1; y < h; ++y) {
    for (size_t x = 1; x < w; ++x) {
      size_t i = y * pw + x, l = i - 1, u = i - pw;
      float a = fabsf(X[i] - X[l]), b = fabsf(X[i] - X[u]);
      float m = a > b ? a : b;
      if (m > xe) xe = m;
      float d = B[i] - Y[i];
      a = fabsf(d - (B[l] - Y[l]));
      b = fabsf(d - (B[u] - Y[u]));
      m = a > b ? a : b;
      if (m > be) be = m;
      float e = B[i] - 1.2f * Y[i];
      if (e >= 0.0f) {
        e *= fabsf(B[i] - B[l]) + fabsf(B[i] - B[u]);
        if (e > eb) eb = e;
      }
    }
  }
  stats[0] = xe;
  stats[1] = be;
  stats[2] = eb;
}

/* src/codestream/workflow.cpp:1435-1483 — x/b quantization-matrix scales. */
API void restate_select_matrix_scales(const float stats[3], float target, int scales[2]) {
  int x = 3, b = 2;
  const float thresholds[3] = {2.5f, 5.5f, 9.5f};
  for (int i = 0; i < 3; ++i) if (target > thresholds[i]) ++x;
  int xa = stats[0] >= 0.026f ? 3 : stats[0] >= 0.022f ? 2 : stats[0] >= 0.015f ? 1 : 0;
  if (x < 2 + xa) x = 2 + xa;
  int eb = stats[2] >= 0.13f ? 1 : 0;
  int ba = stats[1] > 0.38f ? 2 + eb : stats[1] > 0.33f ? 1 + eb : stats[1] > 0.28f ? eb : 0;
  scales[0] = x;
  scales[1] = b + ba;
}
