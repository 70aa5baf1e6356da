// log1pf matching the host C library the reference links against.
//
// The reference's initial quant field calls std::log1p(float) (glibc 2.39's
// log1pf, which is Sun's fdlibm s_log1pf algorithm: argument reduction to
// [sqrt(2)/2, sqrt(2)], then a degree-14 odd polynomial in s = f/(2+f)).
// That function is not correctly rounded, so CUDA's log1pf (and a
// double-precision log1p rounded to float) differ from it on about 0.4% of
// inputs. This restatement of the published fdlibm algorithm agrees with
// glibc bit for bit on every non-negative float (checked exhaustively), which
// is the input range the kernels use.
#pragma once

#include <stdint.h>

namespace gjxl_b200 {

__device__ __forceinline__ float Log1pF(float x) {
  const float ln2_hi = 6.9313812256e-01f, ln2_lo = 9.0580006145e-06f;
  const float Lp1 = 6.6666668653e-01f, Lp2 = 4.0000000596e-01f, Lp3 = 2.8571429849e-01f;
  const float Lp4 = 2.2222198546e-01f, Lp5 = 1.8183572590e-01f, Lp6 = 1.5313838422e-01f;
  const float Lp7 = 1.4798198640e-01f;
  float f = 0.0f, c = 0.0f, u;
  const int32_t hx = static_cast<int32_t>(__float_as_uint(x));
  const int32_t ax = hx & 0x7fffffff;
  int32_t k = 1, hu = 0;
  if (hx < 0x3ed413d7) {
    if (ax >= 0x3f800000) return __int_as_float(0x7fc00000);
    if (ax < 0x31000000) {
      if (ax < 0x24800000) return x;
      return x - x * x * 0.5f;
    }
    if (hx > 0 || hx <= static_cast<int32_t>(0xbe95f61f)) {
      k = 0;
      f = x;
      hu = 1;
    }
  }
  if (hx >= 0x7f800000) return x + x;
  if (k != 0) {
    if (hx < 0x5a000000) {
      u = 1.0f + x;
      hu = static_cast<int32_t>(__float_as_uint(u));
      k = (hu >> 23) - 127;
      c = (k > 0) ? 1.0f - (u - x) : x - (u - 1.0f);
      c /= u;
    } else {
      u = x;
      hu = static_cast<int32_t>(__float_as_uint(u));
      k = (hu >> 23) - 127;
      c = 0.0f;
    }
    hu &= 0x007fffff;
    if (hu < 0x3504f7) {
      u = __uint_as_float(static_cast<uint32_t>(hu) | 0x3f800000u);
    } else {
      k += 1;
      u = __uint_as_float(static_cast<uint32_t>(hu) | 0x3f000000u);
      hu = (0x00800000 - hu) >> 2;
    }
    f = u - 1.0f;
  }
  const float hfsq = 0.5f * f * f;
  const float kf = static_cast<float>(k);
  if (hu == 0) {
    if (f == 0.0f) {
      if (k == 0) return 0.0f;
      c += kf * ln2_lo;
      return kf * ln2_hi + c;
    }
    const float R = hfsq * (1.0f - 0.66666666666666666f * f);
    if (k == 0) return f - R;
    return kf * ln2_hi - ((R - (kf * ln2_lo + c)) - f);
  }
  const float s = f / (2.0f + f);
  const float z = s * s;
  const float R = z * (Lp1 + z * (Lp2 + z * (Lp3 + z * (Lp4 + z * (Lp5 + z * (Lp6 + z * Lp7))))));
  if (k == 0) return f - (hfsq - s * (hfsq + R));
  return kf * ln2_hi - ((hfsq - (s * (hfsq + R) + (kf * ln2_lo + c))) - f);
}

}  // namespace gjxl_b200
