// kbc_math.h — single-precision exp and log of the D3Q39 entropic step, shared by the CUDA kernel
// and the CPU restatement so both round identically.
//
// Method (W. J. Cody and W. Waite, "Software Manual for the Elementary Functions", 1980):
//   exp: n = round(x / ln 2) (x clamped to [-87, 88]), r = (x - n*L1) - n*L2 with
//        ln 2 = L1 + L2 split so n*L1 is exact, exp(r) by its Taylor series to r^7
//        (|r| <= ln2/2, truncation < 2^-26), times 2^n.
//   log: x = m * 2^e with m in [sqrt(1/2), sqrt(2)), f = m - 1, s = f/(m + 1),
//        log m = 2 atanh s = 2s + s R(s^2) with R = 2s^2/3 + 2s^4/5 + ... + 2s^10/11
//        (|s| <= 0.1716), written f - s (f - R) since 2s = f - s f,
//        log x = (e*L2 + log m) + e*L1.
// Every operation is a single IEEE binary32 add, multiply or divide (no contraction), so the
// result is the same bit pattern on the host and on the device. Accuracy: within 2 ulp of the
// correctly rounded value over the ranges the step uses (exp on [-20, 20], log on [1e-14, 1e6]).
#pragma once
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define KBC_HD __host__ __device__ __forceinline__
#else
#define KBC_HD inline
#endif

namespace kbc {

KBC_HD float bits_to_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  std::memcpy(&f, &u, 4);
  return f;
#endif
}
KBC_HD uint32_t float_to_bits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
#endif
}

// ln 2 = L1 + L2: L1 = 22713/32768 has 15 significant bits, so n*L1 is exact for |n| < 512
constexpr float LN2_1 = 0.693145751953125f;
constexpr float LN2_2 = 1.42860682030941723e-6f;
constexpr float INV_LN2 = 1.44269504088896341f;

// adding 1.5 * 2^23 to |v| < 2^22 rounds v to an integer (ties to even) in the low mantissa bits
constexpr float SHIFT = 12582912.0f;

KBC_HD float exp(float x) {
  if (!(x == x)) return x;
  x = x > 88.0f ? 88.0f : x;
  x = x < -87.0f ? -87.0f : x;
  const float t = x * INV_LN2 + SHIFT;
  const float n = t - SHIFT;                                            // exact
  const int32_t e = (int32_t)(float_to_bits(t) - float_to_bits(SHIFT));  // n, in [-126, 127]
  const float r = (x - n * LN2_1) - n * LN2_2;
  // Taylor coefficients 1/k!
  float p = 1.0f / 5040.0f;
  p = p * r + 1.0f / 720.0f;
  p = p * r + 1.0f / 120.0f;
  p = p * r + 1.0f / 24.0f;
  p = p * r + 1.0f / 6.0f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  return p * bits_to_float((uint32_t)(e + 127) << 23);
}

KBC_HD float log(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -__builtin_huge_valf() : __builtin_nanf("");
  if (x == __builtin_huge_valf()) return x;
  int32_t e = 0;
  if (x < 1.17549435e-38f) { x = x * 16777216.0f; e = -24; }  // subnormal: scale by 2^24
  const uint32_t u = float_to_bits(x);
  e += (int32_t)(u >> 23) - 127;
  float m = bits_to_float((u & 0x007fffffu) | 0x3f800000u);  // [1, 2)
  if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
  const float f = m - 1.0f;  // exact
  const float s = f / (m + 1.0f);
  const float z = s * s;
  // 2 atanh s = 2s + s*R(z) with R = z (2/3 + z (2/5 + ... + z 2/11)), and 2s = f - s*f
  float q = 2.0f / 11.0f;
  q = q * z + 2.0f / 9.0f;
  q = q * z + 2.0f / 7.0f;
  q = q * z + 2.0f / 5.0f;
  q = q * z + 2.0f / 3.0f;
  const float R = q * z;
  const float logm = f - s * (f - R);
  const float ef = (float)e;
  return (ef * LN2_2 + logm) + ef * LN2_1;
}

}  // namespace kbc
