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

// ---- D3Q39 domain faces (kernel_entropic_d3q39.jl:898-1330 at the default boundary options) ----
// The velocity set in the reference's order (lattice.jl:177-262), 0-based, and its mirrors.
KBC_HD int q39cx(int k) {
  constexpr int t[39] = {0, -1, 1, 0, 0, 0, 0, -1, -1, -1, -1, 1, 1, 1, 1, -2, 2, 0, 0, 0,
                         0, -2, -2, 2, 2, -2, -2, 2, 2, 0, 0, 0, 0, -3, 3, 0, 0, 0, 0};
  return t[k];
}
KBC_HD int q39cy(int k) {
  constexpr int t[39] = {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, -1, -1, 1, 1, 0, 0, -2, 2, 0,
                         0, -2, 2, -2, 2, 0, 0, 0, 0, -2, -2, 2, 2, 0, 0, -3, 3, 0, 0};
  return t[k];
}
KBC_HD int q39cz(int k) {
  constexpr int t[39] = {0, 0, 0, 0, 0, -1, 1, -1, 1, -1, 1, -1, 1, -1, 1, 0, 0, 0, 0, -2,
                         2, 0, 0, 0, 0, -2, 2, -2, 2, -2, 2, -2, 2, 0, 0, 0, 0, -3, 3};
  return t[k];
}
KBC_HD int q39opp(int k) {
  constexpr int t[39] = {0, 2, 1, 4, 3, 6, 5, 14, 13, 12, 11, 10, 9, 8, 7, 16, 15, 18, 17, 20,
                         19, 24, 23, 22, 21, 28, 27, 26, 25, 32, 31, 30, 29, 34, 33, 36, 35, 38, 37};
  return t[k];
}
KBC_HD int q39my(int k) {  // (cx, -cy, cz)
  constexpr int t[39] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 13, 14, 11, 12, 15, 16, 18, 17, 19,
                         20, 22, 21, 24, 23, 25, 26, 27, 28, 31, 32, 29, 30, 33, 34, 36, 35, 37, 38};
  return t[k];
}
KBC_HD int q39mz(int k) {  // (cx, cy, -cz)
  constexpr int t[39] = {0, 1, 2, 3, 4, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 15, 16, 17, 18, 20,
                         19, 21, 22, 23, 24, 26, 25, 28, 27, 30, 29, 32, 31, 33, 34, 35, 36, 38, 37};
  return t[k];
}
KBC_HD float q39w(int k) {
  return k < 7 ? float(1.0 / 12) : k < 15 ? float(1.0 / 27) : k < 21 ? float(2.0 / 135) : k < 33 ? float(1.0 / 432)
                                                                                             : float(1.0 / 1620);
}

// gradient_noise (physics_utils.jl:5-17): 32-bit hash of the integer position and seed
KBC_HD float gradient_noise(int32_t gx, int32_t gy, int32_t gz, int32_t seed) {
  uint32_t h = (uint32_t)gx * 374761393u + (uint32_t)gy * 668265263u + (uint32_t)gz * 1274126177u + (uint32_t)seed;
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  h = h ^ (h >> 16);
  return ((float)(h & 0xFFFFu) / 32768.0f) - 1.0f;
}

KBC_HD float fmaxnan(float a, float b) { return (a != a || b != b) ? a + b : (a < b ? b : a); }

// The face value of direction k pulled by the cell at global (gx, gy, gz) (1-based) from the
// source position g - c_k outside a domain of nx x ny x nz cells: own = the cell's own populations
// (39, stride apart); feq_in = the host inlet equilibrium. Outlet mode zero-gradient, freestream
// inlet density, no non-reflecting inlet blend (the reference's defaults).
struct FaceParams {
  int32_t nx, ny, nz, ymin_wall, transverse_fs, seed;
  float transverse_blend, inlet_turbulence, u_inlet;
};
KBC_HD float face_value(const FaceParams& F, const float* own, int stride, const float* feq_in, int k, int gx, int gy,
                        int gz) {
  const int cx = q39cx(k), cy = q39cy(k), cz = q39cz(k);
  const int sgx = gx - cx, sgy = gy - cy, sgz = gz - cz;
  const bool is_inlet = sgx < 1, is_outlet = sgx > F.nx;
  const bool at_y = sgy < 1 || sgy > F.ny, at_z = sgz < 1 || sgz > F.nz;
  if (F.transverse_fs == 1 && (at_y || at_z)) {
    const float beta = F.transverse_blend;
    return (1.0f - beta) * own[k * stride] + beta * feq_in[k];
  }
  if ((is_inlet || is_outlet) && at_y && at_z) return own[q39my(q39mz(k)) * stride];
  if ((is_inlet || is_outlet) && at_y) return own[q39my(k) * stride];
  if ((is_inlet || is_outlet) && at_z) return own[q39mz(k) * stride];
  if (is_inlet) {
    const float rho_bc = 1.0f;
    float target = rho_bc * feq_in[k];
    if (F.inlet_turbulence > 0.0f) {
      const float amp = F.inlet_turbulence * fmaxnan(F.u_inlet < 0.0f ? -F.u_inlet : F.u_inlet, 1e-6f);
      const float dux = 0.25f * amp * gradient_noise(gx, gy, gz, F.seed + 1234);
      const float duy = 0.50f * amp * gradient_noise(gx, gy, gz, F.seed + 5678);
      const float duz = amp * gradient_noise(gx, gy, gz, F.seed + 9012);
      const float cxr = float(cx) - 0.0f, cyr = float(cy) - 0.0f, czr = float(cz) - 0.0f;
      target += q39w(k) * rho_bc * (cxr * dux + cyr * duy + czr * duz) / fmaxnan(float(2.0 / 3.0), 1e-6f);
      target = fmaxnan(target, 1e-12f);
    }
    return target;
  }
  if (is_outlet) return own[k * stride];
  if (sgy < 1 && F.ymin_wall == 1) return own[q39opp(k) * stride];
  if (at_y) return own[q39my(k) * stride];
  if (at_z) return own[q39mz(k) * stride];
  return q39w(k);
}

// solve_shell_moment4 (amr_coupling.jl:130-176): 4x4 elimination without pivoting
KBC_HD bool shell_solve4(float m00, float m01, float m02, float m03, float m11, float m12, float m13, float m22,
                         float m23, float m33, float r0, float r1, float r2, float r3, float& x0, float& x1, float& x2,
                         float& x3) {
  const float eps = 1e-12f;
  float a00 = m00 + eps, a01 = m01, a02 = m02, a03 = m03, b0 = r0;
  float a10 = m01, a11 = m11 + eps, a12 = m12, a13 = m13, b1 = r1;
  float a20 = m02, a21 = m12, a22 = m22 + eps, a23 = m23, b2 = r2;
  float a30 = m03, a31 = m13, a32 = m23, a33 = m33 + eps, b3 = r3;
  const bool ok0 = (a00 < 0.0f ? -a00 : a00) > eps;
  const float inv0 = ok0 ? 1.0f / a00 : 0.0f;
  const float f10 = a10 * inv0, f20 = a20 * inv0, f30 = a30 * inv0;
  a11 -= f10 * a01; a12 -= f10 * a02; a13 -= f10 * a03; b1 -= f10 * b0;
  a21 -= f20 * a01; a22 -= f20 * a02; a23 -= f20 * a03; b2 -= f20 * b0;
  a31 -= f30 * a01; a32 -= f30 * a02; a33 -= f30 * a03; b3 -= f30 * b0;
  const bool ok1 = (a11 < 0.0f ? -a11 : a11) > eps;
  const float inv1 = ok1 ? 1.0f / a11 : 0.0f;
  const float f21 = a21 * inv1, f31 = a31 * inv1;
  a22 -= f21 * a12; a23 -= f21 * a13; b2 -= f21 * b1;
  a32 -= f31 * a12; a33 -= f31 * a13; b3 -= f31 * b1;
  const bool ok2 = (a22 < 0.0f ? -a22 : a22) > eps;
  const float inv2 = ok2 ? 1.0f / a22 : 0.0f;
  const float f32 = a32 * inv2;
  a33 -= f32 * a23; b3 -= f32 * b2;
  const bool ok3 = (a33 < 0.0f ? -a33 : a33) > eps;
  const float inv3 = ok3 ? 1.0f / a33 : 0.0f;
  x3 = b3 * inv3;
  x2 = (b2 - a23 * x3) * inv2;
  x1 = (b1 - a12 * x2 - a13 * x3) * inv1;
  x0 = (b0 - a01 * x1 - a02 * x2 - a03 * x3) * inv0;
  return ok0 && ok1 && ok2 && ok3;
}

// apply_4momentum_correction_d3q39! at zero frame shift (physics_utils.jl:830-900): move the
// populations f (39, stride apart) onto the target density and momentum by w_k (a0 + a1 cx +
// a2 cy + a3 cz), a from the weights' Gram system. The inlet-face pin of
// kernel_entropic_d3q39.jl:1313-1352 calls it with the inlet equilibrium's moments.
KBC_HD void four_moment_pin(float* f, int stride, float trho, float tjx, float tjy, float tjz) {
  float rho = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
  for (int k = 0; k < 39; ++k) {
    const float v = f[k * stride];
    const float cx = float(q39cx(k)) - 0.0f, cy = float(q39cy(k)) - 0.0f, cz = float(q39cz(k)) - 0.0f;
    rho += v; jx += v * cx; jy += v * cy; jz += v * cz;
  }
  const float er = trho - rho, ex = tjx - jx, ey = tjy - jy, ez = tjz - jz;
  if ((er < 0.0f ? -er : er) < 1e-9f && (ex < 0.0f ? -ex : ex) < 1e-9f && (ey < 0.0f ? -ey : ey) < 1e-9f &&
      (ez < 0.0f ? -ez : ez) < 1e-9f)
    return;
  float m00 = 0.0f, m01 = 0.0f, m02 = 0.0f, m03 = 0.0f, m11 = 0.0f, m12 = 0.0f, m13 = 0.0f, m22 = 0.0f, m23 = 0.0f,
        m33 = 0.0f;
  for (int k = 0; k < 39; ++k) {
    const float w = q39w(k), cx = float(q39cx(k)) - 0.0f, cy = float(q39cy(k)) - 0.0f, cz = float(q39cz(k)) - 0.0f;
    m00 += w; m01 += w * cx; m02 += w * cy; m03 += w * cz;
    m11 += w * cx * cx; m12 += w * cx * cy; m13 += w * cx * cz;
    m22 += w * cy * cy; m23 += w * cy * cz; m33 += w * cz * cz;
  }
  float a0, a1, a2, a3;
  if (!shell_solve4(m00, m01, m02, m03, m11, m12, m13, m22, m23, m33, er, ex, ey, ez, a0, a1, a2, a3)) return;
  for (int k = 0; k < 39; ++k) {
    const float w = q39w(k), cx = float(q39cx(k)) - 0.0f, cy = float(q39cy(k)) - 0.0f, cz = float(q39cz(k)) - 0.0f;
    f[k * stride] += w * (a0 + a1 * cx + a2 * cy + a3 * cz);
  }
}

}  // namespace kbc
