// pairs_math.cuh — the D3Q27 cumulant collision of the x-pair kernel in scaled-moment form.
//
// Same physics as cumulant_math.cuh (src/collision/kernel_cumulant.jl:597-844): forward chimera
// transform to central moments, cumulants, relaxation with the adaptive omega_4 and the factored
// limiter, reconstruction, backward transform. The arithmetic is rearranged to cut FP32
// operations per cell on a kernel whose FMA pipe, not DRAM, set its time:
//
//  * Raw moments first, velocity shift afterwards. The x, y and z sums of the pulled values
//    (s = a + c, m0 = b + s, m1 = c - a, m2 = s: three operations per line) give every raw moment
//    M_abc; density and momentum are M_000 and M_100, M_010, M_001, so no separate sums are
//    needed; the three binomial shifts then turn raw into central moments. The sums and the
//    shifts act on different axes, so the order is the chimera transform's up to rounding.
//  * 16-bit deviation storage (f = w (1 + d)): the D3Q27 weights factor as
//    w = 8/27 * phi(cx) phi(cy) phi(cz), phi(0) = 1, phi(+-1) = 1/4, so the sums run on d with
//    m0 = b + s/4 and m1, m2 kept four times too large (their quarter is folded into the later
//    constants); the lattice weights' own moments are constants added once. Moment (a, b, c)
//    then carries 27/8 * 4^n, n = number of nonzero indices, which the reciprocal of the
//    density absorbs (i4, i16, i64 below). FP32 storage sums f itself (no factors).
//  * Backward transform on the normalised post-collision moments (the reference multiplies
//    every one by the density first) with unhalved end populations (m2 -+ m1 instead of
//    (m2 -+ m1) / 2): population k comes out as f_k 2^n / rho, n = |cx| + |cy| + |cz|, and the
//    store's one multiply-add per direction applies rho 2^-n (FP32) or rho 27/8 2^n together
//    with the deviation codec (16-bit).
//  * GEN = false is the configuration default omega_bulk = omega3 = omega4 = 1: third- and
//    fifth-order post-collision cumulants and the off-diagonal fourth-order ones vanish and the
//    trace relaxes to its equilibrium, so only the ten central moments the relaxation reads are
//    formed. GEN = true forms every moment and relaxes with the case's rates.
//
// The WALE eddy viscosity takes the velocity differences v(x+1) - v(x-1) without their factor
// 1/2: the eddy viscosity is homogeneous of degree one in the gradient and the scale is a power
// of two, so with the thresholds and the constant rescaled the result is bit for bit that of
// the halved gradient.
#pragma once
#include "common.cuh"
#include "vmath.cuh"
#include "cumulant_math.cuh"

namespace oal {

// max(v, c) per lane with NaN propagating (Julia's max), one instruction per lane
__device__ __forceinline__ float fmax_nan(float a, float b) { float r; asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b)); return r; }
__device__ __forceinline__ float fmin_nan(float a, float b) { float r; asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b)); return r; }
__device__ __forceinline__ F2 pmaxc(F2 v, float c) { return f2(fmax_nan(f2lo(v), c), fmax_nan(f2hi(v), c)); }
// clamp to [lo, hi] (lo <= hi), NaN passes
__device__ __forceinline__ F2 pclamp(F2 v, F2 lo, F2 hi) {
  return f2(fmin_nan(fmax_nan(f2lo(v), f2lo(lo)), f2lo(hi)), fmin_nan(fmax_nan(f2hi(v), f2hi(lo)), f2hi(hi)));
}
__device__ __forceinline__ F2 pclampc(F2 v, float lo, float hi) {
  return f2(fmin_nan(fmax_nan(f2lo(v), lo), hi), fmin_nan(fmax_nan(f2hi(v), lo), hi));
}

template <bool DEV>
struct PairScale {
  static constexpr float L = DEV ? 4.0f : 1.0f;       // relative scale of m1, m2 along each axis
  static constexpr float E = DEV ? 3.375f : 1.0f;     // 27/8: the weights' common factor
};

// number of nonzero indices of moment position k = a + 3b + 9c
__host__ __device__ constexpr int mom_nz(int k) { return (k % 3 != 0) + ((k / 3) % 3 != 0) + (k / 9 != 0); }
__host__ __device__ constexpr bool mom_even(int k) { return k % 3 != 1 && (k / 3) % 3 != 1 && k / 9 != 1; }
// moments of the lattice weights in the scaled form: prod chi(index), chi(0) = 3/2, chi(2) = 2
__host__ __device__ constexpr float mom_w(int k) {
  return (k % 3 == 0 ? 1.5f : 2.0f) * ((k / 3) % 3 == 0 ? 1.5f : 2.0f) * (k / 9 == 0 ? 1.5f : 2.0f);
}

// one line of the raw sums: (a, b, c) at c_axis = -1, 0, +1 -> (m0, m1, m2)
template <bool DEV>
__device__ __forceinline__ void raw_line(F2& a, F2& b, F2& c) {
  const F2 s = a + c, d = c - a;
  a = DEV ? vfma(splat<F2>(0.25f), s, b) : s + b;
  b = d;
  c = s;
}
template <bool DEV>
__device__ __forceinline__ F2 raw_m0(F2 a, F2 b, F2 c) {
  const F2 s = a + c;
  return DEV ? vfma(splat<F2>(0.25f), s, b) : s + b;
}

// raw moments in place: A[a + 3b + 9c] = M_abc (scaled). GEN = false leaves the moments with
// three nonzero indices unformed (unused at the default rates).
template <bool DEV, bool GEN>
__device__ __forceinline__ void raw_moments(F2 (&A)[kQ27]) {
#pragma unroll
  for (int n = 0; n < 9; ++n) raw_line<DEV>(A[3 * n], A[3 * n + 1], A[3 * n + 2]);
#pragma unroll
  for (int iz = 0; iz < 3; ++iz)
#pragma unroll
    for (int ma = 0; ma < 3; ++ma) raw_line<DEV>(A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz]);
#pragma unroll
  for (int n = 0; n < 9; ++n) {
    if (GEN || (n % 3 == 0) || (n / 3 == 0)) raw_line<DEV>(A[n], A[n + 9], A[n + 18]);
    else A[n] = raw_m0<DEV>(A[n], A[n + 9], A[n + 18]);
  }
  if constexpr (DEV) {
#pragma unroll
    for (int k = 0; k < kQ27; ++k)
      if (mom_even(k) && (GEN || mom_nz(k) < 3) && k != 26) A[k] = A[k] + splat<F2>(mom_w(k));
  }
}

// the shift of one line to central moments, scaled: (m0, m1', m2') -> (m0, k1', k2')
struct Shift {
  F2 nLu, n2u, Lu2;
};
template <bool DEV>
__device__ __forceinline__ Shift make_shift(F2 u) {
  constexpr float L = PairScale<DEV>::L;
  Shift s;
  s.n2u = u * splat<F2>(-2.0f);
  s.nLu = DEV ? s.n2u + s.n2u : u * splat<F2>(-1.0f);
  s.Lu2 = u * (u * splat<F2>(L));
  return s;
}
__device__ __forceinline__ F2 sh1(const Shift& s, F2 m0, F2 m1) { return vfma(s.nLu, m0, m1); }
__device__ __forceinline__ F2 sh2(const Shift& s, F2 m0, F2 m1, F2 m2) { return vfma(s.Lu2, m0, vfma(s.n2u, m1, m2)); }
__device__ __forceinline__ void sh12(const Shift& s, F2 m0, F2& m1, F2& m2) {
  const F2 k2 = sh2(s, m0, m1, m2);
  m1 = sh1(s, m0, m1);
  m2 = k2;
}

// backward line on normalised moments: (k0, k1, k2) -> (m2 - m1, k0 - m2, m2 + m1), i.e. twice
// the c = -1 population, the c = 0 one and twice the c = +1 one
struct Back {
  F2 u, tu, u2;
};
__device__ __forceinline__ Back make_back(F2 u) { return Back{u, u + u, u * u}; }
__device__ __forceinline__ void bwd_line(const Back& q, F2& a, F2& b, F2& c) {
  const F2 m1 = vfma(q.u, a, b);
  const F2 m2 = vfma(q.u2, a, vfma(q.tu, b, c));
  const F2 k0 = a;
  a = m2 - m1;
  b = k0 - m2;
  c = m2 + m1;
}
// (k0, 0, k2)
__device__ __forceinline__ void bwd_line_a(const Back& q, F2 k0, F2 k2, F2& a, F2& b, F2& c) {
  const F2 m1 = q.u * k0;
  const F2 m2 = vfma(q.u2, k0, k2);
  a = m2 - m1;
  b = k0 - m2;
  c = m2 + m1;
}
// (0, k1, 0)
__device__ __forceinline__ void bwd_line_b(const Back& q, F2 k1, F2& a, F2& b, F2& c) {
  const F2 m2 = q.tu * k1;
  a = m2 - k1;
  b = m2 * splat<F2>(-1.0f);
  c = m2 + k1;
}
// (1, 0, k2)
__device__ __forceinline__ void bwd_line_o(const Back& q, F2 k2, F2& a, F2& b, F2& c) {
  const F2 m2 = k2 + q.u2;
  a = m2 - q.u;
  b = splat<F2>(1.0f) - m2;
  c = m2 + q.u;
}

// WALE eddy viscosity from the doubled velocity differences d_ij = 2 g_ij (wale_nu's arithmetic
// with every operand scaled by a power of two; bit-identical to wale_nu on g)
__device__ __forceinline__ F2 wale_nu_2g(F2 g11, F2 g12, F2 g13, F2 g21, F2 g22, F2 g23, F2 g31, F2 g32, F2 g33,
                                         float c_wale) {
  const F2 third = splat<F2>(1.0f / 3.0f), half = splat<F2>(0.5f);
  const F2 gsq11 = vfma(g13, g31, vfma(g12, g21, g11 * g11));
  const F2 gsq22 = vfma(g23, g32, vfma(g22, g22, g21 * g12));
  const F2 gsq33 = vfma(g33, g33, vfma(g32, g23, g31 * g13));
  const F2 gsq12 = vfma(g13, g32, vfma(g12, g22, g11 * g12));
  const F2 gsq13 = vfma(g13, g33, vfma(g12, g23, g11 * g13));
  const F2 gsq21 = vfma(g23, g31, vfma(g22, g21, g21 * g11));
  const F2 gsq23 = vfma(g23, g33, vfma(g22, g23, g21 * g13));
  const F2 gsq31 = vfma(g33, g31, vfma(g32, g21, g31 * g11));
  const F2 gsq32 = vfma(g33, g32, vfma(g32, g22, g31 * g12));
  const F2 tr = ((gsq11 + gsq22) + gsq33) * third;
  const F2 Sd11 = gsq11 - tr, Sd22 = gsq22 - tr, Sd33 = gsq33 - tr;
  // 2 Sd_ij^2 = (gsq_ij + gsq_ji)^2 / 2 and 2 S_ij^2 = (g_ij + g_ji)^2 / 2, exactly
  const F2 s12 = gsq12 + gsq21, s13 = gsq13 + gsq31, s23 = gsq23 + gsq32;
  const F2 t12 = g12 + g21, t13 = g13 + g31, t23 = g23 + g32;
  const F2 OP1 = vfma(half, vfma(s23, s23, vfma(s13, s13, s12 * s12)), vfma(Sd33, Sd33, vfma(Sd22, Sd22, Sd11 * Sd11)));
  const F2 OP2 = vfma(half, vfma(t23, t23, vfma(t13, t13, t12 * t12)), vfma(g33, g33, vfma(g22, g22, g11 * g11)));
  // OP1 and OP2 are 16x and 4x those of the halved gradient: thresholds 16e-12, 4e-12, 32e-12
  const F2 OP1_32 = OP1 * vsqrt(OP1);
  const F2 OP2_52 = OP2 * OP2 * vsqrt(pmaxc(OP2, 4e-12f));
  const F2 den = vfma(OP1, vsqrt(vsqrt(pmaxc(OP1, 16e-12f))), OP2_52);
  const F2 cw2 = splat<F2>(c_wale * c_wale * 0.5f);
  const F2 nu = cw2 * OP1_32 * vrcp(den);
  const F2 zero = splat<F2>(0.0f);
  return vsel_gt(OP1, splat<F2>(16e-12f), vsel_gt(den, splat<F2>(32e-12f), nu, zero), zero);
}

// omega_1 from the eddy viscosity (omega1_from with the one-instruction NaN-propagating max)
__device__ __forceinline__ F2 omega1_pairs(F2 nu_eddy, const CaseParams& cp) {
  nu_eddy = nu_eddy * splat<F2>(cp.amr_sgs_scale);
  nu_eddy = pmaxc(nu_eddy, cp.nu_sgs_bg * cp.amr_sgs_scale);
  const float nu_mol = (cp.tau - 0.5f) * (1.0f / 3.0f);
  const F2 tau_eff = vfma(splat<F2>(3.0f), splat<F2>(nu_mol) + nu_eddy, splat<F2>(0.5f));
  return vrcp(pmaxc(tau_eff, 0.500001f));
}

// adaptive omega_4 of the diagonal fourth-order group (kernel_cumulant.jl:602-610): 1 - omega_4
__device__ __forceinline__ F2 one_minus_omega4_diag(F2 omega1, const CaseParams& cp) {
  if (cp.flags & CF_ADAPTIVE_OMEGA4) {
    const F2 om = omega1 - splat<F2>(2.0f);
    const F2 Av = (om * om) * splat<F2>(-1.0f) * vrcp(vfma(splat<F2>(cp.lambda_param), omega1, splat<F2>(1e-10f)));
    return splat<F2>(1.0f) - pclampc(Av, 0.01f, 2.0f);
  }
  return splat<F2>(1.0f - cp.omega4);
}

// factored limiter of the off-diagonal second-order cumulants (kernel_cumulant.jl:726-735)
__device__ __forceinline__ F2 factored_limit(F2 c, F2 a, F2 b) {
  const F2 bnd = vsqrt(pmaxc(a * b, 0.0f));
  return pclamp(c, bnd * splat<F2>(-1.0f), bnd);
}

// The collision after the raw moments: A holds M_abc (scaled, raw_moments), m000 = E rho_raw,
// inv = 1 / max(m000, 0.01 E), (ux, uy, uz) the velocity. On return A[k] holds f_k 2^n / rho_raw
// (n = |c_k|_1), every population of the post-collision state.
template <bool DEV, bool GEN>
__device__ __forceinline__ void collide_scaled(F2 (&A)[kQ27], F2 inv, F2 ux, F2 uy, F2 uz, F2 omega1,
                                               const CaseParams& cp) {
  constexpr float L = PairScale<DEV>::L;
  const F2 one = splat<F2>(1.0f), two = splat<F2>(2.0f), third = splat<F2>(1.0f / 3.0f);
  const F2 i4 = DEV ? inv * splat<F2>(1.0f / L) : inv;
  const F2 i16 = DEV ? inv * splat<F2>(1.0f / (L * L)) : inv;
  const Shift sx = make_shift<DEV>(ux), sy = make_shift<DEV>(uy), sz = make_shift<DEV>(uz);
  const F2 om1c = one - omega1;
  const F2 o4d = one_minus_omega4_diag(omega1, cp);

  if constexpr (!GEN) {
    // ---- central moments at the default rates: the ten the relaxation reads ----
    sh12(sx, A[0], A[1], A[2]);
    sh12(sx, A[3], A[4], A[5]);
    sh12(sx, A[6], A[7], A[8]);
    sh12(sx, A[9], A[10], A[11]);
    sh12(sx, A[18], A[19], A[20]);
    sh12(sy, A[0], A[3], A[6]);
    sh12(sy, A[9], A[12], A[15]);
    sh12(sy, A[18], A[21], A[24]);
    A[4] = sh1(sy, A[1], A[4]);
    A[8] = sh2(sy, A[2], A[5], A[8]);
    A[18] = sh2(sz, A[0], A[9], A[18]);
    A[10] = sh1(sz, A[1], A[10]);
    A[12] = sh1(sz, A[3], A[12]);
    A[20] = sh2(sz, A[2], A[11], A[20]);
    A[24] = sh2(sz, A[6], A[15], A[24]);

    // ---- cumulants and relaxation (kernel_cumulant.jl:661-754) ----
    const F2 c200 = A[2] * i4, c020 = A[6] * i4, c002 = A[18] * i4;
    const F2 c110 = A[4] * i16, c101 = A[10] * i16, c011 = A[12] * i16;
    const F2 C220 = A[8] * i16 - vfma(c200, c020, (c110 + c110) * c110);
    const F2 C202 = A[20] * i16 - vfma(c200, c002, (c101 + c101) * c101);
    const F2 C022 = A[24] * i16 - vfma(c020, c002, (c011 + c011) * c011);
    // the trace relaxes to its equilibrium 1 (omega_bulk = 1)
    const F2 D1_s = om1c * (c200 - c020);
    const F2 D2_s = om1c * (c200 - c002);
    const F2 t1 = one + D1_s;
    const F2 c200s = (t1 + D2_s) * third;
    const F2 c020s = (vfma(splat<F2>(-2.0f), D1_s, one) + D2_s) * third;
    const F2 c002s = vfma(splat<F2>(-2.0f), D2_s, t1) * third;
    F2 c110s = om1c * c110, c101s = om1c * c101, c011s = om1c * c011;
    if (cp.flags & CF_LIMITER_FACTORED) {
      c110s = factored_limit(c110s, c200s, c020s);
      c101s = factored_limit(c101s, c200s, c002s);
      c011s = factored_limit(c011s, c020s, c002s);
    }
    const F2 C220s = o4d * C220, C202s = o4d * C202, C022s = o4d * C022;
    // ---- reconstruction (kernel_cumulant.jl:759-781) ----
    const F2 t110 = c110s + c110s, t101 = c101s + c101s, t011 = c011s + c011s;
    const F2 c220s = vfma(t110, c110s, vfma(c200s, c020s, C220s));
    const F2 c202s = vfma(t101, c101s, vfma(c200s, c002s, C202s));
    const F2 c022s = vfma(t011, c011s, vfma(c020s, c002s, C022s));
    const F2 c211s = vfma(t110, c101s, c200s * c011s);
    const F2 c121s = vfma(t110, c011s, c020s * c101s);
    const F2 c112s = vfma(t101, c011s, c002s * c110s);
    F2 c222s = vfma(c002s, C220s, vfma(c020s, C202s, c200s * C022s));
    const F2 tri = vfma(c002s * c110s, c110s, vfma(c020s * c101s, c101s, c200s * c011s * c011s));
    c222s = c222s + vfma(splat<F2>(8.0f) * c110s, c101s * c011s, vfma(two, tri, c200s * c020s * c002s));

    // ---- backward z on the normalised moments (zero first, third and fifth orders) ----
    const Back bz = make_back(uz);
    bwd_line_o(bz, c002s, A[0], A[9], A[18]);
    bwd_line_b(bz, c101s, A[1], A[10], A[19]);
    bwd_line_a(bz, c200s, c202s, A[2], A[11], A[20]);
    bwd_line_b(bz, c011s, A[3], A[12], A[21]);
    bwd_line_a(bz, c110s, c112s, A[4], A[13], A[22]);
    bwd_line_b(bz, c211s, A[5], A[14], A[23]);
    bwd_line_a(bz, c020s, c022s, A[6], A[15], A[24]);
    bwd_line_b(bz, c121s, A[7], A[16], A[25]);
    bwd_line_a(bz, c220s, c222s, A[8], A[17], A[26]);
  } else {
    // ---- every central moment (any rates) ----
#pragma unroll
    for (int n = 0; n < 9; ++n) sh12(sx, A[3 * n], A[3 * n + 1], A[3 * n + 2]);
#pragma unroll
    for (int iz = 0; iz < 3; ++iz)
#pragma unroll
      for (int ma = 0; ma < 3; ++ma) sh12(sy, A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz]);
#pragma unroll
    for (int n = 0; n < 9; ++n) sh12(sz, A[n], A[n + 9], A[n + 18]);
    const F2 i64 = DEV ? inv * splat<F2>(1.0f / (L * L * L)) : inv;
    const F2 c200 = A[2] * i4, c020 = A[6] * i4, c002 = A[18] * i4;
    const F2 c110 = A[4] * i16, c101 = A[10] * i16, c011 = A[12] * i16;
    const F2 c210 = A[5] * i16, c120 = A[7] * i16, c201 = A[11] * i16;
    const F2 c021 = A[15] * i16, c102 = A[19] * i16, c012 = A[21] * i16;
    const F2 c111 = A[13] * i64;
    const F2 C220 = A[8] * i16 - vfma(c200, c020, (c110 + c110) * c110);
    const F2 C202 = A[20] * i16 - vfma(c200, c002, (c101 + c101) * c101);
    const F2 C022 = A[24] * i16 - vfma(c020, c002, (c011 + c011) * c011);
    const F2 C211 = A[14] * i64 - vfma(c200, c011, (c110 + c110) * c101);
    const F2 C121 = A[16] * i64 - vfma(c020, c101, (c110 + c110) * c011);
    const F2 C112 = A[22] * i64 - vfma(c002, c110, (c101 + c101) * c011);
    const F2 ob = splat<F2>(cp.omega_bulk);
    const F2 Dtr = (c200 + c020) + c002;
    const F2 Dtr_s = vfma(one - ob, Dtr, ob);
    const F2 D1_s = om1c * (c200 - c020);
    const F2 D2_s = om1c * (c200 - c002);
    const F2 c200s = ((Dtr_s + D1_s) + D2_s) * third;
    const F2 c020s = (vfma(splat<F2>(-2.0f), D1_s, Dtr_s) + D2_s) * third;
    const F2 c002s = vfma(splat<F2>(-2.0f), D2_s, Dtr_s + D1_s) * third;
    F2 c110s = om1c * c110, c101s = om1c * c101, c011s = om1c * c011;
    if (cp.flags & CF_LIMITER_FACTORED) {
      c110s = factored_limit(c110s, c200s, c020s);
      c101s = factored_limit(c101s, c200s, c002s);
      c011s = factored_limit(c011s, c020s, c002s);
    }
    const F2 o3 = one - splat<F2>(cp.omega3);
    const F2 c210s = o3 * c210, c120s = o3 * c120, c201s = o3 * c201;
    const F2 c021s = o3 * c021, c102s = o3 * c102, c012s = o3 * c012, c111s = o3 * c111;
    const F2 o4 = one - splat<F2>(cp.omega4);
    const F2 C220s = o4d * C220, C202s = o4d * C202, C022s = o4d * C022;
    const F2 C211s = o4 * C211, C121s = o4 * C121, C112s = o4 * C112;
    const F2 four = splat<F2>(4.0f);
    const F2 c220s = vfma(c110s + c110s, c110s, vfma(c200s, c020s, C220s));
    const F2 c202s = vfma(c101s + c101s, c101s, vfma(c200s, c002s, C202s));
    const F2 c022s = vfma(c011s + c011s, c011s, vfma(c020s, c002s, C022s));
    const F2 c211s = vfma(c110s + c110s, c101s, vfma(c200s, c011s, C211s));
    const F2 c121s = vfma(c110s + c110s, c011s, vfma(c020s, c101s, C121s));
    const F2 c112s = vfma(c101s + c101s, c011s, vfma(c002s, c110s, C112s));
    const F2 c221s = vfma(c011s + c011s, c210s, vfma(c101s + c101s, c120s, vfma(four * c110s, c111s, vfma(c020s, c201s, c200s * c021s))));
    const F2 c212s = vfma(c011s + c011s, c201s, vfma(four * c101s, c111s, vfma(c110s + c110s, c102s, vfma(c002s, c210s, c200s * c012s))));
    const F2 c122s = vfma(c101s + c101s, c021s, vfma(four * c011s, c111s, vfma(c110s + c110s, c012s, vfma(c002s, c120s, c020s * c102s))));
    F2 c222s = vfma(c002s, C220s, vfma(c020s, C202s, c200s * C022s));
    c222s = vfma(four, vfma(c011s, C211s, vfma(c101s, C121s, c110s * C112s)), c222s);
    c222s = c222s + vfma(four * c111s, c111s, two * vfma(c120s, c102s, vfma(c201s, c021s, c210s * c012s)));
    const F2 tri = vfma(c002s * c110s, c110s, vfma(c020s * c101s, c101s, c200s * c011s * c011s));
    c222s = c222s + vfma(splat<F2>(8.0f) * c110s, c101s * c011s, vfma(two, tri, c200s * c020s * c002s));
    const F2 zero = splat<F2>(0.0f);
    A[0] = one; A[1] = zero; A[3] = zero; A[9] = zero;
    A[2] = c200s; A[6] = c020s; A[18] = c002s;
    A[4] = c110s; A[10] = c101s; A[12] = c011s;
    A[5] = c210s; A[7] = c120s; A[11] = c201s;
    A[15] = c021s; A[19] = c102s; A[21] = c012s;
    A[13] = c111s;
    A[8] = c220s; A[20] = c202s; A[24] = c022s;
    A[14] = c211s; A[16] = c121s; A[22] = c112s;
    A[17] = c221s; A[23] = c212s; A[25] = c122s;
    A[26] = c222s;
    const Back bz = make_back(uz);
#pragma unroll
    for (int n = 0; n < 9; ++n) bwd_line(bz, A[n], A[n + 9], A[n + 18]);
  }
  // ---- backward y, x (kernel_cumulant.jl:810-844) ----
  const Back by = make_back(uy), bx = make_back(ux);
#pragma unroll
  for (int iz = 0; iz < 3; ++iz)
#pragma unroll
    for (int ma = 0; ma < 3; ++ma) bwd_line(by, A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz]);
#pragma unroll
  for (int n = 0; n < 9; ++n) bwd_line(bx, A[3 * n], A[3 * n + 1], A[3 * n + 2]);
}

}  // namespace oal
