// cumulant_math.cuh — the D3Q27 cumulant collision, WALE eddy viscosity and equilibria, written
// once for any lane type V (float, double, or F2 = two cells per thread).
//
// Arithmetic follows src/collision/kernel_cumulant.jl with three deliberate changes of rounding
// only: multiply-adds are fused (explicit vfma), divisions by 3 are multiplications by 1/3, and
// in float the reciprocals and square roots are the hardware approximations (<= 2 ulp).
#pragma once
#include "common.cuh"
#include "vmath.cuh"

namespace oal {

template <class V>
using SC = typename Lane<V>::S;

// physics_utils.jl:30-109 — f_eq for direction k (compile-time k after unrolling)
template <class V>
__device__ __forceinline__ V feq_k(int k, V rho, V ux, V uy, V uz, bool comp) {
  using T = SC<V>;
  const int cx = q27_cx(k), cy = q27_cy(k), cz = q27_cz(k);
  V cu = splat<V>(T(0));
  if (cx) cu = cx > 0 ? cu + ux : cu - ux;
  if (cy) cu = cy > 0 ? cu + uy : cu - uy;
  if (cz) cu = cz > 0 ? cu + uz : cu - uz;
  const V usq = vfma(uz, uz, vfma(uy, uy, ux * ux));
  // 1 + 3cu + 4.5cu^2 - 1.5usq
  V val = vfma(splat<V>(T(-1.5)), usq, vfma(splat<V>(T(4.5)) * cu, cu, vfma(splat<V>(T(3)), cu, splat<V>(T(1)))));
  if (comp) {
    const V cu2 = cu * cu;
    const V ho3 = vfma(splat<V>(T(4.5)) * cu2, cu, splat<V>(T(-4.5)) * cu * usq);
    const V ho4 = vfma(splat<V>(T(1.125)) * usq, usq, vfma(splat<V>(T(3.375)) * cu2, cu2, splat<V>(T(-6.75)) * cu2 * usq));
    val = val + (ho3 + ho4);
  }
  return rho * splat<V>(T(q27_w(k))) * val;
}

// f_eq with a run-time velocity c and weight w (physics_utils.jl:30-35, 65-95), the reference's
// operation order; the block-AMR transfers evaluate it at interpolated macros
template <class R>
__device__ __forceinline__ R feq_c(R rho, R ux, R uy, R uz, R w, R cx, R cy, R cz, bool comp) {
  const R cu = cx * ux + cy * uy + cz * uz;
  const R usq = ux * ux + uy * uy + uz * uz;
  if (!comp) return rho * w * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq);
  const R cu2 = cu * cu, cu3 = cu2 * cu, cu4 = cu2 * cu2, usq2 = usq * usq;
  R val = R(1) + R(3) * cu + R(4.5) * cu2 - R(1.5) * usq;
  const R ho = (R(4.5) * cu3 - R(4.5) * cu * usq) + (R(3.375) * cu4 - R(6.75) * cu2 * usq + R(1.125) * usq2);
  val += ho;
  return rho * w * val;
}

// WALE eddy viscosity from the velocity gradient g_ij = d u_i / d x_j (kernel_cumulant.jl:505-549)
template <class V>
__device__ __forceinline__ V wale_nu(V g11, V g12, V g13, V g21, V g22, V g23, V g31, V g32, V g33, float c_wale) {
  using T = SC<V>;
  const V h = splat<V>(T(0.5)), third = splat<V>(T(1.0 / 3.0)), two = splat<V>(T(2));
  const V gsq11 = vfma(g13, g31, vfma(g12, g21, g11 * g11));
  const V gsq12 = vfma(g13, g32, vfma(g12, g22, g11 * g12));
  const V gsq13 = vfma(g13, g33, vfma(g12, g23, g11 * g13));
  const V gsq21 = vfma(g23, g31, vfma(g22, g21, g21 * g11));
  const V gsq22 = vfma(g23, g32, vfma(g22, g22, g21 * g12));
  const V gsq23 = vfma(g23, g33, vfma(g22, g23, g21 * g13));
  const V gsq31 = vfma(g33, g31, vfma(g32, g21, g31 * g11));
  const V gsq32 = vfma(g33, g32, vfma(g32, g22, g31 * g12));
  const V gsq33 = vfma(g33, g33, vfma(g32, g23, g31 * g13));
  const V tr = ((gsq11 + gsq22) + gsq33) * third;
  const V Sd11 = gsq11 - tr, Sd22 = gsq22 - tr, Sd33 = gsq33 - tr;
  const V Sd12 = h * (gsq12 + gsq21), Sd13 = h * (gsq13 + gsq31), Sd23 = h * (gsq23 + gsq32);
  const V S12 = h * (g12 + g21), S13 = h * (g13 + g31), S23 = h * (g23 + g32);
  const V OP1 = vfma(two, vfma(Sd23, Sd23, vfma(Sd13, Sd13, Sd12 * Sd12)), vfma(Sd33, Sd33, vfma(Sd22, Sd22, Sd11 * Sd11)));
  const V OP2 = vfma(two, vfma(S23, S23, vfma(S13, S13, S12 * S12)), vfma(g33, g33, vfma(g22, g22, g11 * g11)));
  const V eps = splat<V>(T(1e-12));
  const V OP1_32 = OP1 * vsqrt(OP1);
  const V OP2_52 = OP2 * OP2 * vsqrt(vmaxc(OP2, T(1e-12)));
  const V den = vfma(OP1, vsqrt(vsqrt(vmaxc(OP1, T(1e-12)))), OP2_52);
  const V cw2 = splat<V>(T(c_wale) * T(c_wale));
  const V nu = cw2 * OP1_32 * vrcp(den);
  const V zero = splat<V>(T(0));
  return vsel_gt(OP1, eps, vsel_gt(den, eps, nu, zero), zero);
}

// Germano-Lilly dynamic Smagorinsky coefficient Cs^2 in [0, 0.25] (kernel_dynamic_sgs.jl:128-240):
// 7-point box test filter of the velocity (the cell's current velocity c and its six face
// neighbours' previous-step velocities, the centre value standing in for missing or solid ones),
// Leonard stress, test-scale modelled stress from the grid strain (g11, g22, g33 and the
// symmetric S12, S13, S23), Lilly's least-squares contraction. Dx = 1.
template <class R>
__device__ __forceinline__ R dynamic_cs2(const R (&c)[3], const R (&n)[6][3], R g11, R g22, R g33, R S12, R S13, R S23) {
  const R inv7 = R(1) / R(7);
  R ut[3], uu[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    R sum = c[a];
#pragma unroll
    for (int j = 0; j < 6; ++j) sum = sum + n[j][a];
    ut[a] = inv7 * sum;
  }
  const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    R sum = c[ia[m]] * c[ib[m]];
#pragma unroll
    for (int j = 0; j < 6; ++j) sum = sum + n[j][ia[m]] * n[j][ib[m]];
    uu[m] = inv7 * sum;
  }
  const R Lxx = uu[0] - ut[0] * ut[0], Lyy = uu[1] - ut[1] * ut[1], Lzz = uu[2] - ut[2] * ut[2];
  const R Lxy = uu[3] - ut[0] * ut[1], Lxz = uu[4] - ut[0] * ut[2], Lyz = uu[5] - ut[1] * ut[2];
  const R Ltr = (Lxx + Lyy + Lzz) * (R(1) / R(3));
  const R Lxx_d = Lxx - Ltr, Lyy_d = Lyy - Ltr, Lzz_d = Lzz - Ltr;
  const R S_sq = R(2) * (g11 * g11 + g22 * g22 + g33 * g33) + R(4) * (S12 * S12 + S13 * S13 + S23 * S23);
  const R S_mag = sqrt(S_sq > R(1e-30) ? S_sq : R(1e-30));
  const R M_coeff = R(2) * R(1) * R(1) * R(3.659306f) * S_mag;
  const R Mxx = M_coeff * g11, Myy = M_coeff * g22, Mzz = M_coeff * g33;
  const R Mxy = M_coeff * S12, Mxz = M_coeff * S13, Myz = M_coeff * S23;
  const R Mtr = (Mxx + Myy + Mzz) * (R(1) / R(3));
  const R Mxx_d = Mxx - Mtr, Myy_d = Myy - Mtr, Mzz_d = Mzz - Mtr;
  const R LM = Lxx_d * Mxx_d + Lyy_d * Myy_d + Lzz_d * Mzz_d + R(2) * (Lxy * Mxy + Lxz * Mxz + Lyz * Myz);
  const R MM = Mxx_d * Mxx_d + Myy_d * Myy_d + Mzz_d * Mzz_d + R(2) * (Mxy * Mxy + Mxz * Mxz + Myz * Myz);
  const R cd = R(0.5) * LM / (MM + R(1e-20));
  return cd > R(0.25) ? R(0.25) : (cd < R(0) ? R(0) : cd);
}

// nu_sgs of the stored post-collision Pi_neq (kernel_cumulant.jl:567-586): c_pi |Pi_pre| / (rho cs^2),
// |Pi_pre| = |tau / (tau - 1)| |Pi_post|, capped at 0.1
template <class R>
__device__ __forceinline__ R pi_stress_nu(const R (&pi)[6], R rho, const CaseParams& cp) {
  const R mag = sqrt(pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2] +
                     R(2) * (pi[3] * pi[3] + pi[4] * pi[4] + pi[5] * pi[5]));
  const R denom = R(cp.tau) - R(1);
  const R corr = fabs(denom) < R(1e-3) ? R(1) : R(cp.tau) / denom;
  const R pre = fabs(corr) * mag;
  const R rc = (!isfinite(rho) || rho < R(0.01)) ? R(1) : rho;
  const R nu = R(cp.c_pi) * pre / (rc * (R(1) / R(3)) + R(1e-10)) * R(cp.amr_sgs_scale);
  return nu < R(0.1) ? nu : R(0.1);
}

// Pi_neq_ab = sum_k c_a c_b (f_k - f_eq_k(rho, u)) of one cell (kernel_pi_neq.jl:120-180); zero for
// solid or unphysical cells
template <class R>
__device__ __forceinline__ void pi_neq_of(const R (&f)[kQ27], R rho, R ux, R uy, R uz, bool comp, bool skip, R (&pi)[6]) {
  const R rs = skip ? R(0) : rho, us = skip ? R(0) : ux, vs = skip ? R(0) : uy, ws = skip ? R(0) : uz;
  R p[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R cx = R(q27_cx(k)), cy = R(q27_cy(k)), cz = R(q27_cz(k));
    const R fe = feq_c<R>(rs, us, vs, ws, R(q27_w(k)), cx, cy, cz, comp);
    const R fn = (skip ? R(0) : f[k]) - fe;
    p[0] = p[0] + cx * cx * fn; p[1] = p[1] + cy * cy * fn; p[2] = p[2] + cz * cz * fn;
    p[3] = p[3] + cx * cy * fn; p[4] = p[4] + cx * cz * fn; p[5] = p[5] + cy * cz * fn;
  }
  const R mask = skip ? R(0) : R(1);
#pragma unroll
  for (int m = 0; m < 6; ++m) pi[m] = p[m] * mask;
}

// omega_1 from the final eddy viscosity (kernel_cumulant.jl:591-594)
template <class V>
__device__ __forceinline__ V omega1_of_nu(V nu_eddy, const CaseParams& cp) {
  using T = SC<V>;
  const T nu_mol = (T(cp.tau) - T(0.5)) * T(1.0 / 3.0);
  const V tau_eff = vfma(splat<V>(T(3)), splat<V>(nu_mol) + nu_eddy, splat<V>(T(0.5)));
  return vrcp(vmaxc(tau_eff, T(0.500001)));
}

// omega_1 from the WALE eddy viscosity with the background floor (kernel_cumulant.jl:546-590)
template <class V>
__device__ __forceinline__ V omega1_from(V nu_eddy, const CaseParams& cp) {
  using T = SC<V>;
  nu_eddy = nu_eddy * splat<V>(T(cp.amr_sgs_scale));
  nu_eddy = vmaxc(nu_eddy, T(cp.nu_sgs_bg) * T(cp.amr_sgs_scale));
  return omega1_of_nu<V>(nu_eddy, cp);
}

template <class V>
__device__ __forceinline__ void chimera_fwd3(V& a, V& b, V& c, V nu, V n2u, V u2) {
  const V m0 = (a + b) + c, m1 = c - a, m2 = a + c;
  a = m0;
  b = vfma(nu, m0, m1);
  c = vfma(u2, m0, vfma(n2u, m1, m2));
}
template <class V>
__device__ __forceinline__ void chimera_bwd3(V& a, V& b, V& c, V u, V tu, V u2) {
  const V m0 = a;
  const V m1 = vfma(u, a, b);
  const V m2 = vfma(u2, a, vfma(tu, b, c));
  const V h = splat<V>(SC<V>(0.5));
  a = (m2 - m1) * h;
  b = m0 - m2;
  c = (m2 + m1) * h;
}

// the blend of the positivity limiter in the lanes whose minimum population fmin is negative:
// f = f_eq + alpha (f - f_eq), alpha the largest factor keeping every population >= 0
// (kernel_cumulant.jl:856-884)
// Grad-reconstruction wall at wall velocity 0 (grad_wall_kernel.jl:100-136): Pi_neq of the
// post-collision populations A about (rho, 0), scaled by pineq_scale, then every population
// rebuilt as rho w_k + (1 - omega) w_k 4.5 Q_k : Pi_neq, Q_ab = c_a c_b - delta_ab / 3, floored at
// 1e-12 (NaN passes, as the reference's max).
template <class R>
__device__ __forceinline__ void grad_wall(R (&A)[kQ27], R rho, R omega, R pineq_scale) {
  R pxx = R(0), pyy = R(0), pzz = R(0), pxy = R(0), pyz = R(0), pzx = R(0);
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R cx = R(q27_cx(k)), cy = R(q27_cy(k)), cz = R(q27_cz(k));
    const R fneq = A[k] - rho * R(q27_w(k));
    pxx = pxx + fneq * cx * cx; pyy = pyy + fneq * cy * cy; pzz = pzz + fneq * cz * cz;
    pxy = pxy + fneq * cx * cy; pyz = pyz + fneq * cy * cz; pzx = pzx + fneq * cz * cx;
  }
  pxx = pxx * pineq_scale; pyy = pyy * pineq_scale; pzz = pzz * pineq_scale;
  pxy = pxy * pineq_scale; pyz = pyz * pineq_scale; pzx = pzx * pineq_scale;
  const R cs2 = R(1) / R(3), inv_2cs4 = R(0.5) / (cs2 * cs2), one_m_w = R(1) - omega;
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R cx = R(q27_cx(k)), cy = R(q27_cy(k)), cz = R(q27_cz(k)), wk = R(q27_w(k));
    const R qxx = cx * cx - cs2, qyy = cy * cy - cs2, qzz = cz * cz - cs2;
    const R reg = wk * inv_2cs4 *
                  (pxx * qxx + pyy * qyy + pzz * qzz + R(2) * (pxy * cx * cy + pyz * cy * cz + pzx * cz * cx));
    A[k] = vmaxc(rho * wk + one_m_w * reg, R(1e-12));
  }
}

// opaque copy: the compiler may not assume the value equals its source, so expressions of it are
// recomputed rather than kept alive from earlier
__device__ __forceinline__ float opaque(float v) { asm volatile("" : "+f"(v)); return v; }
__device__ __forceinline__ double opaque(double v) { asm volatile("" : "+d"(v)); return v; }
__device__ __forceinline__ F2 opaque(F2 v) { asm volatile("" : "+l"(v.v)); return v; }

#ifndef OAL_LIMITER_OUTLINE
#define OAL_LIMITER_OUTLINE 0
#endif
#if OAL_LIMITER_OUTLINE
#define OAL_LIMITER_LINKAGE __noinline__
#else
#define OAL_LIMITER_LINKAGE __forceinline__
#endif

template <class V>
__device__ OAL_LIMITER_LINKAGE void positivity_blend(V (&A)[kQ27], V fmin, V rho, V uxe, V uye, V uze, bool comp) {
  using T = SC<V>;
  const V zero = splat<V>(T(0)), one = splat<V>(T(1));
  V alpha = one;
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const V fe = feq_k<V>(k, rho, uxe, uye, uze, comp);
    const V fneq = A[k] - fe;
    const V ak = fe * vrcp((fe - fneq) + splat<V>(T(1e-15)));
    // alpha = min(alpha, ak) where fneq < 0 and fe > 1e-15
    alpha = vsel_gt(zero, fneq, vsel_gt(fe, splat<V>(T(1e-15)), vmin(alpha, ak), alpha), alpha);
  }
  alpha = vmaxc(alpha, T(0));
  // the equilibria again (not 27 values kept alive across the two loops)
  rho = opaque(rho); uxe = opaque(uxe); uye = opaque(uye); uze = opaque(uze);
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const V fe = feq_k<V>(k, rho, uxe, uye, uze, comp);
    A[k] = vsel_gt(zero, fmin, vfma(alpha, A[k] - fe, fe), A[k]);
  }
}

// velocity-free half of the forward x pass: (a, b, c) -> (a + b + c, c - a, a + c)
template <class V>
__device__ __forceinline__ void chimera_xsums(V& a, V& b, V& c) {
  const V m0 = (a + b) + c, m1 = c - a, m2 = a + c;
  a = m0;
  b = m1;
  c = m2;
}

// Cumulant relaxation of A (post-streaming populations) at the equilibrium velocity (uxe,uye,uze)
// with omega_1 (kernel_cumulant.jl:597-844), then the positivity limiter (:849-884).
template <class V, bool POS = true>
__device__ __forceinline__ void cumulant_collide_xsums(V (&A)[kQ27], V rho, V uxe, V uye, V uze, V omega1,
                                                       const CaseParams& cp);
template <class V>
__device__ __forceinline__ void cumulant_collide(V (&A)[kQ27], V rho, V uxe, V uye, V uze, V omega1, const CaseParams& cp) {
#pragma unroll
  for (int n = 0; n < 9; ++n) chimera_xsums(A[3 * n], A[3 * n + 1], A[3 * n + 2]);
  cumulant_collide_xsums<V>(A, rho, uxe, uye, uze, omega1, cp);
}

// The same with the x triplets of A already replaced by their velocity-free sums (chimera_xsums);
// the x pass then only shifts them to the velocity: b = m1 - u m0, c = m2 - 2u m1 + u^2 m0.
// POS = false leaves the positivity limiter out (callers whose cases all run without it).
template <class V, bool POS>
__device__ __forceinline__ void cumulant_collide_xsums(V (&A)[kQ27], V rho, V uxe, V uye, V uze, V omega1,
                                                       const CaseParams& cp) {
  using T = SC<V>;
  const uint32_t flags = cp.flags;
  const V one = splat<V>(T(1)), two = splat<V>(T(2)), four = splat<V>(T(4)), third = splat<V>(T(1.0 / 3.0));

  // adaptive omega_4 of the diagonal group (kernel_cumulant.jl:602-610)
  const V omega4 = splat<V>(T(cp.omega4));
  V omega4_diag = omega4;
  if (flags & CF_ADAPTIVE_OMEGA4) {
    const V om = omega1 - two;
    const V Av = (om * om) * splat<V>(T(-1)) * vrcp(vfma(splat<V>(T(cp.lambda_param)), omega1, splat<V>(T(1e-10))));
    omega4_diag = vclamp(Av, splat<V>(T(0.01)), splat<V>(T(2)));
  }

  // chimera forward x (its velocity shift), y, z (kernel_cumulant.jl:612-656)
  {
    const V nu = uxe * splat<V>(T(-1)), n2u = uxe * splat<V>(T(-2)), u2 = uxe * uxe;
#pragma unroll
    for (int n = 0; n < 9; ++n) {
      const V m0 = A[3 * n], m1 = A[3 * n + 1], m2 = A[3 * n + 2];
      A[3 * n + 1] = vfma(nu, m0, m1);
      A[3 * n + 2] = vfma(u2, m0, vfma(n2u, m1, m2));
    }
  }
  {
    const V nu = uye * splat<V>(T(-1)), n2u = uye * splat<V>(T(-2)), u2 = uye * uye;
#pragma unroll
    for (int iz = 0; iz < 3; ++iz)
#pragma unroll
      for (int ma = 0; ma < 3; ++ma) chimera_fwd3(A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz], nu, n2u, u2);
  }
  {
    const V nu = uze * splat<V>(T(-1)), n2u = uze * splat<V>(T(-2)), u2 = uze * uze;
#pragma unroll
    for (int n = 0; n < 9; ++n) chimera_fwd3(A[n], A[n + 9], A[n + 18], nu, n2u, u2);
  }

  // central moments -> cumulants (kernel_cumulant.jl:661-699)
  const V k000 = A[0];
  const V inv_r = vrcp(vmaxc(k000, T(0.01)));
  const V c200 = A[2] * inv_r, c020 = A[6] * inv_r, c002 = A[18] * inv_r;
  const V c110 = A[4] * inv_r, c101 = A[10] * inv_r, c011 = A[12] * inv_r;
  const V c210 = A[5] * inv_r, c120 = A[7] * inv_r, c201 = A[11] * inv_r;
  const V c021 = A[15] * inv_r, c102 = A[19] * inv_r, c012 = A[21] * inv_r;
  const V c111 = A[13] * inv_r;
  const V C220 = A[8] * inv_r - vfma(c200, c020, (c110 + c110) * c110);
  const V C202 = A[20] * inv_r - vfma(c200, c002, (c101 + c101) * c101);
  const V C022 = A[24] * inv_r - vfma(c020, c002, (c011 + c011) * c011);
  const V C211 = A[14] * inv_r - vfma(c200, c011, (c110 + c110) * c101);
  const V C121 = A[16] * inv_r - vfma(c020, c101, (c110 + c110) * c011);
  const V C112 = A[22] * inv_r - vfma(c002, c110, (c101 + c101) * c011);

  // relaxation (kernel_cumulant.jl:705-754); the trace equilibrium 3 cs^2 is 1
  const V ob = splat<V>(T(cp.omega_bulk));
  const V Dtr = (c200 + c020) + c002;
  const V Dtr_s = vfma(one - ob, Dtr, ob);
  const V om1c = one - omega1;
  const V D1_s = om1c * (c200 - c020);
  const V D2_s = om1c * (c200 - c002);
  const V c200s = ((Dtr_s + D1_s) + D2_s) * third;
  const V c020s = (vfma(splat<V>(T(-2)), D1_s, Dtr_s) + D2_s) * third;
  const V c002s = vfma(splat<V>(T(-2)), D2_s, Dtr_s + D1_s) * third;
  V c110s = om1c * c110, c101s = om1c * c101, c011s = om1c * c011;
  if (flags & CF_LIMITER_FACTORED) {
    const V b110 = vsqrt(vmaxc(c200s * c020s, T(0)));
    const V b101 = vsqrt(vmaxc(c200s * c002s, T(0)));
    const V b011 = vsqrt(vmaxc(c020s * c002s, T(0)));
    const V m1 = splat<V>(T(-1));
    c110s = vclamp(c110s, b110 * m1, b110);
    c101s = vclamp(c101s, b101 * m1, b101);
    c011s = vclamp(c011s, b011 * m1, b011);
  }
  const V o3 = one - splat<V>(T(cp.omega3));
  const V c210s = o3 * c210, c120s = o3 * c120, c201s = o3 * c201;
  const V c021s = o3 * c021, c102s = o3 * c102, c012s = o3 * c012, c111s = o3 * c111;
  const V o4d = one - omega4_diag, o4 = one - omega4;
  const V C220s = o4d * C220, C202s = o4d * C202, C022s = o4d * C022;
  const V C211s = o4 * C211, C121s = o4 * C121, C112s = o4 * C112;

  // reconstruction (kernel_cumulant.jl:759-781)
  const V c220s = vfma(c110s + c110s, c110s, vfma(c200s, c020s, C220s));
  const V c202s = vfma(c101s + c101s, c101s, vfma(c200s, c002s, C202s));
  const V c022s = vfma(c011s + c011s, c011s, vfma(c020s, c002s, C022s));
  const V c211s = vfma(c110s + c110s, c101s, vfma(c200s, c011s, C211s));
  const V c121s = vfma(c110s + c110s, c011s, vfma(c020s, c101s, C121s));
  const V c112s = vfma(c101s + c101s, c011s, vfma(c002s, c110s, C112s));
  const V c221s = vfma(c011s + c011s, c210s, vfma(c101s + c101s, c120s, vfma(four * c110s, c111s, vfma(c020s, c201s, c200s * c021s))));
  const V c212s = vfma(c011s + c011s, c201s, vfma(four * c101s, c111s, vfma(c110s + c110s, c102s, vfma(c002s, c210s, c200s * c012s))));
  const V c122s = vfma(c101s + c101s, c021s, vfma(four * c011s, c111s, vfma(c110s + c110s, c012s, vfma(c002s, c120s, c020s * c102s))));
  V c222s = vfma(c002s, C220s, vfma(c020s, C202s, c200s * C022s));
  c222s = vfma(four, vfma(c011s, C211s, vfma(c101s, C121s, c110s * C112s)), c222s);
  c222s = c222s + vfma(four * c111s, c111s, two * vfma(c120s, c102s, vfma(c201s, c021s, c210s * c012s)));
  const V tri = vfma(c002s * c110s, c110s, vfma(c020s * c101s, c101s, c200s * c011s * c011s));
  c222s = c222s + vfma(splat<V>(T(8)) * c110s, c101s * c011s, vfma(two, tri, c200s * c020s * c002s));

  // post-collision central moments (kernel_cumulant.jl:786-804)
  const V r = k000;
  const V zero = splat<V>(T(0));
  A[0] = r; A[1] = zero; A[3] = zero; A[9] = zero;
  A[2] = r * c200s; A[6] = r * c020s; A[18] = r * c002s;
  A[4] = r * c110s; A[10] = r * c101s; A[12] = r * c011s;
  A[5] = r * c210s; A[7] = r * c120s; A[11] = r * c201s;
  A[15] = r * c021s; A[19] = r * c102s; A[21] = r * c012s;
  A[13] = r * c111s;
  A[8] = r * c220s; A[20] = r * c202s; A[24] = r * c022s;
  A[14] = r * c211s; A[16] = r * c121s; A[22] = r * c112s;
  A[17] = r * c221s; A[23] = r * c212s; A[25] = r * c122s;
  A[26] = r * c222s;

  // chimera backward z, y, x (kernel_cumulant.jl:810-844)
  {
    const V tu = uze + uze, u2 = uze * uze;
#pragma unroll
    for (int n = 0; n < 9; ++n) chimera_bwd3(A[n], A[n + 9], A[n + 18], uze, tu, u2);
  }
  {
    const V tu = uye + uye, u2 = uye * uye;
#pragma unroll
    for (int iz = 0; iz < 3; ++iz)
#pragma unroll
      for (int ma = 0; ma < 3; ++ma) chimera_bwd3(A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz], uye, tu, u2);
  }
  {
    const V tu = uxe + uxe, u2 = uxe * uxe;
#pragma unroll
    for (int n = 0; n < 9; ++n) chimera_bwd3(A[3 * n], A[3 * n + 1], A[3 * n + 2], uxe, tu, u2);
  }

  // positivity limiter (kernel_cumulant.jl:849-884)
  if (POS && (flags & CF_LIMITER_POSITIVITY)) {
    V fmin = A[0];
#pragma unroll
    for (int k = 1; k < kQ27; ++k) fmin = vmin(fmin, A[k]);
    if (vany_gt(zero, fmin)) positivity_blend<V>(A, fmin, rho, uxe, uye, uze, (flags & CF_COMPRESSIBLE) != 0);
  }
}

}  // namespace oal
