// oal_oracle_q39.cpp — CPU ORACLE (test infrastructure only) of the reference's D3Q39 entropic KBC
// level step (OpenAeroLab src/collision, Julia/KernelAbstractions, GPU), restated in binary32 with
// -ffp-contract=off, for a level without sponge, wall model, AMR parent, thermal coupling or
// lattice shift: periodic boxes (every block has its 26 neighbours), and levels with domain faces
// and obstacle cells (ora_q39_step_ex).
//
// Followed (paths inside the reference project):
//   D3Q39 velocity set, weights, opposites ........ src/collision/lattice.jl:177-262
//   13-moment Newton equilibrium, warm start and
//   staleness gate, evaluation, mass correction ... src/collision/physics_utils.jl:493-796
//   host inlet equilibrium (NaN-reset populations)  physics_utils.jl:280-460, timestep.jl:1169-1188
//   pull over |c| <= 3 through the neighbour table  src/collision/kernel_entropic_d3q39.jl:898-1290
//   domain faces (default boundary options) ...... kernel_entropic_d3q39.jl:983-1278 (kbc::face_value)
//   inlet-face mass + momentum pin ................ kernel_entropic_d3q39.jl:1313-1352,
//                                                   physics_utils.jl:830-900 (kbc::four_moment_pin)
//   obstacle cells (full-way bounce-back) ......... kernel_entropic_d3q39.jl:1602-1613
//   gradient neighbours: own value across a missing
//   block or into a solid cell .................... physics_utils.jl:1981-2035
//   macros, density floor, NaN reset .............. kernel_entropic_d3q39.jl:1616-1650
//   macro realizability clamp (far bulk), equilibrium
//   velocity cap .................................. kernel_entropic_d3q39.jl:2112-2287
//   13-moment f_eq with the lambda cache .......... kernel_entropic_d3q39.jl:2330-2385
//   velocity gradient (previous velocity) ......... physics_utils.jl:2217-2233
//   WALE, Mach-pocket viscosity, floors, tau_eff .. kernel_entropic_d3q39.jl:2588-2876
//   positivity clamp and realizability guard ...... kernel_entropic_d3q39.jl:2885-2958
//   mirror split, HRR blend, sigma damping ........ kernel_entropic_d3q39.jl:2962-3108
//   alpha solvers (bisection, Newton, approximate,
//   Taylor) and the entropy ....................... kernel_entropic_d3q39.jl:47-528, 3109-3150
//   KBC update, post blend, post guard, output .... kernel_entropic_d3q39.jl:3153-3368
//   sponge toward the inlet state, near-wall clamp  kernel_entropic_d3q39.jl:1662, 1787-1841, 2149-2168
//   spectral vanishing viscosity (y-z, then x) and
//   the positivity re-enforcement after it ....... kernel_entropic_d3q39.jl:3256-3310,
//                                                   kernel_svv_yz_d3q39.jl:78-213, 225-298
// Terms that vanish on such a level are written out where they change rounding (0 force, 0 frame
// shift); switches that are off there are left out: shock sensor, Knudsen-adaptive tau, variable
// nu_sgs / sigma, dynamic SGS, feathering, RR-LBM, Gendre correction, wall model.
// min/max propagate NaN as Julia's do. exp and log are kbc::exp / kbc::log (Cody-Waite reduction
// and series), shared with the CUDA kernel so the two agree bit for bit; the reference calls the
// Float32 exp / log of its backend.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <limits>

#include "../include/oal.h"
#include "../openaerolab_alpha_01_b200/csrc/kbc_math.h"

namespace {

constexpr int Q = 39;
int CX[Q], CY[Q], CZ[Q], OPP[Q];
float WT[Q];
bool tables_ready = false;

void build_tables() {
  if (tables_ready) return;
  int n = 0;
  auto push = [&](int x, int y, int z, float w) { CX[n] = x; CY[n] = y; CZ[n] = z; WT[n] = w; ++n; };
  push(0, 0, 0, float(1.0 / 12));
  for (int dim = 0; dim < 3; ++dim)
    for (int s : {-1, 1}) { int c[3] = {0, 0, 0}; c[dim] = s; push(c[0], c[1], c[2], float(1.0 / 12)); }
  for (int sx : {-1, 1})
    for (int sy : {-1, 1})
      for (int sz : {-1, 1}) push(sx, sy, sz, float(1.0 / 27));
  for (int dim = 0; dim < 3; ++dim)
    for (int s : {-1, 1}) { int c[3] = {0, 0, 0}; c[dim] = 2 * s; push(c[0], c[1], c[2], float(2.0 / 135)); }
  for (int d1 = 0; d1 < 3; ++d1)
    for (int d2 = d1 + 1; d2 < 3; ++d2)
      for (int s1 : {-1, 1})
        for (int s2 : {-1, 1}) { int c[3] = {0, 0, 0}; c[d1] = 2 * s1; c[d2] = 2 * s2; push(c[0], c[1], c[2], float(1.0 / 432)); }
  for (int dim = 0; dim < 3; ++dim)
    for (int s : {-1, 1}) { int c[3] = {0, 0, 0}; c[dim] = 3 * s; push(c[0], c[1], c[2], float(1.0 / 1620)); }
  for (int i = 0; i < Q; ++i)
    for (int j = 0; j < Q; ++j)
      if (CX[j] == -CX[i] && CY[j] == -CY[i] && CZ[j] == -CZ[i]) OPP[i] = j;
  tables_ready = true;
}

const float F_FLOOR = 1e-15f;
const float CS2 = float(2.0 / 3.0);

inline float clampf(float v, float lo, float hi) { return v > hi ? hi : (v < lo ? lo : v); }
inline float maxf(float a, float b) { return (a != a || b != b) ? std::numeric_limits<float>::quiet_NaN() : (a < b ? b : a); }
inline float minf(float a, float b) { return (a != a || b != b) ? std::numeric_limits<float>::quiet_NaN() : (a < b ? a : b); }
inline float smooth(float t) { return t * t * (3.0f - 2.0f * t); }

// physics_utils.jl:493-736: the 13 Lagrange multipliers by block-Jacobi Newton sweeps (mass and
// momentum, second moments, energy fluxes), started from the warm start when it passes the gate
void solve_lambdas(float rho, float ux, float uy, float uz, int max_iter, const float* warm, float* la) {
  const float cs2 = CS2;
  const float F_FLOOR_EQ = 1e-15f, OMEGA = 1.5f;
  const float eps = std::numeric_limits<float>::epsilon();
  const float TOL_SQ = 507.0f * eps * eps * rho * rho * 1.0f;
  const float eR = cs2;  // eos_R < 0: cs2
  const float usq = ux * ux + uy * uy + uz * uz;
  const float dT = 1.0f - 1.0f;
  const float dplus2_cs2 = 5.0f * cs2;
  const float ef = usq + 5.0f * eR * dT;
  const float mt[13] = {rho, rho * ux, rho * uy, rho * uz, rho * (ux * ux + eR * dT), rho * (uy * uy + eR * dT),
                        rho * (uz * uz + eR * dT), rho * ux * uy, rho * ux * uz, rho * uy * uz,
                        rho * ux * ef, rho * uy * ef, rho * uz * ef};
  const float inv_cs2 = 1.0f / cs2, inv_cs4 = inv_cs2 * inv_cs2;
  const float pl[13] = {-0.5f * usq * inv_cs2, ux * inv_cs2, uy * inv_cs2, uz * inv_cs2, 0.5f * inv_cs4 * ux * ux,
                        0.5f * inv_cs4 * uy * uy, 0.5f * inv_cs4 * uz * uz, inv_cs4 * ux * uy, inv_cs4 * ux * uz,
                        inv_cs4 * uy * uz, 0.0f, 0.0f, 0.0f};
  const bool use_warm = warm && !(warm[0] != warm[0]);
  for (int i = 0; i < 13; ++i) la[i] = use_warm ? warm[i] : pl[i];
  auto basis = [&](int i, float* b) {  // (cx, cy, cz, a5 .. a13), rho w_i
    const float cxi = float(CX[i]) - 0.0f, cyi = float(CY[i]) - 0.0f, czi = float(CZ[i]) - 0.0f;
    const float csqi = cxi * cxi + cyi * cyi + czi * czi;
    const float efli = csqi - dplus2_cs2;
    b[0] = cxi; b[1] = cyi; b[2] = czi;
    b[3] = cxi * cxi - cs2; b[4] = cyi * cyi - cs2; b[5] = czi * czi - cs2;
    b[6] = cxi * cyi; b[7] = cxi * czi; b[8] = cyi * czi;
    b[9] = cxi * efli; b[10] = cyi * efli; b[11] = czi * efli;
    b[12] = rho * WT[i];
  };
  auto fi_of = [&](const float* b) {
    const float lda = la[0] + la[1] * b[0] + la[2] * b[1] + la[3] * b[2] + la[4] * b[3] + la[5] * b[4] + la[6] * b[5] +
                      la[7] * b[6] + la[8] * b[7] + la[9] * b[8] + la[10] * b[9] + la[11] * b[10] + la[12] * b[11];
    return maxf(b[12] * kbc::exp(clampf(lda, -20.0f, 20.0f)), F_FLOOR_EQ);
  };
  auto step = [&](int m, float d, float j) {
    la[m] += j > F_FLOOR_EQ ? clampf(OMEGA * (mt[m] - d) / j, -2.0f, 2.0f) : 0.0f;
  };
  if (use_warm) {
    const float GATE_FACTOR = 100.0f;
    float gd[13] = {0};
    for (int i = 0; i < Q; ++i) {
      float b[13];
      basis(i, b);
      const float fi = fi_of(b);
      gd[0] += fi;
      for (int m = 1; m < 13; ++m) gd[m] += fi * b[m - 1];
    }
    float gres = 0.0f;
    for (int m = 0; m < 13; ++m) gres += (mt[m] - gd[m]) * (mt[m] - gd[m]);
    if (gres > GATE_FACTOR * TOL_SQ)
      for (int m = 0; m < 13; ++m) la[m] = pl[m];
  }
  for (int sweep = 0; sweep < max_iter; ++sweep) {
    float d[13] = {0}, j[13] = {0};
    for (int i = 0; i < Q; ++i) {
      float b[13];
      basis(i, b);
      const float fi = fi_of(b);
      d[0] += fi; j[0] += fi;
      for (int m = 1; m < 4; ++m) { d[m] += fi * b[m - 1]; j[m] += fi * b[m - 1] * b[m - 1]; }
    }
    for (int m = 0; m < 4; ++m) step(m, d[m], j[m]);
    for (int i = 0; i < Q; ++i) {
      float b[13];
      basis(i, b);
      const float fi = fi_of(b);
      for (int m = 4; m < 10; ++m) { d[m] += fi * b[m - 1]; j[m] += fi * b[m - 1] * b[m - 1]; }
    }
    for (int m = 4; m < 10; ++m) step(m, d[m], j[m]);
    for (int i = 0; i < Q; ++i) {
      float b[13];
      basis(i, b);
      const float fi = fi_of(b);
      for (int m = 10; m < 13; ++m) { d[m] += fi * b[m - 1]; j[m] += fi * b[m - 1] * b[m - 1]; }
    }
    for (int m = 10; m < 13; ++m) step(m, d[m], j[m]);
    float res = 0.0f;
    for (int m = 0; m < 13; ++m) res += (mt[m] - d[m]) * (mt[m] - d[m]);
    if (res < TOL_SQ) break;
  }
}

// physics_utils.jl:738-776: f_eq of one direction (before the mass correction)
float eval_feq(float rho, const float* la, int k) {
  const float cx = float(CX[k]) - 0.0f, cy = float(CY[k]) - 0.0f, cz = float(CZ[k]) - 0.0f;
  const float csq = cx * cx + cy * cy + cz * cz, dplus2 = 5.0f * CS2;
  const float a[13] = {1.0f, cx, cy, cz, cx * cx - CS2, cy * cy - CS2, cz * cz - CS2, cx * cy, cx * cz, cy * cz,
                       cx * (csq - dplus2), cy * (csq - dplus2), cz * (csq - dplus2)};
  float lda = la[0] * a[0];
  for (int m = 1; m < 13; ++m) lda += la[m] * a[m];
  return maxf(rho * WT[k] * kbc::exp(clampf(lda, -20.0f, 20.0f)), 1e-15f);
}

// physics_utils.jl:778-795 and the kernel's f_eq loop (kernel_entropic_d3q39.jl:2365-2385)
void equilibrium(float rho, const float* la, float* feq) {
  float sum = 0.0f;
  for (int k = 0; k < Q; ++k) sum += eval_feq(rho, la, k);
  const float corr = sum > 1e-15f ? rho / sum : 1.0f;
  for (int k = 0; k < Q; ++k) feq[k] = corr * eval_feq(rho, la, k);
}

// physics_utils.jl:280-460 + timestep.jl:1169-1188: the host-side inlet equilibrium at
// (1, u_inlet, -0, -0) with its own sweep (parenthesised basis products), mass correction and floor
void inlet_equilibrium(float u_inlet, float* out) {
  const float cs2 = CS2, rho = 1.0f, ux = u_inlet, uy = -0.0f, uz = -0.0f;
  const float F_FLOOR_EQ = 1e-15f, OMEGA = 1.5f;
  const float eps = std::numeric_limits<float>::epsilon();
  const float TOL_SQ = 507.0f * eps * eps * rho * rho;
  const float eR = cs2, usq = ux * ux + uy * uy + uz * uz, dT = 1.0f - 1.0f, dplus2_cs2 = 5.0f * cs2;
  const float ef = usq + 5.0f * eR * dT;
  const float mt[13] = {rho, rho * ux, rho * uy, rho * uz, rho * (ux * ux + eR * dT), rho * (uy * uy + eR * dT),
                        rho * (uz * uz + eR * dT), rho * ux * uy, rho * ux * uz, rho * uy * uz,
                        rho * ux * ef, rho * uy * ef, rho * uz * ef};
  const float inv_cs2 = 1.0f / cs2, inv_cs4 = inv_cs2 * inv_cs2;
  float la[13] = {-0.5f * usq * inv_cs2, ux * inv_cs2, uy * inv_cs2, uz * inv_cs2, 0.5f * inv_cs4 * ux * ux,
                  0.5f * inv_cs4 * uy * uy, 0.5f * inv_cs4 * uz * uz, inv_cs4 * ux * uy, inv_cs4 * ux * uz,
                  inv_cs4 * uy * uz, 0.0f, 0.0f, 0.0f};
  auto f_of = [&](int i, float* a) {
    const float cx = float(CX[i]) - 0.0f, cy = float(CY[i]) - 0.0f, cz = float(CZ[i]) - 0.0f;
    const float csq = cx * cx + cy * cy + cz * cz, efl = csq - dplus2_cs2;
    a[0] = cx; a[1] = cy; a[2] = cz;
    a[3] = cx * cx - cs2; a[4] = cy * cy - cs2; a[5] = cz * cz - cs2;
    a[6] = cx * cy; a[7] = cx * cz; a[8] = cy * cz;
    a[9] = cx * efl; a[10] = cy * efl; a[11] = cz * efl;
    const float lda = la[0] + la[1] * cx + la[2] * cy + la[3] * cz + la[4] * (cx * cx - cs2) +
                      la[5] * (cy * cy - cs2) + la[6] * (cz * cz - cs2) + la[7] * cx * cy + la[8] * cx * cz +
                      la[9] * cy * cz + la[10] * cx * efl + la[11] * cy * efl + la[12] * cz * efl;
    return maxf(rho * WT[i] * kbc::exp(clampf(lda, -20.0f, 20.0f)), F_FLOOR_EQ);
  };
  const int g0[4] = {0, 4, 10, 13};
  for (int sweep = 0; sweep < 200; ++sweep) {
    float d[13] = {0}, j[13] = {0};
    for (int g = 0; g < 3; ++g) {
      for (int i = 0; i < Q; ++i) {
        float a[12];
        const float fi = f_of(i, a);
        for (int m = g0[g]; m < g0[g + 1]; ++m) {
          if (m == 0) { d[0] += fi; j[0] += fi; } else { d[m] += fi * a[m - 1]; j[m] += fi * a[m - 1] * a[m - 1]; }
        }
      }
      for (int m = g0[g]; m < g0[g + 1]; ++m)
        la[m] += j[m] > F_FLOOR_EQ ? clampf(OMEGA * (mt[m] - d[m]) / j[m], -2.0f, 2.0f) : 0.0f;
    }
    float res = 0.0f;
    for (int m = 0; m < 13; ++m) res += (mt[m] - d[m]) * (mt[m] - d[m]);
    if (res < TOL_SQ) break;
  }
  float fe[Q], sum = 0.0f;
  for (int i = 0; i < Q; ++i) { float a[12]; fe[i] = f_of(i, a); }
  for (int i = 0; i < Q; ++i) sum += fe[i];
  if (sum > 1e-15f) {
    const float corr = rho / sum;
    for (int i = 0; i < Q; ++i) fe[i] *= corr;
  }
  for (int i = 0; i < Q; ++i) out[i] = maxf(fe[i], 1e-10f);
}

inline float safe_log(float x) { return x > 0.0f ? kbc::log(x) : -88.0f; }

// kernel_entropic_d3q39.jl:55-62
float entropy(const float* f) {
  float H = 0.0f;
  for (int k = 0; k < Q; ++k) {
    const float fk = maxf(f[k], F_FLOOR);
    H += fk * safe_log(fk / WT[k]);
  }
  return H;
}

// kernel_entropic_d3q39.jl:64-83 (s and h given per direction)
float entropy_at_alpha(const float* feq, const float* s, const float* h, float beta, float alpha) {
  const float coeff_s = 1.0f - 2.0f * beta, coeff_h = 1.0f - 2.0f * beta * alpha;
  float H = 0.0f;
  for (int k = 0; k < Q; ++k) {
    float fk = feq[k] + coeff_s * s[k] + coeff_h * h[k];
    fk = maxf(fk, F_FLOOR);
    H += fk * safe_log(fk / WT[k]);
  }
  return H;
}

// kernel_entropic_d3q39.jl:217-238
void entropy_and_deriv(const float* feq, const float* s, const float* h, float beta, float alpha, float& H, float& dH) {
  const float coeff_s = 1.0f - 2.0f * beta, coeff_h = 1.0f - 2.0f * beta * alpha;
  H = 0.0f; dH = 0.0f;
  for (int k = 0; k < Q; ++k) {
    float fk = feq[k] + coeff_s * s[k] + coeff_h * h[k];
    fk = maxf(fk, F_FLOOR);
    const float lr = safe_log(fk / WT[k]);
    H += fk * lr;
    dH += (-2.0f * beta * h[k]) * (1.0f + lr);
  }
}

// kernel_entropic_d3q39.jl:240-284
float alpha_bisection(const float* feq, const float* s, const float* h, float beta, float H_pre, int max_iter) {
  const float inv_2beta = 0.5f / maxf(beta, 0.01f);
  float lo = maxf(inv_2beta - 0.1f, 0.1f), hi = maxf(inv_2beta + 3.0f, 4.0f);
  float H_lo = entropy_at_alpha(feq, s, h, beta, lo);
  const float H_hi = entropy_at_alpha(feq, s, h, beta, hi);
  if (!((H_lo - H_pre) * (H_hi - H_pre) < 0.0f)) return inv_2beta;
  for (int it = 0; it < max_iter; ++it) {
    const float mid = 0.5f * (lo + hi);
    const float H_mid = entropy_at_alpha(feq, s, h, beta, mid);
    if ((H_mid - H_pre) * (H_lo - H_pre) > 0.0f) { lo = mid; H_lo = H_mid; } else { hi = mid; }
    if ((hi - lo) < 0.005f * (inv_2beta + 1e-6f)) break;
  }
  return 0.5f * (lo + hi);
}

// kernel_entropic_d3q39.jl:286-321
float alpha_newton(const float* feq, const float* s, const float* h, float beta, float H_pre, int max_iter, float tol) {
  float alpha = 2.0f;
  const float inv_2beta = 0.5f / maxf(beta, 0.01f);
  for (int it = 0; it < max_iter; ++it) {
    float H, dH;
    entropy_and_deriv(feq, s, h, beta, alpha, H, dH);
    const float residual = H - H_pre;
    if (std::fabs(residual) < tol) break;
    if (std::fabs(dH) < 1e-12f) break;
    const float delta = residual / dH;
    alpha -= delta;
    alpha = clampf(alpha, maxf(inv_2beta - 0.1f, 0.1f), 6.0f);
    if (std::fabs(delta) < 1e-5f) break;
  }
  if (!(alpha > 0.0f)) alpha = inv_2beta;
  return alpha;
}

// kernel_entropic_d3q39.jl:323-345
float alpha_approximate(const float* feq, const float* h, float beta) {
  float hn = 0.0f, fn = 0.0f;
  for (int k = 0; k < Q; ++k) { hn += h[k] * h[k]; fn += feq[k] * feq[k]; }
  const float ratio = hn / maxf(fn, 1e-15f);
  const float inv_2beta = 0.5f / maxf(beta, 0.01f);
  return clampf(2.0f - 0.5f * ratio, inv_2beta, 4.0f);
}

// kernel_entropic_d3q39.jl:347-415
float alpha_taylor(const float* feq, const float* s, const float* h, float beta, float H_pre, int max_iter) {
  float dev = 0.0f;
  for (int k = 0; k < Q; ++k) {
    const float fneq = s[k] + h[k];
    const float fk = maxf(feq[k] + fneq, F_FLOOR);
    const float t = std::fabs(fneq) / fk;
    dev = maxf(dev, t);
    if (dev > 0.01f) break;
  }
  const float inv_2beta = 0.5f / maxf(beta, 0.01f);
  if (dev < 1e-6f) return 2.0f;
  if (dev < 0.01f) {
    float a1 = 0.0f, a2 = 0.0f, a3 = 0.0f, a4 = 0.0f;
    for (int k = 0; k < Q; ++k) {
      const float t = s[k] + h[k];
      const float fk = maxf(feq[k] + t, F_FLOOR);
      const float inv = 1.0f / fk;
      float p = t * t * inv; a1 += p;
      p *= t * inv; a2 += p;
      p *= t * inv; a3 += p;
      p *= t * inv; a4 += p;
    }
    a1 *= 0.5f; a2 *= -1.0f / 6.0f; a3 *= 1.0f / 12.0f; a4 *= -0.05f;
    if (std::fabs(a1) > 1e-20f) {
      const float i1 = 1.0f / a1;
      const float alpha = 2.0f - 4.0f * a2 * i1 + 16.0f * a2 * a2 * i1 * i1 - 8.0f * a3 * i1 +
                          80.0f * a2 * a3 * i1 * i1 - 80.0f * a2 * a2 * a2 * i1 * i1 * i1 - 16.0f * a4 * i1;
      return clampf(alpha, inv_2beta, 6.0f);
    }
    return 2.0f;
  }
  return alpha_bisection(feq, s, h, beta, H_pre, max_iter);
}

struct CellOut {
  float rho, u[3];
};

// The step's input populations around one cell, for the SVV taps: fin (8,8,8,nb,39), nbr (nb,27)
// 1-based with 0 for a missing block, obstacle (8,8,8,nb) or null.
struct SvvTaps {
  const float* fin;
  int64_t N;
  const int32_t* nbr;
  const uint8_t* obst;
  int nb, b, x, y, z;
  float eps_x, eps_yz;
  // population k of (x, y, z) + d (one axis); the cell's own input population past a missing block
  // or in a solid cell (get_pop_neighbor_yz / _x, kernel_svv_yz_d3q39.jl:78-116, 225-250)
  float tap(int dx, int dy, int dz, int k) const {
    const int64_t own = x + 8 * y + 64 * z + 512 * (int64_t)b;
    const int nx = x + dx, ny = y + dy, nz = z + dz;
    const int ox = nx < 0 ? -1 : (nx > 7 ? 1 : 0), oy = ny < 0 ? -1 : (ny > 7 ? 1 : 0), oz = nz < 0 ? -1 : (nz > 7 ? 1 : 0);
    const int bo = (ox | oy | oz) == 0 ? b : nbr[b + (int64_t)nb * ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))] - 1;
    if (bo < 0) return fin[own + N * k];
    const int64_t c = (nx - 8 * ox) + 8 * (ny - 8 * oy) + 64 * (nz - 8 * oz) + 512 * (int64_t)bo;
    if (obst && obst[c]) return fin[own + N * k];
    return fin[c + N * k];
  }
};

// apply_svv_yz_d3q39_inline! (axis 1) and apply_svv_x_d3q39_inline! (axis 0), frame shift 0:
// the bi-Laplacian of the input populations about the post-collision f_k, then the 4-moment
// correction that restores the cell's mass and momentum.
void svv_axis(const SvvTaps& t, int yz, float eps, float* fp) {
  float d_rho = 0.0f, d_jx = 0.0f, d_jy = 0.0f, d_jz = 0.0f;
  for (int k = 0; k < Q; ++k) {
    const float fc = fp[k];
    float ff;
    if (yz) {
      const float by = t.tap(0, -2, 0, k) - 4.0f * t.tap(0, -1, 0, k) + 6.0f * fc - 4.0f * t.tap(0, 1, 0, k) + t.tap(0, 2, 0, k);
      const float bz = t.tap(0, 0, -2, k) - 4.0f * t.tap(0, 0, -1, k) + 6.0f * fc - 4.0f * t.tap(0, 0, 1, k) + t.tap(0, 0, 2, k);
      ff = fc - eps * (by + bz);
    } else {
      const float bx = t.tap(-2, 0, 0, k) - 4.0f * t.tap(-1, 0, 0, k) + 6.0f * fc - 4.0f * t.tap(1, 0, 0, k) + t.tap(2, 0, 0, k);
      ff = fc - eps * bx;
    }
    const float diff = ff - fc;
    d_rho += diff;
    d_jx += diff * (float(CX[k]) - 0.0f);
    d_jy += diff * (float(CY[k]) - 0.0f);
    d_jz += diff * (float(CZ[k]) - 0.0f);
    fp[k] = ff;
  }
  const float inv_cs2 = 1.0f / CS2;
  for (int k = 0; k < Q; ++k) {
    const float cx = float(CX[k]) - 0.0f, cy = float(CY[k]) - 0.0f, cz = float(CZ[k]) - 0.0f;
    const float cu = cx * d_jx + cy * d_jy + cz * d_jz;
    fp[k] -= WT[k] * (d_rho + inv_cs2 * cu);
  }
}

// One cell of the step after the pull: f (39, pulled), g (d u_a / d x_b, 9, previous velocity),
// lam (13, warm start in, solution out), f_eq_inlet (39) -> fout (39), rho and u for the level's
// macro arrays.
void collide_cell(float* f, const float* g, const oal_step_params& P, const float* f_eq_inlet, float* lam,
                  float* fout, CellOut& out, float sp = 0.0f, float wd = std::numeric_limits<float>::quiet_NaN(),
                  const SvvTaps* svv = nullptr) {
  // moments of the pulled populations (kernel_entropic_d3q39.jl:1281-1287)
  float rho = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
  for (int k = 0; k < Q; ++k) {
    rho += f[k];
    jx += f[k] * float(CX[k]);
    jy += f[k] * float(CY[k]);
    jz += f[k] * float(CZ[k]);
  }
  // STEP 2 (:1616-1650)
  const float rho_raw = rho;
  rho = maxf(rho_raw, 0.01f);
  float inv_rho = 1.0f / rho;
  float ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  const bool is_nan = !(rho_raw == rho_raw) || !(ux == ux) || !(uy == uy) || !(uz == uz);
  if (is_nan || rho_raw < 0.01f) {
    rho = 1.0f; ux = P.u_inlet; uy = 0.0f; uz = 0.0f; inv_rho = 1.0f;
    for (int k = 0; k < Q; ++k) f[k] = f_eq_inlet[k];
  }
  // sponge (:1662, 1787-1841; athermal, pre-collision form)
  if (sp > 0.0f) {
    rho = rho * (1.0f - sp) + 1.0f * sp;
    ux = ux * (1.0f - sp) + P.u_inlet * sp;
    uy = uy * (1.0f - sp);
    uz = uz * (1.0f - sp);
    if (P.sponge_blend_distributions == 1) {
      for (int k = 0; k < Q; ++k) f[k] = f[k] * (1.0f - sp) + f_eq_inlet[k] * sp;
      rho = 0.0f;
      float sjx = 0.0f, sjy = 0.0f, sjz = 0.0f;
      for (int k = 0; k < Q; ++k) {
        rho += f[k];
        sjx += f[k] * float(CX[k]);
        sjy += f[k] * float(CY[k]);
        sjz += f[k] * float(CZ[k]);
      }
      rho = maxf(rho, 0.01f);
      inv_rho = 1.0f / rho;
      ux = sjx * inv_rho; uy = sjy * inv_rho; uz = sjz * inv_rho;
    }
  }
  // macro realizability (:2112-2229): far-bulk bounds away from walls and sponges, near-wall ones
  // (MacroBoundsPack defaults 0.35 / 2.40) elsewhere
  const bool far_bulk = (wd != wd || wd > 16.0f) && sp < 0.03f;
  bool macro_limited = false;
  {
    const float u_trans = std::sqrt(uy * uy + uz * uz);
    const float uxr = ux - 0.0f;
    float uyr = uy - 0.0f, uzr = uz - 0.0f;
    float u_rel = std::sqrt(uxr * uxr + uyr * uyr + uzr * uzr);
    const float u_ref = maxf(maxf(P.u_inlet, 0.1f), 0.1f);
    float u_cap = minf(1.00f, maxf(0.80f, 1.35f * u_ref + 0.15f));
    float u_trans_cap = minf(0.92f, maxf(0.55f, 1.15f * u_ref + 0.12f));
    if (far_bulk) {
      u_cap = minf(u_cap, minf(0.78f, maxf(0.48f, 1.12f * u_ref + 0.08f)));
      u_trans_cap = minf(u_trans_cap, minf(0.46f, maxf(0.18f, 0.68f * u_ref + 0.04f)));
    }
    const bool speed_path = u_rel > u_cap;
    const bool trans_path = u_trans > u_trans_cap;
    const float rho_floor = far_bulk ? 0.42f : 0.35f, rho_ceil = far_bulk ? 2.10f : 2.40f;  // MacroBoundsPack defaults
    const bool density_path = rho < 0.30f || rho > 2.80f || (far_bulk && (rho < rho_floor || rho > rho_ceil)) ||
                              ((rho < 0.45f || rho > 2.20f) && (speed_path || trans_path));
    if (density_path) {
      rho = clampf(rho, rho_floor, rho_ceil);
      inv_rho = 1.0f / maxf(rho, 0.01f);
      macro_limited = true;
    }
    if (trans_path && u_trans > 1e-8f) {
      const float ts = u_trans_cap / maxf(u_trans, 1e-8f);
      uy *= ts;
      uz *= ts;
      uyr = uy - 0.0f; uzr = uz - 0.0f;
      u_rel = std::sqrt(uxr * uxr + uyr * uyr + uzr * uzr);
      macro_limited = true;
    }
    if (speed_path && u_rel > 1e-8f) {
      const float ss = u_cap / maxf(u_rel, 1e-8f);
      ux = 0.0f + uxr * ss;
      uy = 0.0f + uyr * ss;
      uz = 0.0f + uzr * ss;
      macro_limited = true;
    }
  }
  // equilibrium velocity (no wall force, no frame shift) and its cap (:2262-2282)
  float ux_rel = (ux + 0.5f * 0.0f * inv_rho) - 0.0f;
  float uy_rel = (uy + 0.5f * 0.0f * inv_rho) - 0.0f;
  float uz_rel = (uz + 0.5f * 0.0f * inv_rho) - 0.0f;
  bool eq_limited = false;
  {
    const float m = std::sqrt(ux_rel * ux_rel + uy_rel * uy_rel + uz_rel * uz_rel);
    if (m > 0.82f) {
      const float sc = 0.82f / maxf(m, 1e-6f);
      ux_rel *= sc; uy_rel *= sc; uz_rel *= sc;
      eq_limited = true;
    }
  }
  out.rho = rho; out.u[0] = ux; out.u[1] = uy; out.u[2] = uz;
  // STEP 3a: f_eq from the warm-started 13-moment solve (:2330-2385)
  float la[13];
  solve_lambdas(rho, ux_rel, uy_rel, uz_rel, 200, lam, la);
  for (int m = 0; m < 13; ++m) lam[m] = la[m];
  float feq[Q];
  equilibrium(rho, la, feq);
  // STEP 3: WALE (:2588-2700)
  const float g11 = g[0], g12 = g[1], g13 = g[2], g21 = g[3], g22 = g[4], g23 = g[5], g31 = g[6], g32 = g[7], g33 = g[8];
  const float q11 = g11 * g11 + g12 * g21 + g13 * g31, q12 = g11 * g12 + g12 * g22 + g13 * g32, q13 = g11 * g13 + g12 * g23 + g13 * g33;
  const float q21 = g21 * g11 + g22 * g21 + g23 * g31, q22 = g21 * g12 + g22 * g22 + g23 * g32, q23 = g21 * g13 + g22 * g23 + g23 * g33;
  const float q31 = g31 * g11 + g32 * g21 + g33 * g31, q32 = g31 * g12 + g32 * g22 + g33 * g32, q33 = g31 * g13 + g32 * g23 + g33 * g33;
  const float tr = (q11 + q22 + q33) / 3.0f;
  const float Sd11 = q11 - tr, Sd22 = q22 - tr, Sd33 = q33 - tr;
  const float Sd12 = 0.5f * (q12 + q21), Sd13 = 0.5f * (q13 + q31), Sd23 = 0.5f * (q23 + q32);
  const float S12 = 0.5f * (g12 + g21), S13 = 0.5f * (g13 + g31), S23 = 0.5f * (g23 + g32);
  const float OP1 = Sd11 * Sd11 + Sd22 * Sd22 + Sd33 * Sd33 + 2.0f * (Sd12 * Sd12 + Sd13 * Sd13 + Sd23 * Sd23);
  const float OP2 = g11 * g11 + g22 * g22 + g33 * g33 + 2.0f * (S12 * S12 + S13 * S13 + S23 * S23);
  const float bg = P.nu_sgs_background * P.amr_sgs_scale;
  float nu_eddy = 0.0f;
  if (OP1 > 1e-12f) {
    const float OP1_32 = OP1 * std::sqrt(OP1);
    const float OP2_52 = OP2 * OP2 * std::sqrt(maxf(OP2, 1e-12f));
    const float denom = OP2_52 + OP1 * std::sqrt(std::sqrt(maxf(OP1, 1e-12f)));
    if (denom > 1e-12f) nu_eddy = (P.c_wale * P.c_wale) * OP1_32 / denom;
  }
  nu_eddy = maxf(nu_eddy, bg);
  // Mach-pocket viscosity (:2777-2806), shock sensor off
  const float shock_boost = 0.0f;
  float pocket = 0.0f;
  {
    const float T_local = 1.0f;
    const float cs_local = std::sqrt(maxf(CS2 * maxf(T_local, 0.2f), 1e-6f));
    const float inv_cs = 1.0f / cs_local;
    const float u_mag = std::sqrt(ux * ux + uy * uy + uz * uz);
    const float u_perp = std::sqrt(uy * uy + uz * uz);
    const float mach_boost = smooth(clampf((u_mag * inv_cs - 0.50f) / 0.25f, 0.0f, 1.0f));
    const float perp_boost = smooth(clampf((u_perp * inv_cs - 0.32f) / 0.25f, 0.0f, 1.0f));
    const float rho_lo = smooth(clampf((0.90f - rho) / 0.26f, 0.0f, 1.0f));
    const float rho_hi = smooth(clampf((rho - 1.30f) / 0.70f, 0.0f, 1.0f));
    const float rho_split = maxf(rho_lo, rho_hi);
    const float transverse_only = perp_boost * mach_boost;
    pocket = maxf(maxf(perp_boost * maxf(rho_split, shock_boost), mach_boost * rho_split),
                  maxf(shock_boost * mach_boost, transverse_only));
    if (pocket > 0.0f) {
      const float pocket_nu_max = maxf(5.00f * P.shock_nu_max, 0.24f);
      nu_eddy = maxf(nu_eddy, pocket * pocket_nu_max * P.amr_sgs_scale);
    }
  }
  nu_eddy = maxf(nu_eddy, P.nu_sgs_lattice_floor);
  const float nu_mol = (P.tau - 0.5f) * CS2;
  const float nu_eff = nu_mol + nu_eddy;
  const float tau_eff = 0.5f + nu_eff / CS2;
  const float omega = 1.0f / maxf(tau_eff, 0.500001f);
  const float beta = 0.5f * omega;
  // STEP 4b: positivity of the arriving populations (:2885-2906)
  bool any_negative = false;
  for (int k = 0; k < Q; ++k) if (f[k] < F_FLOOR) any_negative = true;
  if (any_negative) {
    float worst = 1.0f;
    for (int k = 0; k < Q; ++k) {
      const float fneq = f[k] - feq[k];
      if (fneq < 0.0f && feq[k] > F_FLOOR) worst = minf(worst, (feq[k] - F_FLOOR) / (-fneq + F_FLOOR));
    }
    worst = clampf(worst, 0.0f, 1.0f);
    for (int k = 0; k < Q; ++k) {
      f[k] = feq[k] + worst * (f[k] - feq[k]);
      f[k] = maxf(f[k], F_FLOOR);
    }
  }
  // realizability guard (:2907-2958), Knudsen epsilon off
  float guard;
  {
    const float knudsen_eps = 0.0f;
    const float u_g = std::sqrt(ux * ux + uy * uy + uz * uz);
    const float cs_g = std::sqrt(maxf(CS2 * maxf(1.0f, 0.2f), 1e-6f));
    const float mach_g = u_g / cs_g;
    const float trans_g = std::sqrt(uy * uy + uz * uz);
    const float mach_trans_g = trans_g / cs_g;
    const float mach_gb = smooth(clampf((mach_g - 0.62f) / 0.22f, 0.0f, 1.0f));
    const float trans_gb = smooth(clampf((mach_trans_g - 0.38f) / 0.22f, 0.0f, 1.0f));
    const float rho_low_g = clampf((0.88f - rho) / 0.28f, 0.0f, 1.0f);
    const float rho_high_g = clampf((rho - 1.35f) / 0.65f, 0.0f, 1.0f);
    const float u_ref_g = maxf(maxf(P.u_inlet, 0.1f), 0.54f);
    const float u_spike = maxf(clampf((u_g - u_ref_g) / 0.24f, 0.0f, 1.0f), 0.85f * maxf(mach_gb, trans_gb));
    const float neq_g = clampf((knudsen_eps - 0.12f) / 0.35f, 0.0f, 1.0f);
    const float pocket_neq = maxf(maxf(shock_boost, neq_g), maxf(mach_gb, trans_gb));
    guard = maxf(maxf(shock_boost * maxf(neq_g, mach_gb), rho_low_g * pocket_neq), maxf(rho_high_g, u_spike * pocket_neq));
    guard = maxf(guard, pocket);
    if (eq_limited || macro_limited) guard = maxf(guard, 1.0f);
    if (guard > 0.0f) {
      float reps = knudsen_eps;
      if (reps <= 1e-6f) {
        float sdf = 0.0f, sfe = 0.0f;
        for (int k = 0; k < Q; ++k) { sdf += std::fabs(f[k] - feq[k]); sfe += std::fabs(feq[k]); }
        reps = sfe > 1e-10f ? sdf / sfe : 0.0f;
      }
      const float cap = maxf(0.025f, 0.18f - 0.155f * guard);
      if (reps > cap) {
        const float th = clampf(cap / maxf(reps, 1e-12f), 0.0f, 1.0f);
        for (int k = 0; k < Q; ++k) {
          f[k] = feq[k] + th * (f[k] - feq[k]);
          f[k] = maxf(f[k], F_FLOOR);
        }
      }
    }
  }
  // STEP 5: mirror split, HRR blend of s, sigma damping of h (:2962-3095)
  float s[Q], h[Q];
  for (int k = 0; k < Q; ++k) {
    const int kb = OPP[k];
    const float df = f[k] - feq[k], dfb = f[kb] - feq[kb];
    s[k] = 0.5f * (df + dfb);
    h[k] = 0.5f * (df - dfb);
  }
  if (P.hrr_hybrid == 1 && P.hrr_sigma < 0.999f) {
    const float tmh = maxf(tau_eff - 0.5f, 0.0f);
    const float c = -2.0f * rho * CS2 * tmh;
    const float pxx = c * g11, pyy = c * g22, pzz = c * g33, pxy = c * S12, pxz = c * S13, pyz = c * S23;
    const float inv_2cs4 = 0.5f / (CS2 * CS2);
    const float oms = 1.0f - P.hrr_sigma;
    for (int k = 0; k < Q; ++k) {
      const float cx = float(CX[k]) - 0.0f, cy = float(CY[k]) - 0.0f, cz = float(CZ[k]) - 0.0f;
      const float Qxx = cx * cx - CS2, Qyy = cy * cy - CS2, Qzz = cz * cz - CS2;
      const float Qxy = cx * cy, Qxz = cx * cz, Qyz = cy * cz;
      const float contraction = Qxx * pxx + Qyy * pyy + Qzz * pzz + 2.0f * (Qxy * pxy + Qxz * pxz + Qyz * pyz);
      const float s_fd = WT[k] * contraction * inv_2cs4;
      s[k] = P.hrr_sigma * s[k] + oms * s_fd;
    }
  }
  float sigma = P.lambda_param;
  if (pocket > 0.0f) sigma = maxf(sigma, minf(0.995f, 0.80f + 0.195f * pocket));
  const float h_scale = sigma > 0.0f ? 1.0f - sigma : 1.0f;
  if (sigma > 0.0f)
    for (int k = 0; k < Q; ++k) h[k] *= h_scale;
  float h_norm_sq = 0.0f;
  for (int k = 0; k < Q; ++k) h_norm_sq += h[k] * h[k];
  // STEP 6: alpha (:3109-3150)
  const float inv_2beta = 0.5f / maxf(beta, 0.01f);
  float alpha = 2.0f;
  if (h_norm_sq > 1e-20f) {
    const float H_pre = entropy(f);
    switch (P.adaptive_omega4) {
      case 1: alpha = alpha_newton(feq, s, h, beta, H_pre, 8, 1e-5f); break;
      case 2: alpha = alpha_approximate(feq, h, beta); break;
      case 3: alpha = alpha_taylor(feq, s, h, beta, H_pre, 10); break;
      default: alpha = alpha_bisection(feq, s, h, beta, H_pre, 10); break;
    }
    if (!(alpha > 0.0f)) alpha = inv_2beta;
    alpha = clampf(alpha, inv_2beta, 6.0f);
  }
  // STEP 7-8: KBC, zero force, post-collision blend and guard, output (:3153-3368)
  const float coeff_s = 1.0f - 2.0f * beta, coeff_h = 1.0f - 2.0f * beta * alpha;
  const float inv_cs2 = 1.0f / CS2;
  float fp[Q];
  float fmin = 1.0f;
  for (int k = 0; k < Q; ++k) {
    const float cx = float(CX[k]) - 0.0f, cy = float(CY[k]) - 0.0f, cz = float(CZ[k]) - 0.0f;
    const float fc = feq[k] + coeff_s * s[k] + coeff_h * h[k];
    const float cu = cx * ux_rel + cy * uy_rel + cz * uz_rel;
    const float force_term = WT[k] * inv_cs2 *
                             ((cx - ux_rel + inv_cs2 * cu * cx) * 0.0f + (cy - uy_rel + inv_cs2 * cu * cy) * 0.0f +
                              (cz - uz_rel + inv_cs2 * cu * cz) * 0.0f);
    fp[k] = fc + (1.0f - 0.5f * omega) * force_term;
    fmin = minf(fmin, fp[k]);
  }
  if (fmin < 0.0f) {
    float blend = 1.0f;
    for (int k = 0; k < Q; ++k) {
      const float fneq = fp[k] - feq[k];
      if (fneq < 0.0f && feq[k] > F_FLOOR) blend = minf(blend, feq[k] / (feq[k] - fneq + F_FLOOR));
    }
    blend = maxf(blend, 0.0f);
    for (int k = 0; k < Q; ++k) fp[k] = feq[k] + blend * (fp[k] - feq[k]);
  }
  if (guard > 0.0f) {
    float sdf = 0.0f, sfe = 0.0f;
    for (int k = 0; k < Q; ++k) { sdf += std::fabs(fp[k] - feq[k]); sfe += std::fabs(feq[k]); }
    const float ep = sfe > 1e-10f ? sdf / sfe : 0.0f;
    const float cap = maxf(0.025f, 0.22f - 0.195f * guard);
    if (ep > cap) {
      const float th = clampf(cap / maxf(ep, 1e-12f), 0.0f, 1.0f);
      for (int k = 0; k < Q; ++k) {
        fp[k] = feq[k] + th * (fp[k] - feq[k]);
        fp[k] = maxf(fp[k], F_FLOOR);
      }
    }
  }
  if (svv && (svv->eps_yz > 0.0f || svv->eps_x > 0.0f)) {
    if (svv->eps_yz > 0.0f) svv_axis(*svv, 1, svv->eps_yz, fp);
    if (svv->eps_x > 0.0f) svv_axis(*svv, 0, svv->eps_x, fp);
    // positivity re-enforcement after the add-on (:3296-3318)
    float fmin_post = fp[0];
    for (int k = 1; k < Q; ++k) fmin_post = minf(fmin_post, fp[k]);
    if (fmin_post < 0.0f) {
      float blend = 1.0f;
      for (int k = 0; k < Q; ++k) {
        const float fneq = fp[k] - feq[k];
        if (fneq < 0.0f && feq[k] > F_FLOOR) blend = minf(blend, feq[k] / (feq[k] - fneq + F_FLOOR));
      }
      blend = maxf(blend, 0.0f);
      for (int k = 0; k < Q; ++k) fp[k] = feq[k] + blend * (fp[k] - feq[k]);
    }
  }
  for (int k = 0; k < Q; ++k) {
    float fc = fp[k];
    if (!(fc == fc) || fc > 1e3f) fc = feq[k];
    fout[k] = fc;
  }
}

// central differences of the previous step's velocity, g[3a+b] = d u_a / d x_b
// (physics_utils.jl:2217-2233), every neighbour block present
void velocity_gradient(int b, int x, int y, int z, int nb, const int32_t* nbr, const float* vel, int64_t N, float* g) {
  float ue[3][2][3];
  for (int ax = 0; ax < 3; ++ax)
    for (int s = 0; s < 2; ++s) {
      int p[3] = {x, y, z};
      p[ax] += s == 0 ? 1 : -1;
      const int ox = p[0] < 0 ? -1 : (p[0] > 7 ? 1 : 0), oy = p[1] < 0 ? -1 : (p[1] > 7 ? 1 : 0),
                oz = p[2] < 0 ? -1 : (p[2] > 7 ? 1 : 0);
      const int bo = nbr[b + (int64_t)nb * ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))] - 1;
      const int64_t c = (p[0] - 8 * ox) + 8 * (p[1] - 8 * oy) + 64 * (p[2] - 8 * oz) + 512 * (int64_t)bo;
      for (int a = 0; a < 3; ++a) ue[ax][s][a] = vel[c + N * a];
    }
  for (int a = 0; a < 3; ++a)
    for (int bb = 0; bb < 3; ++bb) g[3 * a + bb] = 0.5f * (ue[bb][0][a] - ue[bb][1][a]);
}

// the same with the level's faces and obstacles: a missing neighbour block or a solid neighbour
// cell contributes the own velocity (get_velocity_neighbor_fluid, physics_utils.jl:1981-2035)
void velocity_gradient_ex(int b, int x, int y, int z, int nb, const int32_t* nbr, const uint8_t* obst,
                          const float* vel, int64_t N, float* g) {
  const int64_t own = x + 8 * y + 64 * z + 512 * (int64_t)b;
  float ue[3][2][3];
  for (int ax = 0; ax < 3; ++ax)
    for (int s = 0; s < 2; ++s) {
      int p[3] = {x, y, z};
      p[ax] += s == 0 ? 1 : -1;
      const int ox = p[0] < 0 ? -1 : (p[0] > 7 ? 1 : 0), oy = p[1] < 0 ? -1 : (p[1] > 7 ? 1 : 0),
                oz = p[2] < 0 ? -1 : (p[2] > 7 ? 1 : 0);
      const int bo = (ox | oy | oz) == 0 ? b : nbr[b + (int64_t)nb * ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))] - 1;
      int64_t c = own;
      if (bo >= 0) {
        const int64_t cn = (p[0] - 8 * ox) + 8 * (p[1] - 8 * oy) + 64 * (p[2] - 8 * oz) + 512 * (int64_t)bo;
        if (!(obst && obst[cn])) c = cn;
      }
      for (int a = 0; a < 3; ++a) ue[ax][s][a] = vel[c + N * a];
    }
  for (int a = 0; a < 3; ++a)
    for (int bb = 0; bb < 3; ++bb) g[3 * a + bb] = 0.5f * (ue[bb][0][a] - ue[bb][1][a]);
}

}  // namespace

extern "C" {

void ora_q39_tables(int32_t* cx, int32_t* cy, int32_t* cz, float* w, int32_t* opp) {
  build_tables();
  for (int i = 0; i < Q; ++i) { cx[i] = CX[i]; cy[i] = CY[i]; cz[i] = CZ[i]; w[i] = WT[i]; opp[i] = OPP[i]; }
}

void ora_q39_exp(int64_t n, const float* x, float* y) { for (int64_t i = 0; i < n; ++i) y[i] = kbc::exp(x[i]); }
void ora_q39_log(int64_t n, const float* x, float* y) { for (int64_t i = 0; i < n; ++i) y[i] = kbc::log(x[i]); }

// Equilibrium of n cells from the polynomial start: rho (n), u (n,3) -> feq (n,39), lambdas (n,13)
void ora_q39_equilibrium(int64_t n, const float* rho, const float* u, float* feq, float* lam) {
  build_tables();
  for (int64_t c = 0; c < n; ++c) {
    float la[13];
    solve_lambdas(rho[c], u[3 * c], u[3 * c + 1], u[3 * c + 2], 200, nullptr, la);
    equilibrium(rho[c], la, feq + 39 * c);
    if (lam) for (int m = 0; m < 13; ++m) lam[13 * c + m] = la[m];
  }
}

void ora_q39_inlet_equilibrium(float u_inlet, float* out39) {
  build_tables();
  inlet_equilibrium(u_inlet, out39);
}

// Collision of n independent cells: f (n,39) pulled populations, g (n,9) velocity gradients,
// lam (n,13) warm start in / solution out -> fout (n,39), rho (n), u (n,3)
void ora_q39_collide_cells(int64_t n, const oal_step_params* P, const float* f, const float* g, float* lam,
                           float* fout, float* rho, float* u) {
  build_tables();
  float fin[Q];
  inlet_equilibrium(P->u_inlet, fin);
  for (int64_t c = 0; c < n; ++c) {
    float fc[Q];
    for (int k = 0; k < Q; ++k) fc[k] = f[39 * c + k];
    CellOut o;
    collide_cell(fc, g + 9 * c, *P, fin, lam + 13 * c, fout + 39 * c, o);
    rho[c] = o.rho;
    for (int a = 0; a < 3; ++a) u[3 * c + a] = o.u[a];
  }
}

// One step of a level in the reference layout: f (8,8,8,nb,39), rho (8,8,8,nb), vel (8,8,8,nb,3),
// lambda cache (8,8,8,nb,13); nbr (nb,27) 1-based with every entry present.
void ora_q39_step(int32_t nb, const int32_t* nbr, const oal_step_params* P, const float* fin, float* fout,
                  const float* vel_in, float* vel_out, float* rho_out, float* lam) {
  build_tables();
  const int64_t N = (int64_t)nb * 512;
  float f_eq_inlet[Q];
  inlet_equilibrium(P->u_inlet, f_eq_inlet);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b)
    for (int cell = 0; cell < 512; ++cell) {
      const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
      float f[Q];
      for (int k = 0; k < Q; ++k) {
        const int sx = x - CX[k], sy = y - CY[k], sz = z - CZ[k];
        const int ox = sx < 0 ? -1 : (sx > 7 ? 1 : 0), oy = sy < 0 ? -1 : (sy > 7 ? 1 : 0), oz = sz < 0 ? -1 : (sz > 7 ? 1 : 0);
        const int bo = (ox | oy | oz) == 0 ? b : nbr[b + (int64_t)nb * ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))] - 1;
        f[k] = fin[(sx - 8 * ox) + 8 * (sy - 8 * oy) + 64 * (sz - 8 * oz) + 512 * (int64_t)bo + N * k];
      }
      float g[9];
      velocity_gradient(b, x, y, z, nb, nbr, vel_in, N, g);
      const int64_t ci = cell + 512 * (int64_t)b;
      float la[13];
      for (int m = 0; m < 13; ++m) la[m] = lam[ci + N * m];
      float fo[Q];
      CellOut o;
      const SvvTaps taps{fin, N, nbr, nullptr, nb, b, x, y, z, P->svv_x_epsilon, P->svv_yz_epsilon};
      collide_cell(f, g, *P, f_eq_inlet, la, fo, o, 0.0f, std::numeric_limits<float>::quiet_NaN(), &taps);
      for (int m = 0; m < 13; ++m) lam[ci + N * m] = la[m];
      for (int k = 0; k < Q; ++k) fout[ci + N * k] = fo[k];
      rho_out[ci] = o.rho;
      for (int a = 0; a < 3; ++a) vel_out[ci + N * a] = o.u[a];
    }
}

// One step of a level with domain faces and obstacle cells, reference layout as ora_q39_step;
// nbr (nb,27) 1-based with 0 for a missing neighbour block, coords (nb,3) 1-based block
// coordinates, domain nx x ny x nz cells, obstacle (8,8,8,nb) uint8 or null.
void ora_q39_step_ex(int32_t nb, const int32_t* nbr, const int32_t* coords, int32_t nx, int32_t ny, int32_t nz,
                     const uint8_t* obstacle, const float* sponge, const float* wall_dist, const oal_step_params* P,
                     const float* fin, float* fout, const float* vel_in, float* vel_out, float* rho_out, float* lam) {
  build_tables();
  const int64_t N = (int64_t)nb * 512;
  float f_eq_inlet[Q];
  inlet_equilibrium(P->u_inlet, f_eq_inlet);
  // moments of the inlet equilibrium, the target of the inlet-face pin (:1315-1326)
  float trho = 0.0f, tjx = 0.0f, tjy = 0.0f, tjz = 0.0f;
  for (int k = 0; k < Q; ++k) {
    const float fe = f_eq_inlet[k];
    trho += fe;
    tjx += fe * float(CX[k]);
    tjy += fe * float(CY[k]);
    tjz += fe * float(CZ[k]);
  }
  kbc::FaceParams F{nx, ny, nz, P->ymin_wall_bc, P->transverse_freestream, P->time_step_seed,
                    P->transverse_freestream_blend, P->inlet_turbulence, P->u_inlet};
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b)
    for (int cell = 0; cell < 512; ++cell) {
      const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
      const int gx = (coords[3 * b] - 1) * 8 + x + 1, gy = (coords[3 * b + 1] - 1) * 8 + y + 1,
                gz = (coords[3 * b + 2] - 1) * 8 + z + 1;
      const int64_t ci = cell + 512 * (int64_t)b;
      float f[Q];
      bool saw_inlet = false;
      for (int k = 0; k < Q; ++k) {
        const int sx = x - CX[k], sy = y - CY[k], sz = z - CZ[k];
        const int ox = sx < 0 ? -1 : (sx > 7 ? 1 : 0), oy = sy < 0 ? -1 : (sy > 7 ? 1 : 0), oz = sz < 0 ? -1 : (sz > 7 ? 1 : 0);
        const int bo = (ox | oy | oz) == 0 ? b : nbr[b + (int64_t)nb * ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))] - 1;
        if (bo >= 0) {
          f[k] = fin[(sx - 8 * ox) + 8 * (sy - 8 * oy) + 64 * (sz - 8 * oz) + 512 * (int64_t)bo + N * k];
        } else {
          saw_inlet = saw_inlet || gx - CX[k] < 1;
          f[k] = kbc::face_value(F, fin + ci, (int)N, f_eq_inlet, k, gx, gy, gz);
        }
      }
      if (obstacle && obstacle[ci]) {
        // simple bounce-back inside the obstacle; the multiplier cache is left as it is
        vel_out[ci] = 0.0f; vel_out[ci + N] = 0.0f; vel_out[ci + 2 * N] = 0.0f;
        rho_out[ci] = 1.0f;
        for (int k = 0; k < Q; ++k) fout[ci + N * k] = f[OPP[k]];
        continue;
      }
      if (saw_inlet && gx == 1) kbc::four_moment_pin(f, 1, trho, tjx, tjy, tjz);
      float g[9];
      velocity_gradient_ex(b, x, y, z, nb, nbr, obstacle, vel_in, N, g);
      float la[13];
      for (int m = 0; m < 13; ++m) la[m] = lam[ci + N * m];
      float fo[Q];
      CellOut o;
      const SvvTaps taps{fin, N, nbr, obstacle, nb, b, x, y, z, P->svv_x_epsilon, P->svv_yz_epsilon};
      collide_cell(f, g, *P, f_eq_inlet, la, fo, o, sponge ? sponge[ci] : 0.0f,
                   wall_dist ? wall_dist[ci] : std::numeric_limits<float>::quiet_NaN(), &taps);
      for (int m = 0; m < 13; ++m) lam[ci + N * m] = la[m];
      for (int k = 0; k < Q; ++k) fout[ci + N * k] = fo[k];
      rho_out[ci] = o.rho;
      for (int a = 0; a < 3; ++a) vel_out[ci + N * a] = o.u[a];
    }
}

}  // extern "C"
