// oal_oracle_q19.cpp — CPU ORACLE (test infrastructure only) of the reference's D3Q19 octree solver
// (OpenAeroLab src/octree_q19, Julia, CPU), restated operation for operation in C++ and templated
// on the floating type (float / double, the solver's two precisions). Built with
// -ffp-contract=off: no fused multiply-add, like Julia without @fastmath/@muladd.
//
// Followed (paths inside the reference project):
//   tables CX/CY/CZ/WT/OPP ........ src/octree_q19/src/lattice.jl:8-31
//   moments / Pi_neq / rebuild ..... src/octree_q19/src/kernel.jl:26-70
//   collide_q19 (RR/HRR + Guo) ..... src/octree_q19/src/kernel.jl:92-120
//   below_floor .................... src/octree_q19/src/kernel.jl:72-83
//   positivity safeguard ........... src/octree_q19/src/collision.jl:18-75
//   WALE / Smagorinsky / Vreman .... src/octree_q19/src/collision.jl:77-127
//   velocity gradient .............. src/octree_q19/src/stream.jl:13-30
//   plain-fluid level step ......... src/octree_q19/src/stream.jl:358-370
//   pull tables SRC_OFF/SRC_CHILD .. src/octree_q19/src/octree.jl:139-150, neighbour_slot :152-159
//   oct layout, Morton order ....... src/octree_q19/src/octree.jl:16-33,45-58
//   initialise (Chapman-Enskog) .... src/octree_q19/src/state.jl:267-305, coupling.jl:26-30
//   totals ......................... src/octree_q19/src/state.jl:333-356
//   per-direction reference collision (the known-answer test's definition)
//                                    tools/tests/q19_kernel.jl:20-44
//   face conditions ................ src/octree_q19/src/stream.jl:32-78
//   arriving populations, Bouzidi,
//   momentum exchange .............. src/octree_q19/src/stream.jl:205-257
//   cut-direction tables ........... src/octree_q19/src/state.jl:135-142
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../include/oal.h"

namespace {

constexpr int Q = 19;
// lattice.jl:8-11 (0-based here)
const int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
const int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
const int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
const double WT[Q] = {1.0 / 3, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 36, 1.0 / 36, 1.0 / 36,
                      1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};

template <class T> using Pop = T[Q];

// lattice.jl:27-30
template <class T>
T feq(int i, T rho, T ux, T uy, T uz, T usq) {
  T cu = T(CX[i]) * ux + T(CY[i]) * uy + T(CZ[i]) * uz;
  return T(WT[i]) * rho * (T(1) + T(3) * cu + T(4.5) * cu * cu - T(1.5) * usq);
}
template <class T>
T feq_shifted(int i, T rho, T ux, T uy, T uz, T usq) { return feq<T>(i, rho, ux, uy, uz, usq) - T(WT[i]); }

// kernel.jl:26-45
template <class T>
void moments_q19(const T* f, T& drho, T& mx, T& my, T& mz, T* P) {
  T sx = f[1] + f[2], dx = f[1] - f[2];
  T sy = f[3] + f[4], dy = f[3] - f[4];
  T sz = f[5] + f[6], dz = f[5] - f[6];
  T sxy = f[7] + f[8], dxy = f[7] - f[8];
  T sxY = f[9] + f[10], dxY = f[9] - f[10];
  T sxz = f[11] + f[12], dxz = f[11] - f[12];
  T sxZ = f[13] + f[14], dxZ = f[13] - f[14];
  T syz = f[15] + f[16], dyz = f[15] - f[16];
  T syZ = f[17] + f[18], dyZ = f[17] - f[18];
  T exy = sxy + sxY, exz = sxz + sxZ, eyz = syz + syZ;
  drho = (f[0] + ((sx + sy) + sz)) + ((exy + exz) + eyz);
  mx = dx + ((dxy + dxY) + (dxz + dxZ));
  my = dy + ((dxy - dxY) + (dyz + dyZ));
  mz = dz + ((dxz - dxZ) + (dyz - dyZ));
  P[0] = sx + (exy + exz); P[1] = sy + (exy + eyz); P[2] = sz + (exz + eyz);
  P[3] = sxy - sxY; P[4] = sxz - sxZ; P[5] = syz - syZ;
}

// kernel.jl:48-53
template <class T>
void pineq_q19(T drho, T rho, T ux, T uy, T uz, const T* P, T* p) {
  T d3 = drho * T(1.0 / 3.0);
  T rx = rho * ux, ry = rho * uy, rz = rho * uz;
  p[0] = P[0] - d3 - rx * ux; p[1] = P[1] - d3 - ry * uy; p[2] = P[2] - d3 - rz * uz;
  p[3] = P[3] - rx * uy; p[4] = P[4] - rx * uz; p[5] = P[5] - ry * uz;
}

// kernel.jl:60-82
template <class T>
void populations_q19(T drho, T rho, T ux, T uy, T uz, const T* a2, T keep, T* out) {
  const T pxx = a2[0], pyy = a2[1], pzz = a2[2], pxy = a2[3], pxz = a2[4], pyz = a2[5];
  const T A = drho - T(1.5) * rho * (ux * ux + uy * uy + uz * uz);
  const T k2 = T(4.5) * keep, k3 = T(13.5) * keep;
  const T r3 = T(3) * rho, r45 = T(4.5) * rho;
  const T t = (pxx + pyy + pzz) * T(1.0 / 3.0);
  const T two = T(2), t3 = T(1.0 / 3.0), t23 = T(2.0 / 3.0);
  const T axxy = two * ux * pxy + uy * pxx, axxz = two * ux * pxz + uz * pxx;
  const T ayyx = two * uy * pxy + ux * pyy, ayyz = two * uy * pyz + uz * pyy;
  const T azzx = two * uz * pxz + ux * pzz, azzy = two * uz * pyz + uy * pzz;
  const T w1 = T(1.0 / 18.0), w2 = T(1.0 / 36.0);
  auto pair = [&](T w, T cu, T h2, T h3, T& a, T& b) {
    T e = A + r45 * cu * cu + k2 * h2;
    T o = r3 * cu + k3 * h3;
    a = w * (e + o); b = w * (e - o);
  };
  out[0] = T(1.0 / 3.0) * (A - k2 * t);
  pair(w1, ux, pxx - t, -(ayyx + azzx) * t3, out[1], out[2]);
  pair(w1, uy, pyy - t, -(axxy + azzy) * t3, out[3], out[4]);
  pair(w1, uz, pzz - t, -(axxz + ayyz) * t3, out[5], out[6]);
  const T hxy = pxx + pyy - t, hxz = pxx + pzz - t, hyz = pyy + pzz - t;
  pair(w2, ux + uy, hxy + two * pxy, t23 * (axxy + ayyx) - t3 * (azzx + azzy), out[7], out[8]);
  pair(w2, ux - uy, hxy - two * pxy, t23 * (ayyx - axxy) - t3 * (azzx - azzy), out[9], out[10]);
  pair(w2, ux + uz, hxz + two * pxz, t23 * (axxz + azzx) - t3 * (ayyx + ayyz), out[11], out[12]);
  pair(w2, ux - uz, hxz - two * pxz, t23 * (azzx - axxz) - t3 * (ayyx - ayyz), out[13], out[14]);
  pair(w2, uy + uz, hyz + two * pyz, t23 * (ayyz + azzy) - t3 * (axxy + axxz), out[15], out[16]);
  pair(w2, uy - uz, hyz - two * pyz, t23 * (azzy - ayyz) - t3 * (axxy - axxz), out[17], out[18]);
}

template <class T>
void equilibrium_q19(T drho, T rho, T ux, T uy, T uz, T* out) {
  const T z[6] = {0, 0, 0, 0, 0, 0};
  populations_q19<T>(drho, rho, ux, uy, uz, z, T(0), out);
}

// kernel.jl:72-83
template <class T>
bool below_floor(const T* out) {
  const T l0 = T(-(1 - 1e-6) / 3), l1 = T(-(1 - 1e-6) / 18), l2 = T(-(1 - 1e-6) / 36);
  bool bad = out[0] < l0;
  for (int i = 1; i < 7; ++i) bad = bad | (out[i] < l1);
  for (int i = 7; i < Q; ++i) bad = bad | (out[i] < l2);
  return bad;
}

// collision.jl:5-13
template <class T>
void macros_shifted(const T* f, T& rho, T& ux, T& uy, T& uz) {
  rho = T(1); T mx = 0, my = 0, mz = 0;
  for (int i = 0; i < Q; ++i) { rho += f[i]; mx += T(CX[i]) * f[i]; my += T(CY[i]) * f[i]; mz += T(CZ[i]) * f[i]; }
  T inv = T(1) / rho;
  ux = mx * inv; uy = my * inv; uz = mz * inv;
}

// collision.jl:23-40; returns true when limited (writes `out`)
template <class T>
void positive_shifted(T* out, const T* eq) {
  T alpha = T(1);
  for (int i = 0; i < Q; ++i) {
    T w = T(WT[i]), fl = T(1e-6) * w;
    T actual = out[i] + w;
    if (actual < fl) {
      T equilibrium = eq[i] + w;
      if (!(std::isfinite(equilibrium) && equilibrium > fl)) return;
      T candidate = (equilibrium - fl) / (equilibrium - actual);
      alpha = std::min(alpha, candidate);
    }
  }
  if (alpha < T(1)) {
    T safe_alpha = std::max(T(0), T(0.99) * alpha);
    for (int i = 0; i < Q; ++i) out[i] = eq[i] + safe_alpha * (out[i] - eq[i]);
  }
}

// collision.jl:45-56
template <class T>
void positive_shifted_forced(T* out) {
  bool needs = false;
  for (int i = 0; i < Q; ++i) { T w = T(WT[i]); needs = needs | (out[i] + w < T(1e-6) * w); }
  if (!needs) return;
  T rho, ux, uy, uz;
  macros_shifted<T>(out, rho, ux, uy, uz);
  T usq = ux * ux + uy * uy + uz * uz;
  T eq[Q];
  for (int i = 0; i < Q; ++i) eq[i] = feq_shifted<T>(i, rho, ux, uy, uz, usq);
  positive_shifted<T>(out, eq);
}

// kernel.jl:92-120 (collide_q19), then collision.jl:63-75 (limit_positive)
template <class T>
void collide_rr(const T* f, T omega, T sigma, const T* pi_fd, const T* F, T* out, T& rho, T& ux, T& uy, T& uz) {
  const bool forced = !(F[0] == T(0) && F[1] == T(0) && F[2] == T(0));
  T drho, mx, my, mz, P[6];
  moments_q19<T>(f, drho, mx, my, mz, P);
  rho = drho + T(1);
  T inv = T(1) / rho;
  T hF = forced ? T(0.5) : T(0);
  ux = (mx + hF * F[0]) * inv; uy = (my + hF * F[1]) * inv; uz = (mz + hF * F[2]) * inv;
  T p[6];
  pineq_q19<T>(drho, rho, ux, uy, uz, P, p);
  T s1 = T(1) - sigma;
  T a2[6];
  if (sigma == T(1)) for (int n = 0; n < 6; ++n) a2[n] = p[n];
  else for (int n = 0; n < 6; ++n) a2[n] = sigma * p[n] + s1 * pi_fd[n];
  T base[Q];
  populations_q19<T>(drho, rho, ux, uy, uz, a2, T(1) - omega, base);
  if (forced) {
    T pre = T(1) - T(0.5) * omega;
    T uF = ux * F[0] + uy * F[1] + uz * F[2];
    for (int i = 0; i < Q; ++i) {
      T cx = T(CX[i]), cy = T(CY[i]), cz = T(CZ[i]);
      T cu = cx * ux + cy * uy + cz * uz, cF = cx * F[0] + cy * F[1] + cz * F[2];
      out[i] = base[i] + T(WT[i]) * (T(1.5) * cF + pre * (T(9) * cu * cF - T(3) * uF));
    }
  } else {
    for (int i = 0; i < Q; ++i) out[i] = base[i];
  }
  if (!below_floor<T>(out)) return;
  if (forced) { positive_shifted_forced<T>(out); return; }
  T eq[Q];
  equilibrium_q19<T>(drho, rho, ux, uy, uz, eq);
  positive_shifted<T>(out, eq);
}

// tools/tests/q19_kernel.jl:20-44: the per-direction collision the closed form replaced
template <class T>
void reference_collide(const T* f, T omega, T sigma, const T* pfd, const T* F, T* out) {
  T rho, mx, my, mz;
  {
    rho = T(1); mx = 0; my = 0; mz = 0;
    for (int i = 0; i < Q; ++i) { rho += f[i]; mx += T(CX[i]) * f[i]; my += T(CY[i]) * f[i]; mz += T(CZ[i]) * f[i]; }
    T inv = T(1) / rho;
    mx = mx * inv; my = my * inv; mz = mz * inv;   // macros_shifted returns velocities
  }
  const bool forced = F[0] != T(0) || F[1] != T(0) || F[2] != T(0);
  T h = forced ? T(0.5) / rho : T(0);
  T u[3] = {mx + h * F[0], my + h * F[1], mz + h * F[2]};
  T usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  T feqs[Q];
  for (int i = 0; i < Q; ++i) feqs[i] = feq_shifted<T>(i, rho, u[0], u[1], u[2], usq);
  T p[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 1; i < Q; ++i) {
    T fn = f[i] - feqs[i], cx = T(CX[i]), cy = T(CY[i]), cz = T(CZ[i]);
    p[0] += cx * cx * fn; p[1] += cy * cy * fn; p[2] += cz * cz * fn;
    p[3] += cx * cy * fn; p[4] += cx * cz * fn; p[5] += cy * cz * fn;
  }
  T a2[6];
  for (int n = 0; n < 6; ++n) a2[n] = sigma * p[n] + (T(1) - sigma) * pfd[n];
  const T ux = u[0], uy = u[1], uz = u[2];
  T a3[6] = {T(2) * ux * a2[3] + uy * a2[0], T(2) * ux * a2[4] + uz * a2[0], T(2) * uy * a2[3] + ux * a2[1],
             T(2) * uy * a2[5] + uz * a2[1], T(2) * uz * a2[4] + ux * a2[2], T(2) * uz * a2[5] + uy * a2[2]};
  T keep = T(1) - omega, pre = T(1) - T(0.5) * omega;
  for (int i = 0; i < Q; ++i) {
    T cx = T(CX[i]), cy = T(CY[i]), cz = T(CZ[i]), third = T(1) / T(3);
    T h2 = (cx * cx - third) * a2[0] + (cy * cy - third) * a2[1] + (cz * cz - third) * a2[2] +
           T(2) * (cx * cy * a2[3] + cx * cz * a2[4] + cy * cz * a2[5]);
    T h3 = cy * (cx * cx - third) * a3[0] + cz * (cx * cx - third) * a3[1] + cx * (cy * cy - third) * a3[2] +
           cz * (cy * cy - third) * a3[3] + cx * (cz * cz - third) * a3[4] + cy * (cz * cz - third) * a3[5];
    T fneq = T(WT[i]) * (T(4.5) * h2 + T(13.5) * h3);
    T cu = cx * ux + cy * uy + cz * uz, cF = cx * F[0] + cy * F[1] + cz * F[2], uF = ux * F[0] + uy * F[1] + uz * F[2];
    out[i] = feqs[i] + keep * fneq + (forced ? T(WT[i]) * (T(1.5) * cF + pre * (T(9) * cu * cF - T(3) * uF)) : T(0));
  }
}

// collision.jl:78-127
template <class T>
T nu_wale(const T* g, T cw) {
  T g11 = g[0], g12 = g[1], g13 = g[2], g21 = g[3], g22 = g[4], g23 = g[5], g31 = g[6], g32 = g[7], g33 = g[8];
  T s11 = g11, s22 = g22, s33 = g33;
  T s12 = T(0.5) * (g12 + g21), s13 = T(0.5) * (g13 + g31), s23 = T(0.5) * (g23 + g32);
  T q11 = g11 * g11 + g12 * g21 + g13 * g31, q12 = g11 * g12 + g12 * g22 + g13 * g32, q13 = g11 * g13 + g12 * g23 + g13 * g33;
  T q21 = g21 * g11 + g22 * g21 + g23 * g31, q22 = g21 * g12 + g22 * g22 + g23 * g32, q23 = g21 * g13 + g22 * g23 + g23 * g33;
  T q31 = g31 * g11 + g32 * g21 + g33 * g31, q32 = g31 * g12 + g32 * g22 + g33 * g32, q33 = g31 * g13 + g32 * g23 + g33 * g33;
  T tr = (q11 + q22 + q33) / T(3);
  T d11 = q11 - tr, d22 = q22 - tr, d33 = q33 - tr;
  T d12 = T(0.5) * (q12 + q21), d13 = T(0.5) * (q13 + q31), d23 = T(0.5) * (q23 + q32);
  T ss = s11 * s11 + s22 * s22 + s33 * s33 + T(2) * (s12 * s12 + s13 * s13 + s23 * s23);
  T dd = d11 * d11 + d22 * d22 + d33 * d33 + T(2) * (d12 * d12 + d13 * d13 + d23 * d23);
  T den = ss * ss * std::sqrt(ss) + dd * std::sqrt(std::sqrt(dd)) + T(1e-20);
  return cw * cw * dd * std::sqrt(dd) / den;
}
template <class T>
T nu_smagorinsky(const T* g, T cs) {
  T s12 = T(0.5) * (g[1] + g[3]), s13 = T(0.5) * (g[2] + g[6]), s23 = T(0.5) * (g[5] + g[7]);
  T ss = g[0] * g[0] + g[4] * g[4] + g[8] * g[8] + T(2) * (s12 * s12 + s13 * s13 + s23 * s23);
  return cs * cs * std::sqrt(T(2) * ss);
}
template <class T>
T nu_vreman(const T* g, T c) {
  T g11 = g[0], g12 = g[1], g13 = g[2], g21 = g[3], g22 = g[4], g23 = g[5], g31 = g[6], g32 = g[7], g33 = g[8];
  T b11 = g11 * g11 + g21 * g21 + g31 * g31, b22 = g12 * g12 + g22 * g22 + g32 * g32, b33 = g13 * g13 + g23 * g23 + g33 * g33;
  T b12 = g11 * g12 + g21 * g22 + g31 * g32, b13 = g11 * g13 + g21 * g23 + g31 * g33, b23 = g12 * g13 + g22 * g23 + g32 * g33;
  T bb = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
  T aa = b11 + b22 + b33;
  bool off = (aa <= T(1e-20)) | (bb <= T(0));
  return off ? T(0) : c * std::sqrt(off ? T(1) : bb / aa);
}
template <class T> T omega_of(T nu) { return T(1) / (T(3) * nu + T(0.5)); }
template <class T>
void pi_fd_from_gradient(const T* g, T rho, T tau, T* p) {
  T c = -rho * tau / T(3);
  p[0] = c * T(2) * g[0]; p[1] = c * T(2) * g[4]; p[2] = c * T(2) * g[8];
  p[3] = c * (g[1] + g[3]); p[4] = c * (g[2] + g[6]); p[5] = c * (g[5] + g[7]);
}

// octree.jl:16-33, 139-159
inline void slot_offset(int k, int& x, int& y, int& z) { x = k & 1; y = (k >> 1) & 1; z = (k >> 2) & 1; }  // k 0-based
inline int slot_index(int x, int y, int z) { return x + 2 * y + 4 * z; }
inline int nbr_index(int dx, int dy, int dz) { return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); }
inline void source(int k, int i, int& off, int& child) {
  int x, y, z;
  slot_offset(k, x, y, z);
  int p[3] = {x - CX[i], y - CY[i], z - CZ[i]}, o[3];
  for (int a = 0; a < 3; ++a) o[a] = p[a] < 0 ? -1 : (p[a] > 1 ? 1 : 0);
  off = nbr_index(o[0], o[1], o[2]);
  child = slot_index(p[0] - 2 * o[0], p[1] - 2 * o[1], p[2] - 2 * o[2]);
}
inline void neighbour_slot(int k, int dx, int dy, int dz, int& ni, int& nk) {
  int x, y, z;
  slot_offset(k, x, y, z);
  int nx = x + dx, ny = y + dy, nz = z + dz;
  int ox = nx < 0 ? -1 : (nx > 1 ? 1 : 0), oy = ny < 0 ? -1 : (ny > 1 ? 1 : 0), oz = nz < 0 ? -1 : (nz > 1 ? 1 : 0);
  ni = nbr_index(ox, oy, oz);
  nk = slot_index(nx - 2 * ox, ny - 2 * oy, nz - 2 * oz);
}

uint64_t spread(uint64_t v) {
  v &= 0x1fffff;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}
uint64_t morton(uint64_t ix, uint64_t iy, uint64_t iz) { return spread(ix) | (spread(iy) << 1) | (spread(iz) << 2); }

struct Q19Level {
  int nocts;
  const int32_t* onbr;  // (27, nocts) 1-based, 0 none
};

// stream.jl:13-30: gradient g[a, b] = d u_b / d x_a; missing neighbour -> own velocity
template <class T>
void velocity_gradient(const Q19Level& L, const T* u, int k, int o, T* g) {
  auto at = [&](int dx, int dy, int dz, T* v) {
    int ni, nk;
    neighbour_slot(k, dx, dy, dz, ni, nk);
    int no = L.onbr[ni + 27 * o];
    if (no == 0) { for (int a = 0; a < 3; ++a) v[a] = u[k + 8 * a + 24 * o]; return; }
    for (int a = 0; a < 3; ++a) v[a] = u[nk + 8 * a + 24 * (no - 1)];
  };
  T xp[3], xm[3], yp[3], ym[3], zp[3], zm[3];
  at(1, 0, 0, xp); at(-1, 0, 0, xm); at(0, 1, 0, yp); at(0, -1, 0, ym); at(0, 0, 1, zp); at(0, 0, -1, zm);
  T h = T(0.5);
  g[0] = h * (xp[0] - xm[0]); g[1] = h * (xp[1] - xm[1]); g[2] = h * (xp[2] - xm[2]);
  g[3] = h * (yp[0] - ym[0]); g[4] = h * (yp[1] - ym[1]); g[5] = h * (yp[2] - ym[2]);
  g[6] = h * (zp[0] - zm[0]); g[7] = h * (zp[1] - zm[1]); g[8] = h * (zp[2] - zm[2]);
}

// stream.jl:358-370 for a level whose slots are all plain fluid (every pull source exists)
template <class T>
void step_level(const Q19Level& L, const oal_q19_params& P, const T* fin, T* fout, const T* uin, T* vout, const T* rho_a,
                T* rhob) {
  const T nu = T(P.nu), cw = T(P.c_wale), cs = T(P.c_smagorinsky), cv = T(2.5 * P.c_smagorinsky * P.c_smagorinsky);
  const T sigma = T(P.hrr_sigma);
  const T F[3] = {T(P.body_force[0]), T(P.body_force[1]), T(P.body_force[2])};
  const bool need_gradient = P.sgs != 0 || sigma != T(1);
  const T omega0 = omega_of<T>(nu);
#pragma omp parallel for schedule(static)
  for (int o = 0; o < L.nocts; ++o) {
    for (int k = 0; k < 8; ++k) {
      T f[Q];
      for (int i = 0; i < Q; ++i) {
        int off, child;
        source(k, i, off, child);
        int so = L.onbr[off + 27 * o] - 1;
        f[i] = fin[child + 8 * i + 152 * so];
      }
      T g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      if (need_gradient) velocity_gradient<T>(L, uin, k, o, g);
      T nut = P.sgs == 1 ? nu_wale<T>(g, cw) : P.sgs == 2 ? nu_smagorinsky<T>(g, cs) : P.sgs == 3 ? nu_vreman<T>(g, cv) : T(0);
      T omega = need_gradient ? omega_of<T>(nu + nut) : omega0;
      T pfd[6] = {0, 0, 0, 0, 0, 0};
      if (sigma != T(1)) pi_fd_from_gradient<T>(g, rho_a[k + 8 * o], T(1) / omega, pfd);
      T out[Q], rho, ux, uy, uz;
      collide_rr<T>(f, omega, sigma, pfd, F, out, rho, ux, uy, uz);
      for (int i = 0; i < Q; ++i) fout[k + 8 * i + 152 * o] = out[i];
      vout[k + 24 * o] = ux; vout[k + 8 + 24 * o] = uy; vout[k + 16 + 24 * o] = uz;
      rhob[k + 8 * o] = rho;
    }
  }
}

// coupling.jl:26-30
template <class T>
void rebuild(T rho, T ux, T uy, T uz, const T* p, T omega, T* out) {
  T drho = rho - T(1);
  populations_q19<T>(drho, rho, ux, uy, uz, p, T(1) - omega, out);
  if (below_floor<T>(out)) {
    T eq[Q];
    equilibrium_q19<T>(drho, rho, ux, uy, uz, eq);
    positive_shifted<T>(out, eq);
  }
}

// state.jl:267-305: per fluid, ghost or covered slot, the Chapman-Enskog non-equilibrium of the initial field (du given,
// (8, 9, nocts) with du[k, 3a+b, o] = d u_b / d x_a over one cell) rebuilt at the level's omega,
// or the equilibrium (du null). rho (8, nocts), u (8, 3, nocts), f (8, 19, nocts).
template <class T>
void initialise(int64_t nslots, const uint8_t* kind, const T* rho_a, const T* u, const T* du, double nu_d, T* f,
                T* u_out, T* rho_out) {
  const T nu = T(nu_d);
  const T omega = omega_of<T>(nu), tau = T(1) / omega;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < nslots; ++s) {
    const int64_t o = s / 8;
    const int k = (int)(s % 8);
    if (kind && kind[s] != 1 && kind[s] != 3 && kind[s] != 4) {
      // slots without a state keep the allocation state (state.jl:217-232)
      for (int i = 0; i < Q; ++i) f[k + 8 * i + 152 * o] = T(0);
      for (int a = 0; a < 3; ++a) u_out[k + 8 * a + 24 * o] = T(0);
      rho_out[s] = T(1);
      continue;
    }
    const T rho = rho_a[s], ux = u[k + 24 * o], uy = u[k + 8 + 24 * o], uz = u[k + 16 + 24 * o];
    for (int a = 0; a < 3; ++a) u_out[k + 8 * a + 24 * o] = u[k + 8 * a + 24 * o];
    rho_out[s] = rho;
    T out[Q];
    if (du) {
      T d[9];
      for (int n = 0; n < 9; ++n) d[n] = du[k + 8 * n + 72 * o];
      const T c = -rho * tau / T(3);
      const T pn[6] = {c * T(2) * d[0], c * T(2) * d[4], c * T(2) * d[8], c * (d[1] + d[3]), c * (d[2] + d[6]), c * (d[5] + d[7])};
      rebuild<T>(rho, ux, uy, uz, pn, omega, out);
    } else {
      equilibrium_q19<T>(rho - T(1), rho, ux, uy, uz, out);
    }
    for (int i = 0; i < Q; ++i) f[k + 8 * i + 152 * o] = out[i];
  }
}

// ---- a level with domain faces and cut links (stream.jl:32-78, 205-257, 280-370) ----------------

inline int dir_index(int x, int y, int z) {
  for (int i = 0; i < Q; ++i)
    if (CX[i] == x && CY[i] == y && CZ[i] == z) return i;
  return -1;
}
inline int opp_of(int i) { return dir_index(-CX[i], -CY[i], -CZ[i]); }
inline int mirror_of(int i, int axis) {
  return dir_index(axis == 0 ? -CX[i] : CX[i], axis == 1 ? -CY[i] : CY[i], axis == 2 ? -CZ[i] : CZ[i]);
}

// stream.jl:32-47 (face conditions: OAL_Q19_FACE_*)
template <class T>
T face_dirichlet(int cond, int j, const T* fo, T rho, T ux, T uy, T uz, const T* uin) {
  const int i = opp_of(j);
  const T usq = ux * ux + uy * uy + uz * uz;
  if (cond == OAL_Q19_FACE_INLET) {
    const T vsq = uin[0] * uin[0] + uin[1] * uin[1] + uin[2] * uin[2];
    return feq_shifted<T>(j, rho, uin[0], uin[1], uin[2], vsq) + (fo[i] - feq_shifted<T>(i, rho, ux, uy, uz, usq));
  } else if (cond == OAL_Q19_FACE_OUTLET) {
    return feq_shifted<T>(j, T(1), ux, uy, uz, usq) + (fo[i] - feq_shifted<T>(i, rho, ux, uy, uz, usq));
  }
  const T vsq = uin[0] * uin[0] + uin[1] * uin[1] + uin[2] * uin[2];
  return feq_shifted<T>(j, T(1), uin[0], uin[1], uin[2], vsq) + (fo[i] - feq_shifted<T>(i, rho, ux, uy, uz, usq));
}

// stream.jl:49-78
template <class T>
T face_population(uint8_t mask, const int32_t* faces, int j, const T* fo, T rho, T ux, T uy, T uz, const T* uin) {
  const int i = opp_of(j);
  if (__builtin_popcount(mask) == 1) {
    const int f = __builtin_ctz(mask);
    const int cond = faces[f];
    if (cond == OAL_Q19_FACE_NOSLIP || cond == OAL_Q19_FACE_GROUND) return fo[i];
    if (cond == OAL_Q19_FACE_SLIP || cond == OAL_Q19_FACE_SYMMETRY) return fo[mirror_of(j, f <= 1 ? 0 : f <= 3 ? 1 : 2)];
    return face_dirichlet<T>(cond, j, fo, rho, ux, uy, uz, uin);
  }
  bool wall = false, open = false;
  for (int f = 0; f < 6; ++f) {
    if (!((mask >> f) & 1)) continue;
    const int c = faces[f];
    if (c == OAL_Q19_FACE_NOSLIP || c == OAL_Q19_FACE_GROUND) wall = true;
    if (c == OAL_Q19_FACE_INLET || c == OAL_Q19_FACE_OUTLET || c == OAL_Q19_FACE_FREESTREAM) open = true;
  }
  if (wall) return fo[i];
  if (open) return face_dirichlet<T>(OAL_Q19_FACE_FREESTREAM, j, fo, rho, ux, uy, uz, uin);
  int m = j;
  if (mask & 0x03) m = mirror_of(m, 0);
  if (mask & 0x0c) m = mirror_of(m, 1);
  if (mask & 0x30) m = mirror_of(m, 2);
  return fo[m];
}

template <class T>
void step_level_walls(const oal_q19_level_desc& d, const oal_q19_params& P, const T* fin, T* fout, const T* uin,
                      T* vout, const T* rho_a, T* rhob, double* mom) {
  const T nu = T(P.nu), cw = T(P.c_wale), cs = T(P.c_smagorinsky), cv = T(2.5 * P.c_smagorinsky * P.c_smagorinsky);
  const T sigma = T(P.hrr_sigma);
  const T F[3] = {T(P.body_force[0]), T(P.body_force[1]), T(P.body_force[2])};
  const T uinlet[3] = {T(P.u_inlet[0]), T(P.u_inlet[1]), T(P.u_inlet[2])};
  const bool need_gradient = P.sgs != 0 || sigma != T(1);
  const T omega0 = omega_of<T>(nu);
  const int64_t nslots = (int64_t)d.nocts * 8;
  // cut_direction_tables (state.jl:135-142): q per direction of each cut cell (0.5 elsewhere), partner flag
  std::vector<float> qdir((size_t)std::max(d.ncut, 1) * Q, 0.5f);
  std::vector<uint8_t> okdir((size_t)std::max(d.ncut, 1) * Q, 0);
  for (int c = 0; c < d.ncut; ++c)
    for (int li = d.cut_off[c] - 1; li < d.cut_off[c + 1] - 1; ++li) {
      qdir[(size_t)c * Q + d.cut_dir[li] - 1] = d.cut_q[li];
      okdir[(size_t)c * Q + d.cut_dir[li] - 1] = d.cut_partner[li];
    }
  auto kind = [&](int64_t s) -> uint8_t { return d.kind ? d.kind[s] : 1; };
#pragma omp parallel for schedule(dynamic, 64)
  for (int o = 0; o < d.nocts; ++o) {
    if (d.real && !d.real[o]) continue;
    for (int k = 0; k < 8; ++k) {
      const int64_t s = 8 * (int64_t)o + k;
      if (kind(s) != 1) continue;
      const uint32_t sp = d.special ? d.special[s] : 0u;
      T f[Q];
      if (sp == 0) {
        for (int j = 0; j < Q; ++j) {
          int off, child;
          source(k, j, off, child);
          f[j] = fin[child + 8 * j + 152 * (int64_t)(d.onbr[off + 27 * (int64_t)o] - 1)];
        }
      } else {
        // stream.jl:205-246: the own post-collision populations and the previous macros
        T fo[Q];
        for (int j = 0; j < Q; ++j) fo[j] = fin[k + 8 * j + 152 * (int64_t)o];
        const T rho0 = rho_a[s], ux0 = uin[k + 24 * (int64_t)o], uy0 = uin[k + 8 + 24 * (int64_t)o],
                uz0 = uin[k + 16 + 24 * (int64_t)o];
        const int ci = d.cutidx ? d.cutidx[s] : 0;
        for (int j = 0; j < Q; ++j) {
          int off, child;
          source(k, j, off, child);
          const int so = d.onbr[off + 27 * (int64_t)o];
          if (!((sp >> j) & 1u)) {
            f[j] = fin[child + 8 * j + 152 * (int64_t)(so - 1)];
          } else if (so != 0 && kind(8 * (int64_t)(so - 1) + child) == 5) {
            f[j] = face_population<T>(d.face[8 * (int64_t)(so - 1) + child], d.faces, j, fo, rho0, ux0, uy0, uz0, uinlet);
          } else {
            const int i = opp_of(j);
            const T q = T(qdir[(size_t)(ci - 1) * Q + i]);
            const bool ok = okdir[(size_t)(ci - 1) * Q + i] != 0;
            if (!ok) {
              f[j] = fo[i];
            } else if (q < T(0.5)) {
              int pi_, pk_;
              neighbour_slot(k, -CX[i], -CY[i], -CZ[i], pi_, pk_);
              const int po = d.onbr[pi_ + 27 * (int64_t)o];
              f[j] = T(2) * q * fo[i] + (T(1) - T(2) * q) * fin[pk_ + 8 * i + 152 * (int64_t)(po - 1)];
            } else {
              const T inv2q = T(1) / (T(2) * q);
              f[j] = inv2q * fo[i] + (T(1) - inv2q) * fo[j];
            }
          }
        }
        if (mom && ci != 0) {
          // momentum exchange per cut link, added up over the collecting steps: scale (f_i* + f_j(t+1)),
          // i toward the wall (stream.jl:248-256)
          for (int li = d.cut_off[ci - 1] - 1; li < d.cut_off[ci] - 1; ++li) {
            const int i = d.cut_dir[li] - 1, j = opp_of(i);
            mom[li] += P.force_scale * (double)(fo[i] + f[j]);
          }
        }
      }
      // gradient of the previous velocity: missing or boundary neighbours give the own value (stream.jl:13-30)
      T g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      if (need_gradient) {
        auto at = [&](int ex, int ey, int ez, T* v) {
          int ni, nk;
          neighbour_slot(k, ex, ey, ez, ni, nk);
          const int no = d.onbr[ni + 27 * (int64_t)o];
          if (no == 0 || kind(8 * (int64_t)(no - 1) + nk) == 5) {
            for (int a = 0; a < 3; ++a) v[a] = uin[k + 8 * a + 24 * (int64_t)o];
            return;
          }
          for (int a = 0; a < 3; ++a) v[a] = uin[nk + 8 * a + 24 * (int64_t)(no - 1)];
        };
        T xp[3], xm[3], yp[3], ym[3], zp[3], zm[3];
        at(1, 0, 0, xp); at(-1, 0, 0, xm); at(0, 1, 0, yp); at(0, -1, 0, ym); at(0, 0, 1, zp); at(0, 0, -1, zm);
        const T h = T(0.5);
        g[0] = h * (xp[0] - xm[0]); g[1] = h * (xp[1] - xm[1]); g[2] = h * (xp[2] - xm[2]);
        g[3] = h * (yp[0] - ym[0]); g[4] = h * (yp[1] - ym[1]); g[5] = h * (yp[2] - ym[2]);
        g[6] = h * (zp[0] - zm[0]); g[7] = h * (zp[1] - zm[1]); g[8] = h * (zp[2] - zm[2]);
      }
      const T nut = P.sgs == 1 ? nu_wale<T>(g, cw) : P.sgs == 2 ? nu_smagorinsky<T>(g, cs) : P.sgs == 3 ? nu_vreman<T>(g, cv) : T(0);
      const T omega = need_gradient ? omega_of<T>(nu + nut) : omega0;
      T pfd[6] = {0, 0, 0, 0, 0, 0};
      if (sigma != T(1)) pi_fd_from_gradient<T>(g, rho_a[s], T(1) / omega, pfd);
      T out[Q], rho, ux, uy, uz;
      collide_rr<T>(f, omega, sigma, pfd, F, out, rho, ux, uy, uz);
      for (int i = 0; i < Q; ++i) fout[k + 8 * i + 152 * (int64_t)o] = out[i];
      vout[k + 24 * (int64_t)o] = ux;
      vout[k + 8 + 24 * (int64_t)o] = uy;
      vout[k + 16 + 24 * (int64_t)o] = uz;
      rhob[s] = rho;
    }
  }
  (void)nslots;
}

// ---- transfers between levels (coupling.jl:16-238) -------------------------------------------

template <class T>
void slot_moments(const T* f, int64_t s, T* m) {  // coupling.jl:16-23
  const int64_t o = s / 8;
  const int k = (int)(s % 8);
  T fs[Q];
  for (int i = 0; i < Q; ++i) fs[i] = f[k + 8 * i + 152 * o];
  T drho, mx, my, mz, P[6];
  moments_q19<T>(fs, drho, mx, my, mz, P);
  const T rho = drho + T(1), inv = T(1) / rho;
  const T ux = mx * inv, uy = my * inv, uz = mz * inv;
  T p[6];
  pineq_q19<T>(drho, rho, ux, uy, uz, P, p);
  m[0] = rho; m[1] = ux; m[2] = uy; m[3] = uz;
  for (int i = 0; i < 6; ++i) m[4 + i] = p[i];
}

template <class T>
T pre_collision_factor(T omega) {  // coupling.jl:32-35
  return std::abs(T(1) - omega) > T(0.05) ? T(1) / (T(1) - omega) : T(0);
}

template <class T>
void write_rebuilt(const T* acc, T scale, T omega, int64_t s, T* f, T* u, T* rho) {
  const T p[6] = {scale * acc[4], scale * acc[5], scale * acc[6], scale * acc[7], scale * acc[8], scale * acc[9]};
  T out[Q];
  rebuild<T>(acc[0], acc[1], acc[2], acc[3], p, omega, out);
  const int64_t o = s / 8;
  const int k = (int)(s % 8);
  for (int i = 0; i < Q; ++i) f[k + 8 * i + 152 * o] = out[i];
  u[k + 24 * o] = acc[1]; u[k + 8 + 24 * o] = acc[2]; u[k + 16 + 24 * o] = acc[3];
  rho[s] = acc[0];
}

// fill_ghosts! (coupling.jl:134-174): the ghosts of the fine level from the coarse buffers at `weight`
template <class T>
void fill_ghosts(const oal_q19_level_desc& F, const uint8_t* ckind, const T* cnew, const T* cold, T weight,
                 double nu_c, double nu_f, T* ff, T* fu, T* fr) {
  const T omega_c = omega_of<T>(T(nu_c)), omega_f = omega_of<T>(T(nu_f));
  const T tau_c = T(1) / omega_c, tau_f = T(1) / omega_f;
  const T scale = tau_f / (T(2) * tau_c) * pre_collision_factor<T>(omega_c);
  const T w1 = weight, w0 = T(1) - weight;
#pragma omp parallel for schedule(static)
  for (int g = 0; g < F.nghost; ++g) {
    T acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int n = 0; n < 64; ++n) {
      const int d = F.ghost_donor[64 * (int64_t)g + n];
      if (!d) continue;
      const int64_t ds = d - 1;
      T m[10];
      if (w1 == T(0)) {
        slot_moments<T>(cold, ds, m);
      } else if (w0 == T(0) || (ckind && ckind[ds] == 3)) {
        slot_moments<T>(cnew, ds, m);  // covered donors hold the fine average and enter unblended
      } else {
        T mn[10], mo[10];
        slot_moments<T>(cnew, ds, mn);
        slot_moments<T>(cold, ds, mo);
        for (int i = 0; i < 10; ++i) m[i] = w0 * mo[i] + w1 * mn[i];
      }
      const T wn = T(F.ghost_w[64 * (int64_t)g + n]);
      for (int i = 0; i < 10; ++i) acc[i] += wn * m[i];
    }
    write_rebuilt<T>(acc, scale, omega_f, F.ghost_slot[g] - 1, ff, fu, fr);
  }
}

// restrict! (coupling.jl:176-207): the restricted slots of the coarse level from the fine buffer
template <class T>
void restrict_level(const oal_q19_level_desc& C, const T* ff, double nu_c, double nu_f, T* cf, T* cu, T* cr) {
  const T omega_c = omega_of<T>(T(nu_c)), omega_f = omega_of<T>(T(nu_f));
  const T tau_c = T(1) / omega_c, tau_f = T(1) / omega_f;
  const T scale = T(2) * tau_c / tau_f * pre_collision_factor<T>(omega_f);
  double w1d[4];
  {
    const double t = 0.5;  // cubic_weights(0.5) (octree.jl:84-86)
    w1d[0] = -t * (1 - t) * (2 - t) / 6; w1d[1] = (1 + t) * (1 - t) * (2 - t) / 2;
    w1d[2] = (1 + t) * t * (2 - t) / 2; w1d[3] = -(1 + t) * t * (1 - t) / 6;
  }
#pragma omp parallel for schedule(static)
  for (int r = 0; r < C.nrestrict; ++r) {
    T acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (C.restrict_cubic[r]) {
      for (int n = 0; n < 64; ++n) {
        const T wn = T(w1d[n & 3] * w1d[(n >> 2) & 3] * w1d[n >> 4]);
        T m[10];
        slot_moments<T>(ff, C.restrict_src[64 * (int64_t)r + n] - 1, m);
        for (int i = 0; i < 10; ++i) acc[i] += wn * m[i];
      }
    } else {
      int cnt = 0;
      for (int mm = 0; mm < 8; ++mm) {  // STENCIL_INNER order (octree.jl:82)
        const int nidx = (1 + (mm & 1)) + 4 * (1 + ((mm >> 1) & 1)) + 16 * (1 + ((mm >> 2) & 1));
        const int d = C.restrict_src[64 * (int64_t)r + nidx];
        if (!d) continue;
        T m[10];
        slot_moments<T>(ff, d - 1, m);
        for (int i = 0; i < 10; ++i) acc[i] += m[i];
        ++cnt;
      }
      if (cnt == 0) continue;
      const T inv = T(1) / T(cnt);
      for (int i = 0; i < 10; ++i) acc[i] *= inv;
    }
    write_rebuilt<T>(acc, scale, omega_c, C.restrict_slot[r] - 1, cf, cu, cr);
  }
}

}  // namespace

extern "C" {

#define ORA_Q19_TRANSFER(T, SUF)                                                                              \
  void ora_q19_fill_##SUF(const oal_q19_level_desc* F, const uint8_t* ckind, const T* cnew, const T* cold,     \
                          double weight, double nu_c, double nu_f, T* ff, T* fu, T* fr) {                     \
    fill_ghosts<T>(*F, ckind, cnew, cold, T(weight), nu_c, nu_f, ff, fu, fr);                                 \
  }                                                                                                           \
  void ora_q19_restrict_##SUF(const oal_q19_level_desc* C, const T* ff, double nu_c, double nu_f, T* cf, T* cu, \
                              T* cr) {                                                                        \
    restrict_level<T>(*C, ff, nu_c, nu_f, cf, cu, cr);                                                        \
  }
ORA_Q19_TRANSFER(float, f32)
ORA_Q19_TRANSFER(double, f64)
#undef ORA_Q19_TRANSFER

// per-triangle force in link order (no triangle -> bin 1) and the total as a plain sum over the bins
void ora_q19_forces(const oal_q19_level_desc* d, const double* mom, double* per_tri, double* total) {
  const int ntri = std::max(d->ntri, 1);
  for (int t = 0; t < 3 * ntri; ++t) per_tri[t] = 0;
  for (int li = 0; li < d->nlinks; ++li) {
    const int t = (d->cut_tri && d->cut_tri[li] > 0 ? d->cut_tri[li] : 1) - 1;
    const int i = d->cut_dir[li] - 1;
    per_tri[3 * t] += mom[li] * CX[i];
    per_tri[3 * t + 1] += mom[li] * CY[i];
    per_tri[3 * t + 2] += mom[li] * CZ[i];
  }
  total[0] = total[1] = total[2] = 0;
  for (int t = 0; t < ntri; ++t)
    for (int a = 0; a < 3; ++a) total[a] += per_tri[3 * t + a];
}


void ora_q19_tables(int32_t* cx, int32_t* cy, int32_t* cz, double* w, int32_t* src_off, int32_t* src_child) {
  for (int i = 0; i < Q; ++i) { cx[i] = CX[i]; cy[i] = CY[i]; cz[i] = CZ[i]; w[i] = WT[i]; }
  for (int k = 0; k < 8; ++k)
    for (int i = 0; i < Q; ++i) { int off, child; source(k, i, off, child); src_off[k * Q + i] = off; src_child[k * Q + i] = child; }
}

// Periodic box of (n0,n1,n2) cells (even): octs in Morton order of their origin, 27-entry neighbour
// table with periodic wrap (octree.jl:45-58, oct_key; generator's level 1 of a periodic box).
int ora_q19_periodic_box(int32_t n0, int32_t n1, int32_t n2, int32_t* origin, int32_t* onbr) {
  const int m0 = n0 / 2, m1 = n1 / 2, m2 = n2 / 2;
  const int64_t no = (int64_t)m0 * m1 * m2;
  std::vector<std::pair<uint64_t, int64_t>> keys;
  keys.reserve(no);
  for (int i = 0; i < m0; ++i)
    for (int j = 0; j < m1; ++j)
      for (int k = 0; k < m2; ++k) keys.push_back({morton(i + 1, j + 1, k + 1), ((int64_t)i * m1 + j) * m2 + k});
  std::sort(keys.begin(), keys.end());
  std::vector<int32_t> index((size_t)no);
  for (int64_t o = 0; o < no; ++o) index[(size_t)keys[o].second] = (int32_t)o;
  for (int64_t o = 0; o < no; ++o) {
    const int64_t lin = keys[o].second;
    const int i = (int)(lin / ((int64_t)m1 * m2)), j = (int)((lin / m2) % m1), k = (int)(lin % m2);
    origin[3 * o] = 2 * i; origin[3 * o + 1] = 2 * j; origin[3 * o + 2] = 2 * k;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int a = (i + dx + m0) % m0, b = (j + dy + m1) % m1, c = (k + dz + m2) % m2;
          onbr[nbr_index(dx, dy, dz) + 27 * o] = index[((size_t)a * m1 + b) * m2 + c] + 1;
        }
  }
  return 0;
}

// Closed-form collision of n cells (arrays (n, 19) / (n, 6) / (n, 3)), and the per-direction reference.
#define ORA_Q19_COLLIDE(T, SUF)                                                                                  \
  void ora_q19_collide_##SUF(int64_t n, const T* f, const T* omega, T sigma, const T* pfd, const T* F, T* out,   \
                             T* rho, T* u) {                                                                    \
    for (int64_t c = 0; c < n; ++c)                                                                             \
      collide_rr<T>(f + 19 * c, omega[c], sigma, pfd + 6 * c, F + 3 * c, out + 19 * c, rho[c], u[3 * c],        \
                    u[3 * c + 1], u[3 * c + 2]);                                                                \
  }                                                                                                              \
  void ora_q19_reference_collide_##SUF(int64_t n, const T* f, const T* omega, T sigma, const T* pfd, const T* F, \
                                       T* out) {                                                                \
    for (int64_t c = 0; c < n; ++c) reference_collide<T>(f + 19 * c, omega[c], sigma, pfd + 6 * c, F + 3 * c, out + 19 * c); \
  }                                                                                                              \
  void ora_q19_step_##SUF(int32_t nocts, const int32_t* onbr, const oal_q19_params* P, const T* fin, T* fout,    \
                          const T* uin, T* vout, const T* rho_a, T* rhob) {                                      \
    Q19Level L{nocts, onbr};                                                                                     \
    step_level<T>(L, *P, fin, fout, uin, vout, rho_a, rhob);                                                     \
  }                                                                                                              \
  void ora_q19_initialise_##SUF(int64_t nslots, const uint8_t* kind, const T* rho, const T* u, const T* du,     \
                                double nu, T* f, T* u_out, T* rho_out) {                                         \
    initialise<T>(nslots, kind, rho, u, du, nu, f, u_out, rho_out);                                              \
  }                                                                                                              \
  void ora_q19_step_walls_##SUF(const oal_q19_level_desc* d, const oal_q19_params* P, const T* fin, T* fout,      \
                                const T* uin, T* vout, const T* rho_a, T* rhob, double* mom) {                   \
    step_level_walls<T>(*d, *P, fin, fout, uin, vout, rho_a, rhob, mom);                                         \
  }
ORA_Q19_COLLIDE(float, f32)
ORA_Q19_COLLIDE(double, f64)
#undef ORA_Q19_COLLIDE

}  // extern "C"
