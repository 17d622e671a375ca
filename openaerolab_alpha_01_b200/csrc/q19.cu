// q19.cu — the D3Q19 octree level step: recursive-regularised (RR/HRR) collision in closed form,
// pull streaming over 2x2x2 octs in Morton order, subgrid viscosity from the previous step's
// velocity, Guo body force and the positivity safeguard; FP32 or FP64.
//
// Reference (OpenAeroLab src/octree_q19, Julia, CPU):
//   velocity set and weights ........ src/octree_q19/src/lattice.jl:8-31
//   moments / Pi_neq / populations .. src/octree_q19/src/kernel.jl:26-91
//   collide_q19, below_floor ........ src/octree_q19/src/kernel.jl:92-134, :93-102
//   positivity safeguard ............ src/octree_q19/src/collision.jl:18-75
//   WALE / Smagorinsky / Vreman ..... src/octree_q19/src/collision.jl:77-127
//   level step (plain fluid slots) .. src/octree_q19/src/stream.jl:280-370, gradient :13-30
//   pull tables, neighbour slots .... src/octree_q19/src/octree.jl:139-159
//   rebuild (initial state) ......... src/octree_q19/src/coupling.jl:26-30, state.jl:267-305
//
// Data layout (the reference's own, so state moves in and out by plain copies):
//   f  (8, 19, nocts)  slot k of oct o, direction i at k + 8 i + 152 o (shifted populations f - w_i)
//   u  (8, 3, nocts)   k + 8 a + 24 o;   rho (8, nocts)  k + 8 o
//   onbr (27, nocts)   1-based neighbour oct of offset (dx,dy,dz) at (dx+1)+3(dy+1)+9(dz+1)
// One thread per slot, one CTA per 32 octs; the CTA stages its octs' neighbour rows in shared
// memory. The arithmetic is IEEE (no contraction: the library builds with -fmad=false; division
// and square root are the correctly rounded ones) in the reference's operation order, so a level
// steps to the same bits as the reference's scalar form.
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <unordered_map>

#include "../../include/oal.h"

oal_status oal_internal_set_error(oal_status s, const char* msg);

namespace {

constexpr int Q = 19;
constexpr int kOctsPerCta = 32;
constexpr int kThreads = 8 * kOctsPerCta;

// lattice.jl:8-11 (0-based)
__host__ __device__ constexpr int cx(int i) {
  return (i == 1 || i == 7 || i == 9 || i == 11 || i == 13) ? 1 : (i == 2 || i == 8 || i == 10 || i == 12 || i == 14) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int i) {
  return (i == 3 || i == 7 || i == 10 || i == 15 || i == 17) ? 1 : (i == 4 || i == 8 || i == 9 || i == 16 || i == 18) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int i) {
  return (i == 5 || i == 11 || i == 14 || i == 15 || i == 18) ? 1 : (i == 6 || i == 12 || i == 13 || i == 16 || i == 17) ? -1 : 0;
}
__host__ __device__ constexpr double wt(int i) { return i == 0 ? 1.0 / 3 : i < 7 ? 1.0 / 18 : 1.0 / 36; }

// ---- the cell arithmetic ---------------------------------------------------------------------

template <class T>
__device__ __forceinline__ void moments(const T* f, T& drho, T& mx, T& my, T& mz, T* P) {
  const T sx = f[1] + f[2], dx = f[1] - f[2];
  const T sy = f[3] + f[4], dy = f[3] - f[4];
  const T sz = f[5] + f[6], dz = f[5] - f[6];
  const T sxy = f[7] + f[8], dxy = f[7] - f[8];
  const T sxY = f[9] + f[10], dxY = f[9] - f[10];
  const T sxz = f[11] + f[12], dxz = f[11] - f[12];
  const T sxZ = f[13] + f[14], dxZ = f[13] - f[14];
  const T syz = f[15] + f[16], dyz = f[15] - f[16];
  const T syZ = f[17] + f[18], dyZ = f[17] - f[18];
  const T exy = sxy + sxY, exz = sxz + sxZ, eyz = syz + syZ;
  drho = (f[0] + ((sx + sy) + sz)) + ((exy + exz) + eyz);
  mx = dx + ((dxy + dxY) + (dxz + dxZ));
  my = dy + ((dxy - dxY) + (dyz + dyZ));
  mz = dz + ((dxz - dxZ) + (dyz - dyZ));
  P[0] = sx + (exy + exz);
  P[1] = sy + (exy + eyz);
  P[2] = sz + (exz + eyz);
  P[3] = sxy - sxY;
  P[4] = sxz - sxZ;
  P[5] = syz - syZ;
}

// populations of (1 + drho, u) with second-order non-equilibrium a2 scaled by `keep`
template <class T>
__device__ __forceinline__ void populations(T drho, T rho, T ux, T uy, T uz, const T* a2, T keep, T* out) {
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
    const T e = A + r45 * cu * cu + k2 * h2;
    const T o = r3 * cu + k3 * h3;
    a = w * (e + o);
    b = w * (e - o);
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
__device__ __forceinline__ bool below_floor(const T* out) {
  const T l0 = T(-(1 - 1e-6) / 3), l1 = T(-(1 - 1e-6) / 18), l2 = T(-(1 - 1e-6) / 36);
  bool bad = out[0] < l0;
#pragma unroll
  for (int i = 1; i < 7; ++i) bad = bad | (out[i] < l1);
#pragma unroll
  for (int i = 7; i < Q; ++i) bad = bad | (out[i] < l2);
  return bad;
}

template <class T>
__device__ __forceinline__ T feq_shifted(int i, T rho, T ux, T uy, T uz, T usq) {
  const T cu = T(cx(i)) * ux + T(cy(i)) * uy + T(cz(i)) * uz;
  return T(wt(i)) * rho * (T(1) + T(3) * cu + T(4.5) * cu * cu - T(1.5) * usq) - T(wt(i));
}

// blend toward `eq` until every population clears 1e-6 of its weight (collision.jl:23-40)
template <class T>
__device__ __noinline__ void positive_shifted(T* out, const T* eq) {
  T alpha = T(1);
  for (int i = 0; i < Q; ++i) {
    const T w = T(wt(i)), fl = T(1e-6) * w;
    const T actual = out[i] + w;
    if (actual < fl) {
      const T equilibrium = eq[i] + w;
      if (!(isfinite(equilibrium) && equilibrium > fl)) return;
      const T candidate = (equilibrium - fl) / (equilibrium - actual);
      alpha = candidate < alpha ? candidate : alpha;
    }
  }
  if (alpha < T(1)) {
    const T a99 = T(0.99) * alpha;
    const T safe_alpha = a99 > T(0) ? a99 : T(0);
    for (int i = 0; i < Q; ++i) out[i] = eq[i] + safe_alpha * (out[i] - eq[i]);
  }
}

// the safeguard of a forced collision: equilibrium of the post-force moments (collision.jl:45-56)
template <class T>
__device__ __noinline__ void limit_forced(T* out) {
  bool needs = false;
  for (int i = 0; i < Q; ++i) {
    const T w = T(wt(i));
    needs = needs | (out[i] + w < T(1e-6) * w);
  }
  if (!needs) return;
  T rho = T(1), mx = T(0), my = T(0), mz = T(0);
  for (int i = 0; i < Q; ++i) {
    rho += out[i];
    mx += T(cx(i)) * out[i];
    my += T(cy(i)) * out[i];
    mz += T(cz(i)) * out[i];
  }
  const T inv = T(1) / rho;
  const T ux = mx * inv, uy = my * inv, uz = mz * inv;
  const T usq = ux * ux + uy * uy + uz * uz;
  T eq[Q];
  for (int i = 0; i < Q; ++i) eq[i] = feq_shifted<T>(i, rho, ux, uy, uz, usq);
  positive_shifted<T>(out, eq);
}

template <class T>
__device__ __noinline__ void limit_unforced(T* out, T drho, T rho, T ux, T uy, T uz) {
  const T z[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  T eq[Q];
  populations<T>(drho, rho, ux, uy, uz, z, T(0), eq);
  positive_shifted<T>(out, eq);
}

// collide_q19 + limit_positive: `out` from the arriving `f`; returns rho, u
template <class T>
__device__ __forceinline__ void collide(const T* f, T omega, T sigma, const T* pfd, const T F0, const T F1, const T F2,
                                        bool forced, T* out, T& rho, T& ux, T& uy, T& uz) {
  T drho, mx, my, mz, P[6];
  moments<T>(f, drho, mx, my, mz, P);
  rho = drho + T(1);
  const T inv = T(1) / rho;
  const T hF = forced ? T(0.5) : T(0);
  ux = (mx + hF * F0) * inv;
  uy = (my + hF * F1) * inv;
  uz = (mz + hF * F2) * inv;
  T p[6];
  {
    const T d3 = drho * T(1.0 / 3.0);
    const T rx = rho * ux, ry = rho * uy, rz = rho * uz;
    p[0] = P[0] - d3 - rx * ux;
    p[1] = P[1] - d3 - ry * uy;
    p[2] = P[2] - d3 - rz * uz;
    p[3] = P[3] - rx * uy;
    p[4] = P[4] - rx * uz;
    p[5] = P[5] - ry * uz;
  }
  if (sigma != T(1)) {
    const T s1 = T(1) - sigma;
#pragma unroll
    for (int n = 0; n < 6; ++n) p[n] = sigma * p[n] + s1 * pfd[n];
  }
  populations<T>(drho, rho, ux, uy, uz, p, T(1) - omega, out);
  if (forced) {
    const T pre = T(1) - T(0.5) * omega;
    const T uF = ux * F0 + uy * F1 + uz * F2;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const T ci = T(cx(i)), cj = T(cy(i)), ck = T(cz(i));
      const T cu = ci * ux + cj * uy + ck * uz, cF = ci * F0 + cj * F1 + ck * F2;
      out[i] = out[i] + T(wt(i)) * (T(1.5) * cF + pre * (T(9) * cu * cF - T(3) * uF));
    }
  }
  if (below_floor<T>(out)) {
    if (forced) limit_forced<T>(out);
    else limit_unforced<T>(out, drho, rho, ux, uy, uz);
  }
}

template <class T>
__device__ __forceinline__ T nu_wale(const T* g, T cw) {
  const T g11 = g[0], g12 = g[1], g13 = g[2], g21 = g[3], g22 = g[4], g23 = g[5], g31 = g[6], g32 = g[7], g33 = g[8];
  const T s11 = g11, s22 = g22, s33 = g33;
  const T s12 = T(0.5) * (g12 + g21), s13 = T(0.5) * (g13 + g31), s23 = T(0.5) * (g23 + g32);
  const T q11 = g11 * g11 + g12 * g21 + g13 * g31, q12 = g11 * g12 + g12 * g22 + g13 * g32, q13 = g11 * g13 + g12 * g23 + g13 * g33;
  const T q21 = g21 * g11 + g22 * g21 + g23 * g31, q22 = g21 * g12 + g22 * g22 + g23 * g32, q23 = g21 * g13 + g22 * g23 + g23 * g33;
  const T q31 = g31 * g11 + g32 * g21 + g33 * g31, q32 = g31 * g12 + g32 * g22 + g33 * g32, q33 = g31 * g13 + g32 * g23 + g33 * g33;
  const T tr = (q11 + q22 + q33) / T(3);
  const T d11 = q11 - tr, d22 = q22 - tr, d33 = q33 - tr;
  const T d12 = T(0.5) * (q12 + q21), d13 = T(0.5) * (q13 + q31), d23 = T(0.5) * (q23 + q32);
  const T ss = s11 * s11 + s22 * s22 + s33 * s33 + T(2) * (s12 * s12 + s13 * s13 + s23 * s23);
  const T dd = d11 * d11 + d22 * d22 + d33 * d33 + T(2) * (d12 * d12 + d13 * d13 + d23 * d23);
  const T den = ss * ss * sqrt(ss) + dd * sqrt(sqrt(dd)) + T(1e-20);
  return cw * cw * dd * sqrt(dd) / den;
}
template <class T>
__device__ __forceinline__ T nu_smagorinsky(const T* g, T cs) {
  const T s12 = T(0.5) * (g[1] + g[3]), s13 = T(0.5) * (g[2] + g[6]), s23 = T(0.5) * (g[5] + g[7]);
  const T ss = g[0] * g[0] + g[4] * g[4] + g[8] * g[8] + T(2) * (s12 * s12 + s13 * s13 + s23 * s23);
  return cs * cs * sqrt(T(2) * ss);
}
template <class T>
__device__ __forceinline__ T nu_vreman(const T* g, T c) {
  const T g11 = g[0], g12 = g[1], g13 = g[2], g21 = g[3], g22 = g[4], g23 = g[5], g31 = g[6], g32 = g[7], g33 = g[8];
  const T b11 = g11 * g11 + g21 * g21 + g31 * g31, b22 = g12 * g12 + g22 * g22 + g32 * g32, b33 = g13 * g13 + g23 * g23 + g33 * g33;
  const T b12 = g11 * g12 + g21 * g22 + g31 * g32, b13 = g11 * g13 + g21 * g23 + g31 * g33, b23 = g12 * g13 + g22 * g23 + g32 * g33;
  const T bb = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
  const T aa = b11 + b22 + b33;
  const bool off = (aa <= T(1e-20)) | (bb <= T(0));
  return off ? T(0) : c * sqrt(bb / aa);
}

__device__ __forceinline__ int nbr_slot_index(int dx, int dy, int dz) { return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); }


// direction of velocity (x, y, z), 0-based (lattice.jl:15-25)
__host__ __device__ constexpr int dir_of(int x, int y, int z) {
  return (x == 0 && y == 0 && z == 0) ? 0
         : (x == 1 && y == 0 && z == 0) ? 1 : (x == -1 && y == 0 && z == 0) ? 2
         : (x == 0 && y == 1 && z == 0) ? 3 : (x == 0 && y == -1 && z == 0) ? 4
         : (x == 0 && y == 0 && z == 1) ? 5 : (x == 0 && y == 0 && z == -1) ? 6
         : (x == 1 && y == 1 && z == 0) ? 7 : (x == -1 && y == -1 && z == 0) ? 8
         : (x == 1 && y == -1 && z == 0) ? 9 : (x == -1 && y == 1 && z == 0) ? 10
         : (x == 1 && y == 0 && z == 1) ? 11 : (x == -1 && y == 0 && z == -1) ? 12
         : (x == 1 && y == 0 && z == -1) ? 13 : (x == -1 && y == 0 && z == 1) ? 14
         : (x == 0 && y == 1 && z == 1) ? 15 : (x == 0 && y == -1 && z == -1) ? 16
         : (x == 0 && y == 1 && z == -1) ? 17 : (x == 0 && y == -1 && z == 1) ? 18 : -1;
}
__host__ __device__ constexpr int opp(int i) { return dir_of(-cx(i), -cy(i), -cz(i)); }

enum : uint8_t { K_NONE = 0, K_FLUID = 1, K_SOLID = 2, K_COVERED = 3, K_GHOST = 4, K_BOUNDARY = 5 };

// ---- kernels -----------------------------------------------------------------------------------

template <class T>
struct LevelArgs {
  const T* fin;
  T* fout;
  const T* uin;
  T* uout;
  const T* rhoin;
  T* rhoout;
  const int32_t* onbr;  // (27, nocts) 1-based
  const int32_t* work;  // octs to step (null: octs 0 .. n_work-1)
  int32_t n_work;
  int32_t nocts;
  T nu, omega0, cw, cs, cv, sigma;
  T F0, F1, F2;
};

// the per-slot tables of a level with domain faces and cut links
template <class T>
struct WallArgs {
  const uint8_t* kind;      // (8, nocts)
  const uint8_t* face;      // (8, nocts)
  const uint32_t* special;  // (8, nocts)
  const int32_t* cutidx;    // (8, nocts) 1-based
  const float* qdir;        // (19, ncut)
  const uint8_t* okdir;     // (19, ncut)
  const int32_t* cut_off;   // (ncut + 1) 1-based
  const uint8_t* cut_dir;   // (nlinks) 1-based direction
  double* mom;              // (nlinks) momentum exchanged per link, or null
  double scale;
  int faces[6];
  T uin0, uin1, uin2;
};

// staged neighbour rows of the CTA's octs; returns the number of octs of this CTA
template <class T>
__device__ __forceinline__ int stage_octs(const LevelArgs<T>& a, int32_t* s_nb, int64_t* s_o) {
  const int64_t w0 = (int64_t)blockIdx.x * kOctsPerCta;
  const int64_t total = a.n_work;
  const int64_t left = total - w0;
  const int n_here = left < kOctsPerCta ? (int)left : kOctsPerCta;
  if (threadIdx.x < n_here) s_o[threadIdx.x] = a.work ? (int64_t)a.work[w0 + threadIdx.x] : w0 + threadIdx.x;
  __syncthreads();
  for (int t = threadIdx.x; t < n_here * 27; t += kThreads) s_nb[t] = a.onbr[s_o[t / 27] * 27 + t % 27] - 1;
  __syncthreads();
  return n_here;
}

// central differences of the previous step's velocity over the 6 face neighbours (stream.jl:13-30);
// WALLS: a missing or domain-boundary neighbour contributes the slot's own velocity
template <class T, bool WALLS>
__device__ __forceinline__ void velocity_gradient(const LevelArgs<T>& a, const uint8_t* kind, const int32_t* nb, int64_t o,
                                                  int k, T* g) {
  const int x = k & 1, y = (k >> 1) & 1, z = (k >> 2) & 1;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    T vp[3], vm[3];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int d = s == 0 ? 1 : -1;
      const int nx = x + (ax == 0 ? d : 0), ny = y + (ax == 1 ? d : 0), nz = z + (ax == 2 ? d : 0);
      const int ox = nx < 0 ? -1 : (nx > 1 ? 1 : 0), oy = ny < 0 ? -1 : (ny > 1 ? 1 : 0), oz = nz < 0 ? -1 : (nz > 1 ? 1 : 0);
      int64_t no = nb[nbr_slot_index(ox, oy, oz)];
      int nk = (nx - 2 * ox) + 2 * (ny - 2 * oy) + 4 * (nz - 2 * oz);
      if (WALLS && (no < 0 || kind[no * 8 + nk] == K_BOUNDARY)) {
        no = o;
        nk = k;
      }
      T* v = s == 0 ? vp : vm;
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = __ldg(a.uin + no * 24 + 8 * c + nk);
    }
    const T h = T(0.5);
#pragma unroll
    for (int c = 0; c < 3; ++c) g[3 * ax + c] = h * (vp[c] - vm[c]);
  }
}

// subgrid viscosity, omega and the HRR stress of slot (k, o) (stream.jl:357-360)
template <class T, int SGS, bool GRAD, bool WALLS>
__device__ __forceinline__ T relaxation(const LevelArgs<T>& a, const uint8_t* kind, const int32_t* nb, int64_t o, int k,
                                        T* pfd) {
#pragma unroll
  for (int n = 0; n < 6; ++n) pfd[n] = T(0);
  if (!GRAD) return a.omega0;
  T g[9];
  velocity_gradient<T, WALLS>(a, kind, nb, o, k, g);
  T nut = T(0);
  if (SGS == 1) nut = nu_wale<T>(g, a.cw);
  if (SGS == 2) nut = nu_smagorinsky<T>(g, a.cs);
  if (SGS == 3) nut = nu_vreman<T>(g, a.cv);
  const T omega = T(1) / (T(3) * (a.nu + nut) + T(0.5));
  if (a.sigma != T(1)) {
    const T rho_prev = a.rhoin[o * 8 + k];
    const T tau = T(1) / omega;
    const T c = -rho_prev * tau / T(3);
    pfd[0] = c * T(2) * g[0];
    pfd[1] = c * T(2) * g[4];
    pfd[2] = c * T(2) * g[8];
    pfd[3] = c * (g[1] + g[3]);
    pfd[4] = c * (g[2] + g[6]);
    pfd[5] = c * (g[5] + g[7]);
  }
  return omega;
}

template <class T>
__device__ __forceinline__ void store_cell(const LevelArgs<T>& a, int64_t o, int k, const T* out, T rho, T ux, T uy, T uz) {
  T* fo = a.fout + o * (8 * Q) + k;
#pragma unroll
  for (int i = 0; i < Q; ++i) fo[8 * i] = out[i];
  T* uo = a.uout + o * 24 + k;
  uo[0] = ux;
  uo[8] = uy;
  uo[16] = uz;
  a.rhoout[o * 8 + k] = rho;
}

// octs whose eight slots are plain fluid cells (every pull source is a fluid slot)
// SGS: 0 none, 1 WALE, 2 Smagorinsky, 3 Vreman; GRAD: the velocity gradient is needed (SGS or HRR)
template <class T, int SGS, bool GRAD, bool FORCED>
__global__ void __launch_bounds__(kThreads) k_q19_step(const LevelArgs<T> a) {
  __shared__ int32_t s_nb[kOctsPerCta * 27];
  __shared__ int64_t s_o[kOctsPerCta];
  const int n_here = stage_octs<T>(a, s_nb, s_o);
  const int lo = threadIdx.x >> 3, k = threadIdx.x & 7;
  if (lo >= n_here) return;
  const int64_t o = s_o[lo];
  const int32_t* nb = s_nb + 27 * lo;
  const int x = k & 1, y = (k >> 1) & 1, z = (k >> 2) & 1;

  // pull: slot k takes direction i from slot (x,y,z) - c_i, in this oct or a neighbour (octree.jl:139-150)
  T f[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const int px = x - cx(i), py = y - cy(i), pz = z - cz(i);
    const int ox = px < 0 ? -1 : (px > 1 ? 1 : 0), oy = py < 0 ? -1 : (py > 1 ? 1 : 0), oz = pz < 0 ? -1 : (pz > 1 ? 1 : 0);
    const int src = nb[nbr_slot_index(ox, oy, oz)];
    const int child = (px - 2 * ox) + 2 * (py - 2 * oy) + 4 * (pz - 2 * oz);
    f[i] = __ldg(a.fin + (int64_t)src * (8 * Q) + 8 * i + child);
  }
  T pfd[6];
  const T omega = relaxation<T, SGS, GRAD, false>(a, nullptr, nb, o, k, pfd);
  T out[Q], rho, ux, uy, uz;
  collide<T>(f, omega, a.sigma, pfd, a.F0, a.F1, a.F2, FORCED, out, rho, ux, uy, uz);
  store_cell<T>(a, o, k, out, rho, ux, uy, uz);
}

// fo[m] for a runtime m by selects (keeps the populations in registers)
template <class T>
__device__ __forceinline__ T select_dir(const T* fo, int m) {
  T v = fo[0];
#pragma unroll
  for (int t = 1; t < Q; ++t) v = m == t ? fo[t] : v;
  return v;
}

// the population j arriving from a domain-boundary slot with face mask `mask` (stream.jl:32-78)
template <class T>
__device__ __forceinline__ T face_population(const WallArgs<T>& w, uint32_t mask, int j, const T* fo, T rho, T ux, T uy,
                                             T uz) {
  const int i = opp(j);
  auto feq_s = [](int d, T r, T vx, T vy, T vz, T vsq) { return feq_shifted<T>(d, r, vx, vy, vz, vsq); };
  auto dirichlet = [&](int cond) {
    const T usq = ux * ux + uy * uy + uz * uz;
    const T own = fo[i] - feq_s(i, rho, ux, uy, uz, usq);
    if (cond == OAL_Q19_FACE_INLET) {
      const T vsq = w.uin0 * w.uin0 + w.uin1 * w.uin1 + w.uin2 * w.uin2;
      return feq_s(j, rho, w.uin0, w.uin1, w.uin2, vsq) + own;
    }
    if (cond == OAL_Q19_FACE_OUTLET) return feq_s(j, T(1), ux, uy, uz, usq) + own;
    const T vsq = w.uin0 * w.uin0 + w.uin1 * w.uin1 + w.uin2 * w.uin2;
    return feq_s(j, T(1), w.uin0, w.uin1, w.uin2, vsq) + own;
  };
  auto mirror = [&](int d, int axis) {
    return dir_of(axis == 0 ? -cx(d) : cx(d), axis == 1 ? -cy(d) : cy(d), axis == 2 ? -cz(d) : cz(d));
  };
  if (__popc(mask) == 1) {
    const int f = __ffs(mask) - 1;
    const int cond = w.faces[f];
    if (cond == OAL_Q19_FACE_NOSLIP || cond == OAL_Q19_FACE_GROUND) return fo[i];
    if (cond == OAL_Q19_FACE_SLIP || cond == OAL_Q19_FACE_SYMMETRY) return select_dir<T>(fo, mirror(j, f >> 1));
    return dirichlet(cond);
  }
  bool wall = false, open = false;
  for (int f = 0; f < 6; ++f) {
    if (!((mask >> f) & 1u)) continue;
    const int c = w.faces[f];
    wall = wall || c == OAL_Q19_FACE_NOSLIP || c == OAL_Q19_FACE_GROUND;
    open = open || c == OAL_Q19_FACE_INLET || c == OAL_Q19_FACE_OUTLET || c == OAL_Q19_FACE_FREESTREAM;
  }
  if (wall) return fo[i];
  if (open) return dirichlet(OAL_Q19_FACE_FREESTREAM);
  int m = j;
  if (mask & 0x03u) m = mirror(m, 0);
  if (mask & 0x0cu) m = mirror(m, 1);
  if (mask & 0x30u) m = mirror(m, 2);
  return select_dir<T>(fo, m);
}

// octs with a non-fluid slot or a special direction: fluid slots step with the face conditions, the
// Bouzidi rule on cut links and the momentum exchange (stream.jl:205-257)
template <class T, int SGS, bool GRAD, bool FORCED>
__global__ void __launch_bounds__(kThreads) k_q19_walls(const LevelArgs<T> a, const WallArgs<T> w) {
  __shared__ int32_t s_nb[kOctsPerCta * 27];
  __shared__ int64_t s_o[kOctsPerCta];
  const int n_here = stage_octs<T>(a, s_nb, s_o);
  const int lo = threadIdx.x >> 3, k = threadIdx.x & 7;
  if (lo >= n_here) return;
  const int64_t o = s_o[lo];
  const int64_t s = o * 8 + k;
  if (w.kind[s] != K_FLUID) return;
  const int32_t* nb = s_nb + 27 * lo;
  const int x = k & 1, y = (k >> 1) & 1, z = (k >> 2) & 1;
  const uint32_t sp = w.special[s];
  T f[Q];
  auto pull = [&](int i, int& src, int& child) {
    const int px = x - cx(i), py = y - cy(i), pz = z - cz(i);
    const int ox = px < 0 ? -1 : (px > 1 ? 1 : 0), oy = py < 0 ? -1 : (py > 1 ? 1 : 0), oz = pz < 0 ? -1 : (pz > 1 ? 1 : 0);
    src = nb[nbr_slot_index(ox, oy, oz)];
    child = (px - 2 * ox) + 2 * (py - 2 * oy) + 4 * (pz - 2 * oz);
  };
  if (sp == 0) {
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      int src, child;
      pull(i, src, child);
      f[i] = __ldg(a.fin + (int64_t)src * (8 * Q) + 8 * i + child);
    }
  } else {
    T fo[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) fo[i] = a.fin[o * (8 * Q) + 8 * i + k];
    const T rho0 = a.rhoin[s], ux0 = a.uin[o * 24 + k], uy0 = a.uin[o * 24 + 8 + k], uz0 = a.uin[o * 24 + 16 + k];
    const int ci = w.cutidx[s] - 1;
#pragma unroll
    for (int j = 0; j < Q; ++j) {
      int src, child;
      pull(j, src, child);
      if (!((sp >> j) & 1u)) {
        f[j] = __ldg(a.fin + (int64_t)src * (8 * Q) + 8 * j + child);
      } else if (src >= 0 && w.kind[(int64_t)src * 8 + child] == K_BOUNDARY) {
        f[j] = face_population<T>(w, w.face[(int64_t)src * 8 + child], j, fo, rho0, ux0, uy0, uz0);
      } else {
        // the link opposite to j is cut: Bouzidi from the own populations and the partner x - c_i
        const int i = opp(j);
        const T q = T(w.qdir[(int64_t)ci * Q + i]);
        if (!w.okdir[(int64_t)ci * Q + i]) {
          f[j] = fo[i];
        } else if (q < T(0.5)) {
          int po, pk;
          {
            const int px = x - cx(i), py = y - cy(i), pz = z - cz(i);
            const int ox = px < 0 ? -1 : (px > 1 ? 1 : 0), oy = py < 0 ? -1 : (py > 1 ? 1 : 0), oz = pz < 0 ? -1 : (pz > 1 ? 1 : 0);
            po = nb[nbr_slot_index(ox, oy, oz)];
            pk = (px - 2 * ox) + 2 * (py - 2 * oy) + 4 * (pz - 2 * oz);
          }
          f[j] = T(2) * q * fo[i] + (T(1) - T(2) * q) * a.fin[(int64_t)po * (8 * Q) + 8 * i + pk];
        } else {
          const T inv2q = T(1) / (T(2) * q);
          f[j] = inv2q * fo[i] + (T(1) - inv2q) * fo[j];
        }
      }
    }
    if (w.mom && ci >= 0) {
      // momentum exchange on the cut links: (f_i* + f_j(t+1)) c_i per link, i toward the wall; a cut
      // cell's links are in direction order (checked at level creation)
      int li = w.cut_off[ci] - 1;
      const int end = w.cut_off[ci + 1] - 1;
#pragma unroll
      for (int i = 1; i < Q; ++i) {
        if (li < end && w.cut_dir[li] - 1 == i) {
          w.mom[li] += w.scale * (double)(fo[i] + f[opp(i)]);
          ++li;
        }
      }
    }
  }
  T pfd[6];
  const T omega = relaxation<T, SGS, GRAD, true>(a, w.kind, nb, o, k, pfd);
  T out[Q], rho, ux, uy, uz;
  collide<T>(f, omega, a.sigma, pfd, a.F0, a.F1, a.F2, FORCED, out, rho, ux, uy, uz);
  store_cell<T>(a, o, k, out, rho, ux, uy, uz);
}

// per-triangle force: the triangle's links in ascending order (the reference's accumulator bins)
__global__ void k_q19_tri_forces(int32_t ntri, const int32_t* __restrict__ tri_off, const int32_t* __restrict__ tri_links,
                                 const uint8_t* __restrict__ cut_dir, const double* __restrict__ mom,
                                 double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  double fx = 0, fy = 0, fz = 0;
  for (int n = tri_off[t]; n < tri_off[t + 1]; ++n) {
    const int li = tri_links[n];
    const int i = cut_dir[li] - 1;
    const double m = mom[li];
    fx += m * cx(i);
    fy += m * cy(i);
    fz += m * cz(i);
  }
  out[3 * (int64_t)t] = fx;
  out[3 * (int64_t)t + 1] = fy;
  out[3 * (int64_t)t + 2] = fz;
}

// fixed-order sum of the per-triangle forces: strided per thread, then a fixed tree
__global__ void k_q19_force_total(int32_t ntri, const double* __restrict__ per_tri, double* __restrict__ total) {
  __shared__ double s[3][256];
  const int t = threadIdx.x;
  double a0 = 0, a1 = 0, a2 = 0;
  for (int i = t; i < ntri; i += 256) {
    a0 += per_tri[3 * (int64_t)i];
    a1 += per_tri[3 * (int64_t)i + 1];
    a2 += per_tri[3 * (int64_t)i + 2];
  }
  s[0][t] = a0;
  s[1][t] = a1;
  s[2][t] = a2;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h)
      for (int c = 0; c < 3; ++c) s[c][t] += s[c][t + h];
    __syncthreads();
  }
  if (t < 3) total[t] = s[t][0];
}

// initial state of the fluid, ghost and covered slots from (rho, u[, du]): `rebuild` with the
// Chapman-Enskog non-equilibrium, or the equilibrium when du is null (state.jl:267-305,
// coupling.jl:26-30); the other slots keep the allocation state (f = 0, u = 0, rho = 1)
template <class T>
__global__ void k_q19_initialise(int64_t nslots, const uint8_t* __restrict__ kind, const T* __restrict__ rho_in,
                                 const T* __restrict__ u_in, const T* __restrict__ du, T nu, T* __restrict__ fa,
                                 T* __restrict__ fb, T* __restrict__ ua, T* __restrict__ ub, T* __restrict__ ra,
                                 T* __restrict__ rb) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  const int64_t o = s >> 3;
  const int k = (int)(s & 7);
  const bool fluid = !kind || kind[s] == K_FLUID || kind[s] == K_GHOST || kind[s] == K_COVERED;
  T out[Q];
  T rho = T(1), ux = T(0), uy = T(0), uz = T(0);
  if (fluid) {
    rho = rho_in[s];
    ux = u_in[o * 24 + k];
    uy = u_in[o * 24 + 8 + k];
    uz = u_in[o * 24 + 16 + k];
    const T drho = rho - T(1);
    const T omega = T(1) / (T(3) * nu + T(0.5));
    if (du) {
      T d[9];
#pragma unroll
      for (int n = 0; n < 9; ++n) d[n] = du[o * 72 + 8 * n + k];
      const T tau = T(1) / omega;
      const T c = -rho * tau / T(3);
      const T pn[6] = {c * T(2) * d[0], c * T(2) * d[4], c * T(2) * d[8], c * (d[1] + d[3]), c * (d[2] + d[6]), c * (d[5] + d[7])};
      populations<T>(drho, rho, ux, uy, uz, pn, T(1) - omega, out);
      if (below_floor<T>(out)) limit_unforced<T>(out, drho, rho, ux, uy, uz);
    } else {
      const T zz[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
      populations<T>(drho, rho, ux, uy, uz, zz, T(0), out);
    }
  } else {
#pragma unroll
    for (int i = 0; i < Q; ++i) out[i] = T(0);
  }
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    fa[o * (8 * Q) + 8 * i + k] = out[i];
    fb[o * (8 * Q) + 8 * i + k] = out[i];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T v = c == 0 ? ux : c == 1 ? uy : uz;
    ua[o * 24 + 8 * c + k] = v;
    ub[o * 24 + 8 * c + k] = v;
  }
  ra[s] = rho;
  rb[s] = rho;
}

// the collision alone over n cells in (n, 19) rows (a test hook of the known-answer checks)
template <class T>
__global__ void k_q19_collide_cells(int64_t n, const T* __restrict__ f, const T* __restrict__ omega, T sigma,
                                    const T* __restrict__ pfd, const T* __restrict__ F, T* __restrict__ out,
                                    T* __restrict__ rho, T* __restrict__ u) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  T fl[Q], o[Q], pf[6];
  for (int i = 0; i < Q; ++i) fl[i] = f[c * Q + i];
  for (int i = 0; i < 6; ++i) pf[i] = pfd[c * 6 + i];
  const T F0 = F[3 * c], F1 = F[3 * c + 1], F2 = F[3 * c + 2];
  const bool forced = !(F0 == T(0) && F1 == T(0) && F2 == T(0));
  T r, ux, uy, uz;
  collide<T>(fl, omega[c], sigma, pf, F0, F1, F2, forced, o, r, ux, uy, uz);
  for (int i = 0; i < Q; ++i) out[c * Q + i] = o[i];
  rho[c] = r;
  u[3 * c] = ux;
  u[3 * c + 1] = uy;
  u[3 * c + 2] = uz;
}

// FP64 totals per CTA over the fluid slots: mass, momentum, kinetic energy (state.jl:333-356)
template <class T>
__global__ void k_q19_totals(int64_t nslots, const uint8_t* __restrict__ kind, const T* __restrict__ rho,
                             const T* __restrict__ u, double* __restrict__ part) {
  __shared__ double s[5][8];
  double a[5] = {0, 0, 0, 0, 0};
  for (int64_t sl = (int64_t)blockIdx.x * 256 + threadIdx.x; sl < nslots; sl += (int64_t)gridDim.x * 256) {
    if (kind && kind[sl] != K_FLUID) continue;
    const int64_t o = sl >> 3;
    const int k = (int)(sl & 7);
    const double r = (double)rho[sl];
    const double ux = (double)u[o * 24 + k], uy = (double)u[o * 24 + 8 + k], uz = (double)u[o * 24 + 16 + k];
    a[0] += r;
    a[1] += r * ux;
    a[2] += r * uy;
    a[3] += r * uz;
    a[4] += 0.5 * r * (ux * ux + uy * uy + uz * uz);
  }
#pragma unroll
  for (int c = 0; c < 5; ++c)
    for (int off = 16; off > 0; off >>= 1) a[c] += __shfl_down_sync(0xffffffffu, a[c], off);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 5; ++c) s[c][threadIdx.x >> 5] = a[c];
  __syncthreads();
  if (threadIdx.x < 5) {
    double v = 0;
    for (int w = 0; w < 8; ++w) v += s[threadIdx.x][w];
    part[5 * (int64_t)blockIdx.x + threadIdx.x] = v;
  }
}

__global__ void k_q19_totals_final(const double* __restrict__ part, int n, double* __restrict__ out) {
  if (threadIdx.x < 5) {
    double v = 0;
    for (int b = 0; b < n; ++b) v += part[5 * b + threadIdx.x];
    out[threadIdx.x] = v;
  }
}

template <class T>
__global__ void k_fill(T* p, int64_t n, T v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

constexpr int kTotalsCtas = 592;  // 4 per SM on 148 SMs

oal_status fail(oal_status s, const char* fmt, ...) {
  char buf[400];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return oal_internal_set_error(s, buf);
}

#define Q19_TRY(expr)                                                                                 \
  do {                                                                                                \
    cudaError_t _e = (expr);                                                                          \
    if (_e != cudaSuccess) {                                                                          \
      cudaGetLastError();                                                                             \
      return fail(_e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "%s: %s", #expr, \
                  cudaGetErrorString(_e));                                                            \
    }                                                                                                 \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Morton key of an oct origin in oct units (octree.jl:35-48)
uint64_t spread3(uint64_t v) {
  v &= 0x1fffff;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}
uint64_t morton3(uint64_t ix, uint64_t iy, uint64_t iz) { return spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2); }

template <class X>
cudaError_t upload(X** dst, const X* src, size_t n) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc(dst, sizeof(X) * n);
  if (e == cudaSuccess) e = cudaMemcpy(*dst, src, sizeof(X) * n, cudaMemcpyHostToDevice);
  return e;
}

}  // namespace

struct oal_q19_level {
  int device = 0;
  int precision = OAL_STORE_F32;
  int32_t nocts = 0;
  size_t es = 4;
  int32_t* onbr = nullptr;
  void* f[2] = {nullptr, nullptr};
  void* u[2] = {nullptr, nullptr};
  void* rho[2] = {nullptr, nullptr};
  double* part = nullptr;  // kTotalsCtas * 5 + 5
  int cur = 0;             // buffer holding the current state
  int64_t steps = 0;
  // levels with faces / cut links
  bool walls = false;
  uint8_t* kind = nullptr;
  uint8_t* face = nullptr;
  uint32_t* special = nullptr;
  int32_t* cutidx = nullptr;
  float* qdir = nullptr;
  uint8_t* okdir = nullptr;
  int32_t* cut_off = nullptr;
  uint8_t* cut_dir = nullptr;
  double* mom = nullptr;
  int32_t* tri_off = nullptr;
  int32_t* tri_links = nullptr;
  double* tri_force = nullptr;  // (ntri, 3) then the total (3)
  int32_t* work_plain = nullptr;
  int32_t* work_walls = nullptr;
  int32_t n_plain = 0, n_walls = 0, ncut = 0, nlinks = 0, ntri = 0;
  int faces[6] = {0, 0, 0, 0, 0, 0};
  bool forces_valid = false;
  // the wall octs step on a side stream beside the plain octs (both read the current buffer and
  // write disjoint octs of the other): a fork and a join event around the two launches
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

namespace {

oal_status check_params(const oal_q19_params* p) {
  if (!p) return fail(OAL_E_INVALID_ARG, "null oal_q19_params");
  if (p->abi_version != OAL_ABI_VERSION)
    return fail(OAL_E_ABI_MISMATCH, "oal_q19_params.abi_version %u != %d", p->abi_version, OAL_ABI_VERSION);
  if (!(p->nu > 0) || !std::isfinite(p->nu)) return fail(OAL_E_INVALID_ARG, "nu must be positive (got %g)", p->nu);
  if (p->sgs < OAL_Q19_SGS_NONE || p->sgs > OAL_Q19_SGS_VREMAN) return fail(OAL_E_INVALID_ARG, "sgs model %d", p->sgs);
  if (!(p->hrr_sigma >= 0 && p->hrr_sigma <= 1)) return fail(OAL_E_INVALID_ARG, "hrr_sigma must lie in [0, 1]");
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(p->body_force[a]) || !std::isfinite(p->u_inlet[a]))
      return fail(OAL_E_INVALID_ARG, "body_force and u_inlet must be finite");
  if (!std::isfinite(p->force_scale)) return fail(OAL_E_INVALID_ARG, "force_scale must be finite");
  return OAL_OK;
}

template <class T>
LevelArgs<T> level_args(oal_q19_level* L, const oal_q19_params* p) {
  LevelArgs<T> a;
  const int src = L->cur, dst = 1 - L->cur;
  a.fin = static_cast<const T*>(L->f[src]);
  a.fout = static_cast<T*>(L->f[dst]);
  a.uin = static_cast<const T*>(L->u[src]);
  a.uout = static_cast<T*>(L->u[dst]);
  a.rhoin = static_cast<const T*>(L->rho[src]);
  a.rhoout = static_cast<T*>(L->rho[dst]);
  a.onbr = L->onbr;
  a.work = L->walls ? L->work_plain : nullptr;
  a.n_work = L->walls ? L->n_plain : L->nocts;
  a.nocts = L->nocts;
  a.nu = T(p->nu);
  a.omega0 = T(1) / (T(3) * a.nu + T(0.5));
  a.cw = T(p->c_wale);
  a.cs = T(p->c_smagorinsky);
  a.cv = T(2.5 * p->c_smagorinsky * p->c_smagorinsky);
  a.sigma = T(p->hrr_sigma);
  a.F0 = T(p->body_force[0]);
  a.F1 = T(p->body_force[1]);
  a.F2 = T(p->body_force[2]);
  return a;
}

template <class T, int SGS, bool GRAD>
cudaError_t launch3(const LevelArgs<T>& a, const WallArgs<T>* w, bool forced, cudaStream_t st) {
  const int64_t n = a.n_work;
  if (n > 0) {
    const unsigned grid = (unsigned)((n + kOctsPerCta - 1) / kOctsPerCta);
    if (forced) k_q19_step<T, SGS, GRAD, true><<<grid, kThreads, 0, st>>>(a);
    else k_q19_step<T, SGS, GRAD, false><<<grid, kThreads, 0, st>>>(a);
  }
  (void)w;
  return cudaGetLastError();
}

template <class T, int SGS, bool GRAD>
cudaError_t launch_walls3(const LevelArgs<T>& a, const WallArgs<T>& w, bool forced, cudaStream_t st) {
  if (a.n_work <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((a.n_work + kOctsPerCta - 1) / kOctsPerCta);
  if (forced) k_q19_walls<T, SGS, GRAD, true><<<grid, kThreads, 0, st>>>(a, w);
  else k_q19_walls<T, SGS, GRAD, false><<<grid, kThreads, 0, st>>>(a, w);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_step(const LevelArgs<T>& a, int sgs, bool forced, cudaStream_t st) {
  const bool hrr = a.sigma != T(1);
  switch (sgs) {
    case OAL_Q19_SGS_WALE: return launch3<T, 1, true>(a, nullptr, forced, st);
    case OAL_Q19_SGS_SMAGORINSKY: return launch3<T, 2, true>(a, nullptr, forced, st);
    case OAL_Q19_SGS_VREMAN: return launch3<T, 3, true>(a, nullptr, forced, st);
    default: return hrr ? launch3<T, 0, true>(a, nullptr, forced, st) : launch3<T, 0, false>(a, nullptr, forced, st);
  }
}

template <class T>
cudaError_t launch_walls(const LevelArgs<T>& a, const WallArgs<T>& w, int sgs, bool forced, cudaStream_t st) {
  const bool hrr = a.sigma != T(1);
  switch (sgs) {
    case OAL_Q19_SGS_WALE: return launch_walls3<T, 1, true>(a, w, forced, st);
    case OAL_Q19_SGS_SMAGORINSKY: return launch_walls3<T, 2, true>(a, w, forced, st);
    case OAL_Q19_SGS_VREMAN: return launch_walls3<T, 3, true>(a, w, forced, st);
    default: return hrr ? launch_walls3<T, 0, true>(a, w, forced, st) : launch_walls3<T, 0, false>(a, w, forced, st);
  }
}

// one step of a level (step_level! + swap_buffers!); with `collect` the momentum exchange of its
// cut links is added to the per-link accumulator
template <class T>
cudaError_t step_level_t(oal_q19_level* L, const oal_q19_params* p, bool collect, cudaStream_t st) {
  const bool forced = !(T(p->body_force[0]) == T(0) && T(p->body_force[1]) == T(0) && T(p->body_force[2]) == T(0));
  const LevelArgs<T> a = level_args<T>(L, p);
  // with a side stream the wall octs run beside the plain ones (fork before, join after)
  const bool fork = L->walls && L->side != nullptr;
  cudaError_t e = cudaSuccess;
  if (fork) {
    e = cudaEventRecord(L->fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(L->side, L->fork, 0);
  }
  if (e == cudaSuccess) e = launch_step<T>(a, p->sgs, forced, st);
  if (e == cudaSuccess && L->walls) {
    LevelArgs<T> b = a;
    b.work = L->work_walls;
    b.n_work = L->n_walls;
    WallArgs<T> w;
    w.kind = L->kind;
    w.face = L->face;
    w.special = L->special;
    w.cutidx = L->cutidx;
    w.qdir = L->qdir;
    w.okdir = L->okdir;
    w.cut_off = L->cut_off;
    w.cut_dir = L->cut_dir;
    w.mom = (collect && L->nlinks > 0) ? L->mom : nullptr;
    w.scale = p->force_scale;
    for (int f = 0; f < 6; ++f) w.faces[f] = L->faces[f];
    w.uin0 = T(p->u_inlet[0]);
    w.uin1 = T(p->u_inlet[1]);
    w.uin2 = T(p->u_inlet[2]);
    e = launch_walls<T>(b, w, p->sgs, forced, fork ? L->side : st);
    if (fork && e == cudaSuccess) e = cudaEventRecord(L->join, L->side);
    if (fork && e == cudaSuccess) e = cudaStreamWaitEvent(st, L->join, 0);
  }
  L->cur = 1 - L->cur;
  ++L->steps;
  return e;
}

// per-triangle and total force of a level from its per-link accumulator
cudaError_t level_forces(oal_q19_level* L, cudaStream_t st) {
  if (!L->walls) return cudaSuccess;
  if (L->nlinks > 0)
    k_q19_tri_forces<<<(L->ntri + 127) / 128, 128, 0, st>>>(L->ntri, L->tri_off, L->tri_links, L->cut_dir, L->mom,
                                                           L->tri_force);
  else
    cudaMemsetAsync(L->tri_force, 0, sizeof(double) * 3 * (size_t)L->ntri, st);
  k_q19_force_total<<<1, 256, 0, st>>>(L->ntri, L->tri_force, L->tri_force + 3 * (int64_t)L->ntri);
  L->forces_valid = true;
  return cudaGetLastError();
}

template <class T>
oal_status advance_t(oal_q19_level* L, const oal_q19_params* p, int32_t n, bool collect, cudaStream_t st) {
  for (int32_t s = 0; s < n; ++s) {
    const bool last = s == n - 1;
    if (collect && last && L->walls && L->nlinks > 0)
      Q19_TRY(cudaMemsetAsync(L->mom, 0, sizeof(double) * L->nlinks, st));
    Q19_TRY(step_level_t<T>(L, p, collect && last, st));
    if (collect && last) Q19_TRY(level_forces(L, st));
  }
  return OAL_OK;
}

oal_status alloc_state(oal_q19_level* L) {
  const size_t ns = (size_t)L->nocts * 8;
  cudaError_t e = cudaSuccess;
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    e = cudaMalloc(&L->f[b], L->es * ns * Q);
    if (e == cudaSuccess) e = cudaMalloc(&L->u[b], L->es * ns * 3);
    if (e == cudaSuccess) e = cudaMalloc(&L->rho[b], L->es * ns);
    // the allocation state of the reference: f = 0, u = 0, rho = 1 (state.jl:217-232)
    if (e == cudaSuccess) e = cudaMemset(L->f[b], 0, L->es * ns * Q);
    if (e == cudaSuccess) e = cudaMemset(L->u[b], 0, L->es * ns * 3);
    if (e == cudaSuccess) {
      const unsigned grid = (unsigned)((ns + 255) / 256);
      if (L->precision == OAL_STORE_F64) k_fill<double><<<grid, 256>>>((double*)L->rho[b], (int64_t)ns, 1.0);
      else k_fill<float><<<grid, 256>>>((float*)L->rho[b], (int64_t)ns, 1.0f);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&L->part, sizeof(double) * (kTotalsCtas * 5 + 5));
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "level allocation: %s",
                cudaGetErrorString(e));
  }
  return OAL_OK;
}

oal_status check_device(int32_t device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(OAL_E_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return fail(OAL_E_INVALID_ARG, "device %d of %d", device, ndev);
  return OAL_OK;
}

}  // namespace

static oal_status create_desc_impl(int32_t device, int32_t precision, const oal_q19_level_desc* d, bool transfers,
                                   oal_q19_level** out);

extern "C" {

oal_status oal_q19_default_params(oal_q19_params* p) {
  if (!p) return fail(OAL_E_INVALID_ARG, "null argument");
  std::memset(p, 0, sizeof *p);
  p->abi_version = OAL_ABI_VERSION;
  p->sgs = OAL_Q19_SGS_NONE;
  p->nu = 0.01;
  p->c_wale = 0.5;          // config.jl Numerics defaults
  p->c_smagorinsky = 0.1;
  p->hrr_sigma = 1.0;
  p->force_scale = 1.0;
  return OAL_OK;
}

oal_status oal_q19_periodic_box(int32_t n0, int32_t n1, int32_t n2, int32_t* origin, int32_t* onbr) {
  if (n0 < 2 || n1 < 2 || n2 < 2 || (n0 | n1 | n2) & 1)
    return fail(OAL_E_INVALID_ARG, "a periodic box needs even cell counts >= 2 per axis (got %d %d %d)", n0, n1, n2);
  if (!origin || !onbr) return fail(OAL_E_INVALID_ARG, "null output");
  const int m0 = n0 / 2, m1 = n1 / 2, m2 = n2 / 2;
  if ((int64_t)m0 * m1 * m2 > INT32_MAX / 27) return fail(OAL_E_TOO_LARGE, "too many octs");
  const int64_t no = (int64_t)m0 * m1 * m2;
  std::vector<std::pair<uint64_t, int64_t>> keys((size_t)no);
  for (int i = 0; i < m0; ++i)
    for (int j = 0; j < m1; ++j)
      for (int k = 0; k < m2; ++k) {
        const int64_t lin = ((int64_t)i * m1 + j) * m2 + k;
        keys[(size_t)lin] = {morton3(i + 1, j + 1, k + 1), lin};
      }
  std::sort(keys.begin(), keys.end());
  std::vector<int32_t> index((size_t)no);
  for (int64_t o = 0; o < no; ++o) index[(size_t)keys[(size_t)o].second] = (int32_t)o;
  for (int64_t o = 0; o < no; ++o) {
    const int64_t lin = keys[(size_t)o].second;
    const int i = (int)(lin / ((int64_t)m1 * m2)), j = (int)((lin / m2) % m1), k = (int)(lin % m2);
    origin[3 * o] = 2 * i;
    origin[3 * o + 1] = 2 * j;
    origin[3 * o + 2] = 2 * k;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int a = (i + dx + m0) % m0, b = (j + dy + m1) % m1, c = (k + dz + m2) % m2;
          onbr[27 * o + (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)] = index[((size_t)a * m1 + b) * m2 + c] + 1;
        }
  }
  return OAL_OK;
}

oal_status oal_q19_level_create(int32_t device, int32_t precision, int32_t nocts, const int32_t* onbr, oal_q19_level** out) {
  if (!out || !onbr) return fail(OAL_E_INVALID_ARG, "null argument");
  *out = nullptr;
  if (precision != OAL_STORE_F32 && precision != OAL_STORE_F64)
    return fail(OAL_E_INVALID_ARG, "the octree level stores FP32 or FP64 populations (got storage %d)", precision);
  if (nocts <= 0 || (int64_t)nocts * 27 > INT32_MAX) return fail(OAL_E_INVALID_ARG, "bad oct count %d", nocts);
  for (int64_t t = 0; t < (int64_t)nocts * 27; ++t) {
    if (onbr[t] < 0 || onbr[t] > nocts) return fail(OAL_E_INVALID_ARG, "onbr entry %lld out of range", (long long)t);
    if (onbr[t] == 0)
      return fail(OAL_E_UNSUPPORTED,
                  "oct %lld has no neighbour at offset %d: a level with domain faces or bodies needs its slot "
                  "tables (oal_q19_level_create_desc)", (long long)(t / 27) + 1, (int)(t % 27));
  }
  if (oal_status s = check_device(device)) return s;
  DeviceGuard g(device);
  oal_q19_level* L = new oal_q19_level();
  L->device = device;
  L->precision = precision;
  L->nocts = nocts;
  L->es = precision == OAL_STORE_F64 ? 8 : 4;
  oal_status s = alloc_state(L);
  if (s == OAL_OK) {
    const cudaError_t e = upload(&L->onbr, onbr, (size_t)27 * nocts);
    if (e != cudaSuccess) {
      cudaGetLastError();
      s = fail(OAL_E_OUT_OF_MEMORY, "level tables: %s", cudaGetErrorString(e));
    }
  }
  if (s != OAL_OK) {
    oal_q19_level_destroy(L);
    return s;
  }
  *out = L;
  return OAL_OK;
}

oal_status oal_q19_level_create_desc(int32_t device, int32_t precision, const oal_q19_level_desc* d, oal_q19_level** out) {
  return create_desc_impl(device, precision, d, false, out);
}

}  // extern "C"

static oal_status create_desc_impl(int32_t device, int32_t precision, const oal_q19_level_desc* d, bool transfers,
                                   oal_q19_level** out) {
  if (!out || !d || !d->onbr) return fail(OAL_E_INVALID_ARG, "null argument");
  *out = nullptr;
  if (precision != OAL_STORE_F32 && precision != OAL_STORE_F64)
    return fail(OAL_E_INVALID_ARG, "the octree level stores FP32 or FP64 populations (got storage %d)", precision);
  const int32_t nocts = d->nocts;
  if (nocts <= 0 || (int64_t)nocts * 27 > INT32_MAX) return fail(OAL_E_INVALID_ARG, "bad oct count %d", nocts);
  if (d->ncut < 0 || d->nlinks < 0 || d->ntri < 0) return fail(OAL_E_INVALID_ARG, "negative counts");
  if (d->ncut > 0 && (!d->cutidx || !d->cut_off || !d->cut_dir || !d->cut_q || !d->cut_partner))
    return fail(OAL_E_INVALID_ARG, "cut cells need cutidx, cut_off, cut_dir, cut_q and cut_partner");
  for (int f = 0; f < 6; ++f)
    if (d->faces[f] < OAL_Q19_FACE_PERIODIC || d->faces[f] > OAL_Q19_FACE_FREESTREAM)
      return fail(OAL_E_INVALID_ARG, "face %d: unknown condition %d", f, d->faces[f]);
  const size_t ns = (size_t)nocts * 8;
  // host-side validation of every index the kernels follow
  std::vector<uint8_t> kind(ns, OAL_Q19_K_FLUID);
  if (d->kind) std::memcpy(kind.data(), d->kind, ns);
  for (size_t s = 0; s < ns; ++s) {
    if (kind[s] > OAL_Q19_K_BOUNDARY) return fail(OAL_E_INVALID_ARG, "slot %zu: unknown kind %d", s, kind[s]);
    if (!transfers && (kind[s] == OAL_Q19_K_GHOST || kind[s] == OAL_Q19_K_COVERED))
      return fail(OAL_E_UNSUPPORTED, "ghost and covered slots belong to a refined mesh: create it with oal_q19_octree_create");
  }
  for (int64_t t = 0; t < (int64_t)nocts * 27; ++t)
    if (d->onbr[t] < 0 || d->onbr[t] > nocts) return fail(OAL_E_INVALID_ARG, "onbr entry %lld out of range", (long long)t);
  std::vector<uint32_t> special(ns, 0);
  if (d->special) std::memcpy(special.data(), d->special, ns * 4);
  std::vector<int32_t> cutidx(ns, 0);
  if (d->cutidx) std::memcpy(cutidx.data(), d->cutidx, ns * 4);
  if (d->ncut > 0) {
    if (d->cut_off[0] != 1 || d->cut_off[d->ncut] != d->nlinks + 1)
      return fail(OAL_E_INVALID_ARG, "cut_off must run from 1 to nlinks + 1");
    for (int c = 0; c < d->ncut; ++c) {
      if (d->cut_off[c + 1] < d->cut_off[c]) return fail(OAL_E_INVALID_ARG, "cut_off must not decrease");
      for (int li = d->cut_off[c]; li < d->cut_off[c + 1] - 1; ++li)
        if (d->cut_dir[li] <= d->cut_dir[li - 1])
          return fail(OAL_E_INVALID_ARG, "the links of a cut cell must be in increasing direction order");
    }
    for (int li = 0; li < d->nlinks; ++li) {
      if (d->cut_dir[li] < 2 || d->cut_dir[li] > 19) return fail(OAL_E_INVALID_ARG, "cut_dir %d", d->cut_dir[li]);
      if (!(d->cut_q[li] > 0 && d->cut_q[li] <= 1)) return fail(OAL_E_INVALID_ARG, "cut_q must lie in (0, 1]");
      if (d->cut_tri && (d->cut_tri[li] < 0 || d->cut_tri[li] > d->ntri)) return fail(OAL_E_INVALID_ARG, "cut_tri out of range");
    }
  }
  std::vector<int32_t> plain, walls;
  for (int32_t o = 0; o < nocts; ++o) {
    if (d->real && !d->real[o]) continue;
    bool any_fluid = false, all_plain = true;
    for (int k = 0; k < 8; ++k) {
      const size_t s = (size_t)o * 8 + k;
      const bool fluid = kind[s] == OAL_Q19_K_FLUID;
      any_fluid |= fluid;
      if (!fluid || special[s] != 0) all_plain = false;
      if (cutidx[s] < 0 || cutidx[s] > d->ncut) return fail(OAL_E_INVALID_ARG, "cutidx out of range");
      if (!fluid) continue;
      if (special[s] & 1u) return fail(OAL_E_INVALID_ARG, "the rest direction cannot be special");
      // every pull source of a fluid slot must exist unless its direction is special; a special
      // direction whose source is not a boundary slot needs the slot's cut cell
      const int x = k & 1, y = (k >> 1) & 1, z = (k >> 2) & 1;
      for (int j = 0; j < Q; ++j) {
        const int px = x - cx(j), py = y - cy(j), pz = z - cz(j);
        const int ox = px < 0 ? -1 : (px > 1 ? 1 : 0), oy = py < 0 ? -1 : (py > 1 ? 1 : 0), oz = pz < 0 ? -1 : (pz > 1 ? 1 : 0);
        const int so = d->onbr[(int64_t)o * 27 + (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)] - 1;
        const int child = (px - 2 * ox) + 2 * (py - 2 * oy) + 4 * (pz - 2 * oz);
        const bool boundary_src = so >= 0 && kind[(size_t)so * 8 + child] == OAL_Q19_K_BOUNDARY;
        if (!((special[s] >> j) & 1u)) {
          if (so < 0) return fail(OAL_E_INVALID_ARG, "slot %zu pulls direction %d from a missing oct", s, j + 1);
          continue;
        }
        if (boundary_src) continue;
        const int ci = cutidx[s] - 1;
        if (ci < 0) return fail(OAL_E_INVALID_ARG, "slot %zu: special direction %d without a cut cell", s, j + 1);
        // the Bouzidi q < 1/2 branch reads the partner x - c_i (i = opp j) when the link has one
        const int i = opp(j);
        bool found = false, ok = false;
        for (int li = d->cut_off[ci] - 1; li < d->cut_off[ci + 1] - 1; ++li)
          if (d->cut_dir[li] - 1 == i) {
            found = true;
            ok = d->cut_partner[li] != 0;
          }
        if (!found) return fail(OAL_E_INVALID_ARG, "slot %zu: special direction %d without its cut link", s, j + 1);
        if (ok) {
          const int qx = x - cx(i), qy = y - cy(i), qz = z - cz(i);
          const int px2 = qx < 0 ? -1 : (qx > 1 ? 1 : 0), py2 = qy < 0 ? -1 : (qy > 1 ? 1 : 0), pz2 = qz < 0 ? -1 : (qz > 1 ? 1 : 0);
          if (d->onbr[(int64_t)o * 27 + (px2 + 1) + 3 * (py2 + 1) + 9 * (pz2 + 1)] == 0)
            return fail(OAL_E_INVALID_ARG, "slot %zu: a Bouzidi partner in a missing oct", s);
        }
      }
      // the velocity gradient falls back to the own velocity for missing neighbours (no read)
    }
    if (!any_fluid) continue;
    (all_plain ? plain : walls).push_back(o);
  }
  if (oal_status s = check_device(device)) return s;
  DeviceGuard g(device);
  oal_q19_level* L = new oal_q19_level();
  L->device = device;
  L->precision = precision;
  L->nocts = nocts;
  L->es = precision == OAL_STORE_F64 ? 8 : 4;
  L->walls = true;
  L->ncut = d->ncut;
  L->nlinks = d->nlinks;
  L->ntri = std::max(d->ntri, 1);
  for (int f = 0; f < 6; ++f) L->faces[f] = d->faces[f];
  L->n_plain = (int32_t)plain.size();
  L->n_walls = (int32_t)walls.size();
  std::vector<uint8_t> face(ns, 0);
  if (d->face) std::memcpy(face.data(), d->face, ns);
  std::vector<float> qdir((size_t)std::max(d->ncut, 1) * Q, 0.5f);
  std::vector<uint8_t> okdir((size_t)std::max(d->ncut, 1) * Q, 0);
  std::vector<int32_t> tri_off(L->ntri + 1, 0), tri_links;
  if (d->ncut > 0) {
    for (int c = 0; c < d->ncut; ++c)
      for (int li = d->cut_off[c] - 1; li < d->cut_off[c + 1] - 1; ++li) {
        qdir[(size_t)c * Q + d->cut_dir[li] - 1] = d->cut_q[li];
        okdir[(size_t)c * Q + d->cut_dir[li] - 1] = d->cut_partner[li] != 0;
      }
    // links by triangle bin (no triangle -> bin 1), ascending link order within a bin
    std::vector<int32_t> bin(d->nlinks);
    for (int li = 0; li < d->nlinks; ++li) {
      const int t = d->cut_tri ? d->cut_tri[li] : 0;
      bin[li] = (t > 0 ? t : 1) - 1;
      ++tri_off[bin[li] + 1];
    }
    for (int t = 0; t < L->ntri; ++t) tri_off[t + 1] += tri_off[t];
    tri_links.resize(d->nlinks);
    std::vector<int32_t> fillp(tri_off.begin(), tri_off.end() - 1);
    for (int li = 0; li < d->nlinks; ++li) tri_links[fillp[bin[li]]++] = li;
  }
  oal_status s = alloc_state(L);
  if (s == OAL_OK) {
    cudaError_t e = upload(&L->onbr, d->onbr, (size_t)27 * nocts);
    if (e == cudaSuccess) e = upload(&L->kind, kind.data(), ns);
    if (e == cudaSuccess) e = upload(&L->face, face.data(), ns);
    if (e == cudaSuccess) e = upload(&L->special, special.data(), ns);
    if (e == cudaSuccess) e = upload(&L->cutidx, cutidx.data(), ns);
    if (e == cudaSuccess) e = upload(&L->qdir, qdir.data(), qdir.size());
    if (e == cudaSuccess) e = upload(&L->okdir, okdir.data(), okdir.size());
    if (e == cudaSuccess && d->ncut > 0) e = upload(&L->cut_off, d->cut_off, (size_t)d->ncut + 1);
    if (e == cudaSuccess && d->nlinks > 0) e = upload(&L->cut_dir, d->cut_dir, (size_t)d->nlinks);
    if (e == cudaSuccess && d->nlinks > 0) e = cudaMalloc(&L->mom, sizeof(double) * d->nlinks);
    if (e == cudaSuccess) e = upload(&L->tri_off, tri_off.data(), tri_off.size());
    if (e == cudaSuccess && !tri_links.empty()) e = upload(&L->tri_links, tri_links.data(), tri_links.size());
    if (e == cudaSuccess) e = cudaMalloc(&L->tri_force, sizeof(double) * (3 * (size_t)L->ntri + 3));
    if (e == cudaSuccess) e = cudaMemset(L->tri_force, 0, sizeof(double) * (3 * (size_t)L->ntri + 3));
    if (e == cudaSuccess) e = upload(&L->work_plain, plain.data(), plain.size());
    if (e == cudaSuccess) e = upload(&L->work_walls, walls.data(), walls.size());
    if (e == cudaSuccess && L->n_plain > 0 && L->n_walls > 0) {
      e = cudaStreamCreateWithFlags(&L->side, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L->fork, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L->join, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      s = fail(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "level tables: %s", cudaGetErrorString(e));
    }
  }
  if (s != OAL_OK) {
    oal_q19_level_destroy(L);
    return s;
  }
  *out = L;
  return OAL_OK;
}

extern "C" {

oal_status oal_q19_level_destroy(oal_q19_level* L) {
  if (!L) return OAL_OK;
  {
    DeviceGuard g(L->device);
    cudaFree(L->onbr);
    for (int b = 0; b < 2; ++b) {
      cudaFree(L->f[b]);
      cudaFree(L->u[b]);
      cudaFree(L->rho[b]);
    }
    cudaFree(L->part);
    void* tabs[] = {L->kind, L->face, L->special, L->cutidx, L->qdir, L->okdir, L->cut_off, L->cut_dir, L->mom,
                    L->tri_off, L->tri_links, L->tri_force, L->work_plain, L->work_walls};
    for (void* t : tabs) cudaFree(t);
    if (L->fork) cudaEventDestroy(L->fork);
    if (L->join) cudaEventDestroy(L->join);
    if (L->side) cudaStreamDestroy(L->side);
  }
  delete L;
  return OAL_OK;
}

oal_status oal_q19_level_initialise(oal_q19_level* L, const oal_q19_params* p, const void* rho, const void* u, const void* du) {
  if (!L || !rho || !u) return fail(OAL_E_INVALID_ARG, "null argument");
  if (oal_status s = check_params(p)) return s;
  DeviceGuard g(L->device);
  const size_t ns = (size_t)L->nocts * 8;
  void *d_rho = nullptr, *d_u = nullptr, *d_du = nullptr;
  cudaError_t e = cudaMalloc(&d_rho, L->es * ns);
  if (e == cudaSuccess) e = cudaMalloc(&d_u, L->es * ns * 3);
  if (e == cudaSuccess && du) e = cudaMalloc(&d_du, L->es * ns * 9);
  if (e == cudaSuccess) e = cudaMemcpy(d_rho, rho, L->es * ns, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_u, u, L->es * ns * 3, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && du) e = cudaMemcpy(d_du, du, L->es * ns * 9, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const unsigned grid = (unsigned)((ns + 255) / 256);
    if (L->precision == OAL_STORE_F64) {
      k_q19_initialise<double><<<grid, 256>>>((int64_t)ns, L->kind, (const double*)d_rho, (const double*)d_u,
                                              (const double*)d_du, p->nu, (double*)L->f[0], (double*)L->f[1],
                                              (double*)L->u[0], (double*)L->u[1], (double*)L->rho[0], (double*)L->rho[1]);
    } else {
      k_q19_initialise<float><<<grid, 256>>>((int64_t)ns, L->kind, (const float*)d_rho, (const float*)d_u,
                                             (const float*)d_du, (float)p->nu, (float*)L->f[0], (float*)L->f[1],
                                             (float*)L->u[0], (float*)L->u[1], (float*)L->rho[0], (float*)L->rho[1]);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  cudaFree(d_rho);
  cudaFree(d_u);
  cudaFree(d_du);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(OAL_E_CUDA, "q19 initialise: %s", cudaGetErrorString(e));
  }
  L->cur = 0;
  L->steps = 0;
  L->forces_valid = false;
  return OAL_OK;
}

oal_status oal_q19_level_advance(oal_q19_level* L, const oal_q19_params* p, int32_t n_steps, int32_t collect_forces,
                                 void* stream) {
  if (!L) return fail(OAL_E_INVALID_ARG, "null level");
  if (oal_status s = check_params(p)) return s;
  if (n_steps < 0) return fail(OAL_E_INVALID_ARG, "n_steps < 0");
  DeviceGuard g(L->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool collect = collect_forces != 0;
  return L->precision == OAL_STORE_F64 ? advance_t<double>(L, p, n_steps, collect, st)
                                       : advance_t<float>(L, p, n_steps, collect, st);
}

oal_status oal_q19_level_forces(oal_q19_level* L, double* total, double* per_triangle) {
  if (!L) return fail(OAL_E_INVALID_ARG, "null level");
  DeviceGuard g(L->device);
  if (!L->walls || !L->forces_valid) {
    if (total) total[0] = total[1] = total[2] = 0;
    if (per_triangle && L->walls) std::memset(per_triangle, 0, sizeof(double) * 3 * (size_t)L->ntri);
    return OAL_OK;
  }
  Q19_TRY(cudaDeviceSynchronize());
  if (total) Q19_TRY(cudaMemcpy(total, L->tri_force + 3 * (int64_t)L->ntri, 3 * sizeof(double), cudaMemcpyDeviceToHost));
  if (per_triangle) Q19_TRY(cudaMemcpy(per_triangle, L->tri_force, 3 * sizeof(double) * L->ntri, cudaMemcpyDeviceToHost));
  return OAL_OK;
}

oal_status oal_q19_level_get_state(oal_q19_level* L, void* f, void* u, void* rho) {
  if (!L) return fail(OAL_E_INVALID_ARG, "null level");
  DeviceGuard g(L->device);
  const size_t ns = (size_t)L->nocts * 8;
  Q19_TRY(cudaDeviceSynchronize());
  if (f) Q19_TRY(cudaMemcpy(f, L->f[L->cur], L->es * ns * Q, cudaMemcpyDeviceToHost));
  if (u) Q19_TRY(cudaMemcpy(u, L->u[L->cur], L->es * ns * 3, cudaMemcpyDeviceToHost));
  if (rho) Q19_TRY(cudaMemcpy(rho, L->rho[L->cur], L->es * ns, cudaMemcpyDeviceToHost));
  return OAL_OK;
}

oal_status oal_q19_level_set_state(oal_q19_level* L, const void* f, const void* u, const void* rho) {
  if (!L || !f || !u || !rho) return fail(OAL_E_INVALID_ARG, "null argument");
  DeviceGuard g(L->device);
  const size_t ns = (size_t)L->nocts * 8;
  Q19_TRY(cudaDeviceSynchronize());
  Q19_TRY(cudaMemcpy(L->f[L->cur], f, L->es * ns * Q, cudaMemcpyHostToDevice));
  Q19_TRY(cudaMemcpy(L->u[L->cur], u, L->es * ns * 3, cudaMemcpyHostToDevice));
  Q19_TRY(cudaMemcpy(L->rho[L->cur], rho, L->es * ns, cudaMemcpyHostToDevice));
  return OAL_OK;
}

oal_status oal_q19_level_get_buffer(oal_q19_level* L, int32_t which, void* f, void* u, void* rho) {
  if (!L || (which != 0 && which != 1)) return fail(OAL_E_INVALID_ARG, "null level or buffer %d", which);
  DeviceGuard g(L->device);
  const size_t ns = (size_t)L->nocts * 8;
  const int b = L->cur ^ which;
  Q19_TRY(cudaDeviceSynchronize());
  if (f) Q19_TRY(cudaMemcpy(f, L->f[b], L->es * ns * Q, cudaMemcpyDeviceToHost));
  if (u) Q19_TRY(cudaMemcpy(u, L->u[b], L->es * ns * 3, cudaMemcpyDeviceToHost));
  if (rho) Q19_TRY(cudaMemcpy(rho, L->rho[b], L->es * ns, cudaMemcpyDeviceToHost));
  return OAL_OK;
}

oal_status oal_q19_level_set_buffer(oal_q19_level* L, int32_t which, const void* f, const void* u, const void* rho) {
  if (!L || !f || !u || !rho || (which != 0 && which != 1)) return fail(OAL_E_INVALID_ARG, "null argument or buffer %d", which);
  DeviceGuard g(L->device);
  const size_t ns = (size_t)L->nocts * 8;
  const int b = L->cur ^ which;
  Q19_TRY(cudaDeviceSynchronize());
  Q19_TRY(cudaMemcpy(L->f[b], f, L->es * ns * Q, cudaMemcpyHostToDevice));
  Q19_TRY(cudaMemcpy(L->u[b], u, L->es * ns * 3, cudaMemcpyHostToDevice));
  Q19_TRY(cudaMemcpy(L->rho[b], rho, L->es * ns, cudaMemcpyHostToDevice));
  return OAL_OK;
}

oal_status oal_q19_level_device_state(oal_q19_level* L, void** f, void** u, void** rho, int64_t* steps) {
  if (!L) return fail(OAL_E_INVALID_ARG, "null level");
  if (f) *f = L->f[L->cur];
  if (u) *u = L->u[L->cur];
  if (rho) *rho = L->rho[L->cur];
  if (steps) *steps = L->steps;
  return OAL_OK;
}

oal_status oal_q19_level_totals(oal_q19_level* L, double* out, void* stream) {
  if (!L || !out) return fail(OAL_E_INVALID_ARG, "null argument");
  DeviceGuard g(L->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t ns = (int64_t)L->nocts * 8;
  const int grid = (int)std::min<int64_t>(kTotalsCtas, (ns + 255) / 256);
  if (L->precision == OAL_STORE_F64)
    k_q19_totals<double><<<grid, 256, 0, st>>>(ns, L->kind, (const double*)L->rho[L->cur], (const double*)L->u[L->cur], L->part);
  else
    k_q19_totals<float><<<grid, 256, 0, st>>>(ns, L->kind, (const float*)L->rho[L->cur], (const float*)L->u[L->cur], L->part);
  k_q19_totals_final<<<1, 32, 0, st>>>(L->part, grid, L->part + 5 * kTotalsCtas);
  Q19_TRY(cudaGetLastError());
  Q19_TRY(cudaMemcpyAsync(out, L->part + 5 * kTotalsCtas, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
  Q19_TRY(cudaStreamSynchronize(st));
  return OAL_OK;
}

oal_status oal_q19_collide_cells(int32_t precision, int64_t n, const void* f, const void* omega, double sigma,
                                 const void* pfd, const void* F, void* out, void* rho, void* u, void* stream) {
  if (n < 0 || (n > 0 && (!f || !omega || !pfd || !F || !out || !rho || !u)))
    return fail(OAL_E_INVALID_ARG, "bad arguments");
  if (precision != OAL_STORE_F32 && precision != OAL_STORE_F64) return fail(OAL_E_INVALID_ARG, "precision %d", precision);
  if (n == 0) return OAL_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned grid = (unsigned)((n + 127) / 128);
  if (precision == OAL_STORE_F64)
    k_q19_collide_cells<double><<<grid, 128, 0, st>>>(n, (const double*)f, (const double*)omega, sigma, (const double*)pfd,
                                                      (const double*)F, (double*)out, (double*)rho, (double*)u);
  else
    k_q19_collide_cells<float><<<grid, 128, 0, st>>>(n, (const float*)f, (const float*)omega, (float)sigma, (const float*)pfd,
                                                     (const float*)F, (float*)out, (float*)rho, (float*)u);
  Q19_TRY(cudaGetLastError());
  return OAL_OK;
}

}  // extern "C"

// ---- several levels: transfers and the recursive step (coupling.jl) ------------------------------

namespace {

// rho, u and Pi_neq of slot s of a population buffer (coupling.jl:16-23)
template <class T>
__device__ __forceinline__ void slot_moments(const T* __restrict__ f, int64_t s, T* m) {
  const int64_t o = s >> 3;
  const int k = (int)(s & 7);
  T fl[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) fl[i] = f[o * (8 * Q) + 8 * i + k];
  T drho, mx, my, mz, P[6];
  moments<T>(fl, drho, mx, my, mz, P);
  const T rho = drho + T(1), inv = T(1) / rho;
  const T ux = mx * inv, uy = my * inv, uz = mz * inv;
  const T d3 = drho * T(1.0 / 3.0);
  const T rx = rho * ux, ry = rho * uy, rz = rho * uz;
  m[0] = rho;
  m[1] = ux;
  m[2] = uy;
  m[3] = uz;
  m[4] = P[0] - d3 - rx * ux;
  m[5] = P[1] - d3 - ry * uy;
  m[6] = P[2] - d3 - rz * uz;
  m[7] = P[3] - rx * uy;
  m[8] = P[4] - rx * uz;
  m[9] = P[5] - ry * uz;
}

// the ten moments of the donor cells at the requested time (fill_ghosts! stage 1): mode 0 the old
// buffer, 1 the new one, 2 the blend w0 old + w1 new (covered donors unblended from the new buffer)
template <class T>
__global__ void k_q19_donor_moments(int32_t n, const int32_t* __restrict__ cells, const T* __restrict__ fnew,
                                    const T* __restrict__ fold, int mode, T w0, T w1, const uint8_t* __restrict__ cov,
                                    T* __restrict__ out) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  T m[10];
  if (mode == 0) {
    slot_moments<T>(fold, cells[c], m);
  } else if (mode == 1 || cov[c]) {
    slot_moments<T>(fnew, cells[c], m);
  } else {
    T mo[10];
    slot_moments<T>(fnew, cells[c], m);
    slot_moments<T>(fold, cells[c], mo);
#pragma unroll
    for (int i = 0; i < 10; ++i) m[i] = w0 * mo[i] + w1 * m[i];
  }
#pragma unroll
  for (int i = 0; i < 10; ++i) out[10 * (int64_t)c + i] = m[i];
}

// rebuild slot s from interpolated moments at `omega` (coupling.jl:26-30, rebuild_oct!)
template <class T>
__device__ __forceinline__ void rebuild_slot(const T* acc, T scale, T omega, int64_t s, T* f, T* u, T* rho) {
  const T r = acc[0], ux = acc[1], uy = acc[2], uz = acc[3];
  T p[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) p[i] = scale * acc[4 + i];
  const T drho = r - T(1);
  T out[Q];
  populations<T>(drho, r, ux, uy, uz, p, T(1) - omega, out);
  if (below_floor<T>(out)) limit_unforced<T>(out, drho, r, ux, uy, uz);
  const int64_t o = s >> 3;
  const int k = (int)(s & 7);
#pragma unroll
  for (int i = 0; i < Q; ++i) f[o * (8 * Q) + 8 * i + k] = out[i];
  u[o * 24 + k] = ux;
  u[o * 24 + 8 + k] = uy;
  u[o * 24 + 16 + k] = uz;
  rho[s] = r;
}

// ghost fill (fill_ghosts! stage 2): weighted sums of the donor moments, rebuilt at the fine omega.
// 16 lanes per ghost: lane q < 10 sums moment q over the 64 nodes in node order (the reference's
// order per moment), lane 0 gathers the ten sums and rebuilds the slot.
template <class T>
__global__ void __launch_bounds__(256) k_q19_fill(int32_t ng, const int32_t* __restrict__ ghost_slot,
                                                  const int32_t* __restrict__ dix, const float* __restrict__ gw,
                                                  const T* __restrict__ dm, T scale, T omega, T* f, T* u, T* rho) {
  const int lane = threadIdx.x & 31, q = lane & 15;
  const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
  if (g >= ng) return;  // both lanes groups of a warp test their own g; a group leaves as a whole
  const unsigned gmask = 0xffffu << (lane & 16);
  T acc = T(0);
  if (q < 10) {
    const int32_t* dx = dix + 64 * g;
    const float* w = gw + 64 * g;
#pragma unroll 8
    for (int n = 0; n < 64; ++n) {
      const int32_t d = __ldg(dx + n);
      if (!d) continue;
      acc += T(__ldg(w + n)) * __ldg(dm + 10 * (int64_t)(d - 1) + q);
    }
  }
  T m[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) m[i] = __shfl_sync(gmask, acc, (lane & 16) + i);
  if (q == 0) rebuild_slot<T>(m, scale, omega, ghost_slot[g], f, u, rho);
}

// the ten moments of the restriction sources from the fine buffer (restrict! stage 1)
template <class T>
__global__ void k_q19_source_moments(int32_t n, const int32_t* __restrict__ cells, const T* __restrict__ f,
                                     T* __restrict__ out) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  T m[10];
  slot_moments<T>(f, cells[c], m);
#pragma unroll
  for (int i = 0; i < 10; ++i) out[10 * (int64_t)c + i] = m[i];
}

__host__ __device__ constexpr double restrict_w1(int d) { return d == 0 || d == 3 ? -0.0625 : 0.5625; }  // cubic at 1/2
__device__ __forceinline__ int stencil_inner_node(int m) {
  return (1 + (m & 1)) + 4 * (1 + ((m >> 1) & 1)) + 16 * (1 + ((m >> 2) & 1));
}

// restriction (restrict! stage 2): cubic weights over 64 sources, or the admissible children
// averaged; 16 lanes per restricted slot, lane q < 10 sums moment q in the reference's node order
template <class T>
__global__ void __launch_bounds__(256) k_q19_restrict(int32_t nr, const int32_t* __restrict__ rslot,
                                                      const int32_t* __restrict__ six, const uint8_t* __restrict__ cubic,
                                                      const T* __restrict__ rm, T scale, T omega, T* f, T* u, T* rho) {
  const int lane = threadIdx.x & 31, q = lane & 15;
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
  if (r >= nr) return;
  const unsigned gmask = 0xffffu << (lane & 16);
  const int32_t* sx = six + 64 * r;
  T acc = T(0);
  int cnt = 0;
  if (cubic[r]) {
    if (q < 10) {
#pragma unroll 8
      for (int n = 0; n < 64; ++n) {
        const T wn = T(restrict_w1(n & 3) * restrict_w1((n >> 2) & 3) * restrict_w1(n >> 4));
        acc += wn * __ldg(rm + 10 * (int64_t)(__ldg(sx + n) - 1) + q);
      }
    }
  } else {
#pragma unroll
    for (int mm = 0; mm < 8; ++mm) {
      const int32_t d = __ldg(sx + stencil_inner_node(mm));
      if (!d) continue;
      if (q < 10) acc += __ldg(rm + 10 * (int64_t)(d - 1) + q);
      ++cnt;
    }
    if (cnt == 0) return;  // uniform over the group: nothing to restrict
    acc *= T(1) / T(cnt);
  }
  T m[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) m[i] = __shfl_sync(gmask, acc, (lane & 16) + i);
  if (q == 0) rebuild_slot<T>(m, scale, omega, rslot[r], f, u, rho);
}

// copy slots (the last ghost fill) from the old buffers into the new ones (copy_ghosts!)
template <class T>
__global__ void k_q19_copy_slots(int32_t n, const int32_t* __restrict__ slots, const T* __restrict__ fs, T* fd,
                                 const T* __restrict__ us, T* ud, const T* __restrict__ rs, T* rd) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int64_t s = slots[c], o = s >> 3;
  const int k = (int)(s & 7);
#pragma unroll
  for (int i = 0; i < Q; ++i) fd[o * (8 * Q) + 8 * i + k] = fs[o * (8 * Q) + 8 * i + k];
#pragma unroll
  for (int a = 0; a < 3; ++a) ud[o * 24 + 8 * a + k] = us[o * 24 + 8 * a + k];
  rd[s] = rs[s];
}

__global__ void k_add3(int64_t n, const double* __restrict__ a, double* __restrict__ acc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) acc[i] += a[i];
}

// distinct entries of a (64, n) 1-based slot table, in first-appearance order, and the table
// re-indexed into them (state.jl:144-154 index_table)
void index_table(const int32_t* tab, int32_t n, std::vector<int32_t>& cells, std::vector<int32_t>& ix) {
  std::unordered_map<int32_t, int32_t> idx;
  ix.assign(64 * (size_t)n, 0);
  cells.clear();
  for (int32_t j = 0; j < n; ++j)
    for (int nn = 0; nn < 64; ++nn) {
      const int32_t s = tab[64 * (size_t)j + nn];
      if (!s) continue;
      auto it = idx.find(s);
      if (it == idx.end()) {
        cells.push_back(s - 1);
        it = idx.emplace(s, (int32_t)cells.size()).first;
      }
      ix[64 * (size_t)j + nn] = it->second;
    }
}

struct Transfer {
  // fill of this level from the coarser one
  int32_t ng = 0, nd = 0;
  int32_t* ghost_slot = nullptr;
  int32_t* dix = nullptr;
  float* gw = nullptr;
  int32_t* dcells = nullptr;
  uint8_t* dcov = nullptr;
  void* dm = nullptr;
  // restriction into this level from the finer one
  int32_t nr = 0, ns = 0;
  int32_t* rslot = nullptr;
  int32_t* six = nullptr;
  uint8_t* rcubic = nullptr;
  int32_t* scells = nullptr;
  void* rm = nullptr;
};

}  // namespace

// two coarse steps captured as one CUDA graph: after them every level is back on the buffers it
// started from (level l steps 2^l times), so the graph replays as long as the parameters and the
// coarsest level's starting buffer are those it was captured with
struct CoarseGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<char> key;  // parameters of every level
  int parity = -1;        // the coarsest level's current buffer at capture
};

struct oal_q19_octree {
  int device = 0;
  int precision = OAL_STORE_F32;
  int L = 0;
  size_t es = 4;
  std::vector<oal_q19_level*> lv;
  std::vector<Transfer> tt;
  int32_t ntri = 1;
  double* tri_total = nullptr;  // (ntri, 3) then the total (3)
  double* part = nullptr;       // per-level totals (5 L)
  bool forces_valid = false;
  cudaStream_t capture = nullptr;  // private stream the graphs are captured on
  CoarseGraph graphs[2];           // one per starting parity of the coarsest level
};

namespace {

template <class T>
T omega_of_h(double nu) {
  const T n = T(nu);
  return T(1) / (T(3) * n + T(0.5));
}
template <class T>
T pre_collision_factor_h(T omega) {
  const T d = T(1) - omega;
  return (d < T(0) ? -d : d) > T(0.05) ? T(1) / d : T(0);
}

template <class T>
cudaError_t fill_ghosts_t(oal_q19_octree* tr, const oal_q19_params* p, int l, T weight, cudaStream_t st) {
  const Transfer& t = tr->tt[l - 1];
  if (t.ng == 0) return cudaSuccess;
  oal_q19_level* Lc = tr->lv[l - 2];
  oal_q19_level* Lf = tr->lv[l - 1];
  const T omega_c = omega_of_h<T>(p[l - 2].nu), omega_f = omega_of_h<T>(p[l - 1].nu);
  const T tau_c = T(1) / omega_c, tau_f = T(1) / omega_f;
  const T scale = tau_f / (T(2) * tau_c) * pre_collision_factor_h<T>(omega_c);
  const T w1 = weight, w0 = T(1) - weight;
  const int mode = w1 == T(0) ? 0 : (w0 == T(0) ? 1 : 2);
  k_q19_donor_moments<T><<<(t.nd + 127) / 128, 128, 0, st>>>(t.nd, t.dcells, (const T*)Lc->f[Lc->cur],
                                                             (const T*)Lc->f[1 - Lc->cur], mode, w0, w1, t.dcov, (T*)t.dm);
  k_q19_fill<T><<<(unsigned)((16 * (int64_t)t.ng + 255) / 256), 256, 0, st>>>(t.ng, t.ghost_slot, t.dix, t.gw, (const T*)t.dm, scale, omega_f,
                                                    (T*)Lf->f[Lf->cur], (T*)Lf->u[Lf->cur], (T*)Lf->rho[Lf->cur]);
  return cudaGetLastError();
}

template <class T>
cudaError_t restrict_t(oal_q19_octree* tr, const oal_q19_params* p, int l, cudaStream_t st) {
  const Transfer& t = tr->tt[l - 1];
  if (t.nr == 0) return cudaSuccess;
  oal_q19_level* Lc = tr->lv[l - 1];
  oal_q19_level* Lf = tr->lv[l];
  const T omega_c = omega_of_h<T>(p[l - 1].nu), omega_f = omega_of_h<T>(p[l].nu);
  const T tau_c = T(1) / omega_c, tau_f = T(1) / omega_f;
  const T scale = T(2) * tau_c / tau_f * pre_collision_factor_h<T>(omega_f);
  k_q19_source_moments<T><<<(t.ns + 127) / 128, 128, 0, st>>>(t.ns, t.scells, (const T*)Lf->f[Lf->cur], (T*)t.rm);
  k_q19_restrict<T><<<(unsigned)((16 * (int64_t)t.nr + 255) / 256), 256, 0, st>>>(t.nr, t.rslot, t.six, t.rcubic, (const T*)t.rm, scale, omega_c,
                                                        (T*)Lc->f[Lc->cur], (T*)Lc->u[Lc->cur], (T*)Lc->rho[Lc->cur]);
  return cudaGetLastError();
}

template <class T>
cudaError_t copy_ghosts_t(oal_q19_octree* tr, int l, cudaStream_t st) {
  const Transfer& t = tr->tt[l - 1];
  if (l == tr->L || t.ng == 0) return cudaSuccess;
  oal_q19_level* S = tr->lv[l - 1];
  const int c = S->cur, o = 1 - S->cur;
  k_q19_copy_slots<T><<<(t.ng + 127) / 128, 128, 0, st>>>(t.ng, t.ghost_slot, (const T*)S->f[o], (T*)S->f[c],
                                                          (const T*)S->u[o], (T*)S->u[c], (const T*)S->rho[o], (T*)S->rho[c]);
  return cudaGetLastError();
}

// step_recursive! (coupling.jl:240-254)
template <class T>
cudaError_t step_recursive_t(oal_q19_octree* tr, const oal_q19_params* p, int l, bool collect, cudaStream_t st) {
  cudaError_t e = step_level_t<T>(tr->lv[l - 1], &p[l - 1], collect, st);
  if (e == cudaSuccess) e = copy_ghosts_t<T>(tr, l, st);
  if (e == cudaSuccess && l < tr->L) {
    e = step_recursive_t<T>(tr, p, l + 1, collect, st);
    if (e == cudaSuccess) e = restrict_t<T>(tr, p, l, st);
    if (e == cudaSuccess) e = fill_ghosts_t<T>(tr, p, l + 1, T(0.5), st);
    if (e == cudaSuccess) e = step_recursive_t<T>(tr, p, l + 1, collect, st);
    if (e == cudaSuccess) e = restrict_t<T>(tr, p, l, st);
    if (e == cudaSuccess) e = fill_ghosts_t<T>(tr, p, l + 1, T(1), st);
  }
  return e;
}

// the graph of two non-collecting coarse steps for the current parity and parameters
template <class T>
cudaError_t coarse_graph(oal_q19_octree* tr, const oal_q19_params* p, cudaGraphExec_t* out) {
  const int parity = tr->lv[0]->cur;
  CoarseGraph& g = tr->graphs[parity];
  const char* kp = reinterpret_cast<const char*>(p);
  const size_t kn = sizeof(oal_q19_params) * (size_t)tr->L;
  if (g.exec && g.parity == parity && g.key.size() == kn && std::memcmp(g.key.data(), kp, kn) == 0) {
    *out = g.exec;
    return cudaSuccess;
  }
  if (g.exec) {
    cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
  }
  cudaError_t e = cudaSuccess;
  if (!tr->capture) e = cudaStreamCreateWithFlags(&tr->capture, cudaStreamNonBlocking);
  if (e != cudaSuccess) return e;
  std::vector<int64_t> steps;
  for (oal_q19_level* L : tr->lv) steps.push_back(L->steps);
  cudaGraph_t graph = nullptr;
  e = cudaStreamBeginCapture(tr->capture, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t e1 = step_recursive_t<T>(tr, p, 1, false, tr->capture);
  if (e1 == cudaSuccess) e1 = step_recursive_t<T>(tr, p, 1, false, tr->capture);
  e = cudaStreamEndCapture(tr->capture, &graph);
  for (size_t i = 0; i < tr->lv.size(); ++i) tr->lv[i]->steps = steps[i];  // captured, not run
  if (e1 != cudaSuccess) e = e1;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    g.exec = nullptr;
    return e;
  }
  g.key.assign(kp, kp + kn);
  g.parity = parity;
  *out = g.exec;
  return cudaSuccess;
}

template <class T>
oal_status octree_advance_t(oal_q19_octree* tr, const oal_q19_params* p, int32_t n, bool collect, cudaStream_t st) {
  // pairs of non-collecting coarse steps replay a captured graph; the rest runs launch by launch
  int32_t s = 0;
  while (n - s >= 2 && !(collect && n - s <= 2)) {
    cudaGraphExec_t exec = nullptr;
    Q19_TRY(coarse_graph<T>(tr, p, &exec));
    Q19_TRY(cudaGraphLaunch(exec, st));
    for (size_t l = 0; l < tr->lv.size(); ++l) tr->lv[l]->steps += (int64_t)2 << l;
    s += 2;
  }
  for (; s < n; ++s) {
    const bool last = collect && s == n - 1;
    if (last)
      for (oal_q19_level* L : tr->lv)
        if (L->walls && L->nlinks > 0) Q19_TRY(cudaMemsetAsync(L->mom, 0, sizeof(double) * L->nlinks, st));
    Q19_TRY(step_recursive_t<T>(tr, p, 1, last, st));
    if (last) {
      Q19_TRY(cudaMemsetAsync(tr->tri_total, 0, sizeof(double) * 3 * (size_t)tr->ntri, st));
      for (oal_q19_level* L : tr->lv) {
        if (!L->walls) continue;
        Q19_TRY(level_forces(L, st));
        const int64_t nn = 3 * (int64_t)std::min(L->ntri, tr->ntri);
        k_add3<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(nn, L->tri_force, tr->tri_total);
      }
      k_q19_force_total<<<1, 256, 0, st>>>(tr->ntri, tr->tri_total, tr->tri_total + 3 * (int64_t)tr->ntri);
      Q19_TRY(cudaGetLastError());
      tr->forces_valid = true;
    }
  }
  return OAL_OK;
}

template <class T>
oal_status couple_initial_t(oal_q19_octree* tr, const oal_q19_params* p) {
  // couple_initial! (coupling.jl:257-268): restrict every level into its parent, then fill every
  // level's ghosts; each level's old buffers mirror the new ones
  auto mirror = [&](int l) -> cudaError_t {
    oal_q19_level* S = tr->lv[l - 1];
    const size_t ns = (size_t)S->nocts * 8;
    cudaError_t e = cudaMemcpy(S->f[1 - S->cur], S->f[S->cur], S->es * ns * Q, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(S->u[1 - S->cur], S->u[S->cur], S->es * ns * 3, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(S->rho[1 - S->cur], S->rho[S->cur], S->es * ns, cudaMemcpyDeviceToDevice);
    return e;
  };
  for (int l = tr->L - 1; l >= 1; --l) {
    Q19_TRY(restrict_t<T>(tr, p, l, nullptr));
    Q19_TRY(mirror(l));
  }
  for (int l = 2; l <= tr->L; ++l) {
    Q19_TRY(fill_ghosts_t<T>(tr, p, l, T(1), nullptr));
    Q19_TRY(mirror(l));
  }
  Q19_TRY(cudaDeviceSynchronize());
  return OAL_OK;
}

}  // namespace

extern "C" {

oal_status oal_q19_octree_destroy(oal_q19_octree* tr) {
  if (!tr) return OAL_OK;
  {
    DeviceGuard g(tr->device);
    for (Transfer& t : tr->tt) {
      void* ptrs[] = {t.ghost_slot, t.dix, t.gw, t.dcells, t.dcov, t.dm, t.rslot, t.six, t.rcubic, t.scells, t.rm};
      for (void* q : ptrs) cudaFree(q);
    }
    cudaFree(tr->tri_total);
    cudaFree(tr->part);
    for (CoarseGraph& g : tr->graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    if (tr->capture) cudaStreamDestroy(tr->capture);
  }
  for (oal_q19_level* L : tr->lv) oal_q19_level_destroy(L);
  delete tr;
  return OAL_OK;
}

oal_status oal_q19_octree_create(int32_t device, int32_t precision, int32_t nlevels, const oal_q19_level_desc* d,
                                 oal_q19_octree** out) {
  if (!out || !d) return fail(OAL_E_INVALID_ARG, "null argument");
  *out = nullptr;
  if (nlevels < 1 || nlevels > 12) return fail(OAL_E_INVALID_ARG, "nlevels %d", nlevels);
  // host-side checks of the transfer tables: every slot they name exists and has the right kind
  for (int l = 1; l <= nlevels; ++l) {
    const oal_q19_level_desc& D = d[l - 1];
    const int64_t ns = 8 * (int64_t)D.nocts;
    auto kind_of = [&](const oal_q19_level_desc& X, int64_t s) { return X.kind ? X.kind[s] : (uint8_t)OAL_Q19_K_FLUID; };
    if (D.nghost < 0 || D.nrestrict < 0) return fail(OAL_E_INVALID_ARG, "level %d: negative transfer counts", l);
    if (D.nghost > 0 && (l == 1 || !D.ghost_slot || !D.ghost_donor || !D.ghost_w))
      return fail(OAL_E_INVALID_ARG, "level %d: ghost lists need a coarser level and their arrays", l);
    if (D.nrestrict > 0 && (l == nlevels || !D.restrict_slot || !D.restrict_src || !D.restrict_cubic))
      return fail(OAL_E_INVALID_ARG, "level %d: restriction lists need a finer level and their arrays", l);
    for (int32_t g = 0; g < D.nghost; ++g) {
      const int64_t s = D.ghost_slot[g] - 1;
      if (s < 0 || s >= ns || kind_of(D, s) != OAL_Q19_K_GHOST) return fail(OAL_E_INVALID_ARG, "level %d: ghost_slot %d", l, g);
      const int64_t nsc = 8 * (int64_t)d[l - 2].nocts;
      for (int n = 0; n < 64; ++n) {
        const int64_t ds = D.ghost_donor[64 * (int64_t)g + n];
        if (ds < 0 || ds > nsc) return fail(OAL_E_INVALID_ARG, "level %d: ghost donor out of range", l);
      }
    }
    for (int32_t r = 0; r < D.nrestrict; ++r) {
      const int64_t s = D.restrict_slot[r] - 1;
      if (s < 0 || s >= ns || kind_of(D, s) != OAL_Q19_K_COVERED)
        return fail(OAL_E_INVALID_ARG, "level %d: restrict_slot %d", l, r);
      const int64_t nsf = 8 * (int64_t)d[l].nocts;
      for (int n = 0; n < 64; ++n) {
        const int64_t cs = D.restrict_src[64 * (int64_t)r + n];
        if (cs < 0 || cs > nsf) return fail(OAL_E_INVALID_ARG, "level %d: restriction source out of range", l);
        if (D.restrict_cubic[r] && cs == 0) return fail(OAL_E_INVALID_ARG, "level %d: incomplete cubic stencil", l);
      }
    }
  }
  if (oal_status s = check_device(device)) return s;
  oal_q19_octree* tr = new oal_q19_octree();
  tr->device = device;
  tr->precision = precision;
  tr->L = nlevels;
  tr->es = precision == OAL_STORE_F64 ? 8 : 4;
  tr->tt.resize(nlevels);
  for (int l = 1; l <= nlevels; ++l) {
    oal_q19_level* L = nullptr;
    oal_status s = create_desc_impl(device, precision, &d[l - 1], true, &L);
    if (s != OAL_OK) {
      oal_q19_octree_destroy(tr);
      return s;
    }
    tr->lv.push_back(L);
    tr->ntri = std::max(tr->ntri, std::max(d[l - 1].ntri, 1));
  }
  DeviceGuard g(device);
  cudaError_t e = cudaSuccess;
  for (int l = 1; l <= nlevels && e == cudaSuccess; ++l) {
    const oal_q19_level_desc& D = d[l - 1];
    Transfer& t = tr->tt[l - 1];
    if (D.nghost > 0) {
      std::vector<int32_t> cells, ix, gs(D.nghost);
      index_table(D.ghost_donor, D.nghost, cells, ix);
      for (int32_t i = 0; i < D.nghost; ++i) gs[i] = D.ghost_slot[i] - 1;
      std::vector<uint8_t> cov(cells.size());
      const oal_q19_level_desc& P = d[l - 2];
      for (size_t c = 0; c < cells.size(); ++c) cov[c] = P.kind && P.kind[cells[c]] == OAL_Q19_K_COVERED;
      t.ng = D.nghost;
      t.nd = (int32_t)cells.size();
      e = upload(&t.ghost_slot, gs.data(), gs.size());
      if (e == cudaSuccess) e = upload(&t.dix, ix.data(), ix.size());
      if (e == cudaSuccess) e = upload(&t.gw, D.ghost_w, 64 * (size_t)D.nghost);
      if (e == cudaSuccess) e = upload(&t.dcells, cells.data(), cells.size());
      if (e == cudaSuccess) e = upload(&t.dcov, cov.data(), cov.size());
      if (e == cudaSuccess) e = cudaMalloc(&t.dm, tr->es * 10 * std::max<size_t>(cells.size(), 1));
    }
    if (e == cudaSuccess && D.nrestrict > 0) {
      std::vector<int32_t> cells, ix, rs(D.nrestrict);
      index_table(D.restrict_src, D.nrestrict, cells, ix);
      for (int32_t i = 0; i < D.nrestrict; ++i) rs[i] = D.restrict_slot[i] - 1;
      t.nr = D.nrestrict;
      t.ns = (int32_t)cells.size();
      e = upload(&t.rslot, rs.data(), rs.size());
      if (e == cudaSuccess) e = upload(&t.six, ix.data(), ix.size());
      if (e == cudaSuccess) e = upload(&t.rcubic, D.restrict_cubic, (size_t)D.nrestrict);
      if (e == cudaSuccess) e = upload(&t.scells, cells.data(), cells.size());
      if (e == cudaSuccess) e = cudaMalloc(&t.rm, tr->es * 10 * std::max<size_t>(cells.size(), 1));
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&tr->tri_total, sizeof(double) * (3 * (size_t)tr->ntri + 3));
  if (e == cudaSuccess) e = cudaMemset(tr->tri_total, 0, sizeof(double) * (3 * (size_t)tr->ntri + 3));
  if (e != cudaSuccess) {
    cudaGetLastError();
    oal_q19_octree_destroy(tr);
    return fail(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "octree tables: %s", cudaGetErrorString(e));
  }
  *out = tr;
  return OAL_OK;
}

oal_status oal_q19_octree_level(oal_q19_octree* tr, int32_t level, oal_q19_level** out) {
  if (!tr || !out || level < 1 || level > tr->L) return fail(OAL_E_INVALID_ARG, "bad level");
  *out = tr->lv[level - 1];
  return OAL_OK;
}

oal_status oal_q19_octree_initialise(oal_q19_octree* tr, const oal_q19_params* p, const void* const* rho,
                                     const void* const* u, const void* const* du) {
  if (!tr || !p || !rho || !u) return fail(OAL_E_INVALID_ARG, "null argument");
  for (int l = 1; l <= tr->L; ++l) {
    if (oal_status s = oal_q19_level_initialise(tr->lv[l - 1], &p[l - 1], rho[l - 1], u[l - 1], du ? du[l - 1] : nullptr))
      return s;
  }
  DeviceGuard g(tr->device);
  tr->forces_valid = false;
  return tr->precision == OAL_STORE_F64 ? couple_initial_t<double>(tr, p) : couple_initial_t<float>(tr, p);
}

oal_status oal_q19_octree_advance(oal_q19_octree* tr, const oal_q19_params* p, int32_t n, int32_t collect_forces,
                                  void* stream) {
  if (!tr || !p) return fail(OAL_E_INVALID_ARG, "null argument");
  for (int l = 0; l < tr->L; ++l)
    if (oal_status s = check_params(&p[l])) return s;
  if (n < 0) return fail(OAL_E_INVALID_ARG, "n_coarse_steps < 0");
  DeviceGuard g(tr->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return tr->precision == OAL_STORE_F64 ? octree_advance_t<double>(tr, p, n, collect_forces != 0, st)
                                        : octree_advance_t<float>(tr, p, n, collect_forces != 0, st);
}

oal_status oal_q19_octree_forces(oal_q19_octree* tr, double* total, double* per_triangle) {
  if (!tr) return fail(OAL_E_INVALID_ARG, "null argument");
  DeviceGuard g(tr->device);
  if (!tr->forces_valid) {
    if (total) total[0] = total[1] = total[2] = 0;
    if (per_triangle) std::memset(per_triangle, 0, sizeof(double) * 3 * (size_t)tr->ntri);
    return OAL_OK;
  }
  Q19_TRY(cudaDeviceSynchronize());
  if (total) Q19_TRY(cudaMemcpy(total, tr->tri_total + 3 * (int64_t)tr->ntri, 3 * sizeof(double), cudaMemcpyDeviceToHost));
  if (per_triangle) Q19_TRY(cudaMemcpy(per_triangle, tr->tri_total, 3 * sizeof(double) * tr->ntri, cudaMemcpyDeviceToHost));
  return OAL_OK;
}

oal_status oal_q19_octree_totals(oal_q19_octree* tr, double* out) {
  if (!tr || !out) return fail(OAL_E_INVALID_ARG, "null argument");
  for (int i = 0; i < 5; ++i) out[i] = 0;
  for (int l = 1; l <= tr->L; ++l) {
    double t[5];
    if (oal_status s = oal_q19_level_totals(tr->lv[l - 1], t, nullptr)) return s;
    const double w = std::ldexp(1.0, 3 * (tr->L - l));
    for (int i = 0; i < 5; ++i) out[i] += w * t[i];
  }
  return OAL_OK;
}

}  // extern "C"
