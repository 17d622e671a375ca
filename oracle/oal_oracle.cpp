// oal_oracle.cpp — CPU ORACLE (test infrastructure only; never linked into the product).
//
// A plain C++ restatement of the reference's D3Q27 cumulant lattice-Boltzmann level step
// (OpenAeroLab, Julia), templated on the arithmetic type: instantiated in double it is the
// FP64 oracle; in float it mirrors the reference's Float32 kernel and is the timed CPU
// baseline. Parallelised over blocks with OpenMP. Built with -ffp-contract=off so the float
// instantiation rounds like the reference (no fused multiply-add contraction).
//
// Followed line by line (paths inside the reference project):
//   D3Q27 tables ............ src/collision/lattice.jl:10-60, src/collision/timestep.jl:2005-2023
//   block order ............. src/geometry/domain.jl:785 (sorted active block tuples)
//   neighbour table ......... src/geometry/domain_topology.jl:919-953 (+ periodic wrap per axis)
//   analytic sphere ......... src/geometry/domain_generation.jl:132-150
//   equilibria .............. src/collision/physics_utils.jl:30-109
//   inlet noise hash ........ src/collision/physics_utils.jl:5-17
//   pull + face BCs ......... src/collision/kernel_cumulant.jl:173-400
//   obstacle (full-way) ..... src/collision/kernel_cumulant.jl:402-417
//   macros/sponge/wall model  src/collision/kernel_cumulant.jl:420-491
//   WALE + gradients ........ src/collision/kernel_cumulant.jl:496-595,
//                             src/collision/physics_utils.jl:1981-2035,2217-2233
//   cumulant collision ...... src/collision/kernel_cumulant.jl:1-26,597-844
//   positivity limiter ...... src/collision/kernel_cumulant.jl:849-884
//   Guo forcing + store ..... src/collision/kernel_cumulant.jl:889-908
//   half-way BB + MEM ....... src/octree_q19/src/stream.jl:229-256 (link rule, generalised to the
//                             27 D3Q27 links; the reference's GPU path has no D3Q27 analogue)
//   Grad wall ............... src/geometry/grad_wall_kernel.jl:42-144 (velocity mode 0), called
//                             from src/collision/timestep.jl:1738-1751
//   linear Bouzidi wall ..... src/geometry/bouzidi_kernel.jl:150-380 (unshifted D3Q27), called from
//                             src/collision/timestep.jl:1752-1768 after the step
//   mass / momentum ......... src/octree_q19/src/state.jl:614-637 (Float64 sums)
//   block AMR (default flags): parent interpolation of a refined level's pulls
//                             src/collision/physics_interpolation.jl:10-51,128-137,188-346,705-1198
//                             and kernel_cumulant.jl:286-316,346-388; restriction
//                             src/collision/amr_coupling.jl:130-190,7562-7640 + kernel :1900-3242
//                             (children average, f_neq rescale, two moment-correction passes,
//                             shell macros); the recursion src/solver/solver_control.jl:55-560 is
//                             driven by oracle/__init__.py (OracleAMR)
//
// Parity status: the reference is Julia and cannot run in this environment, so this restatement
// is pinned by the reference's analytic gates (Taylor-Green decay, conservation, rest state) and
// by the reference's own identities for the tables, not by reference-produced vectors.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <array>
#include <tuple>

#include "../include/oal.h"

namespace {

constexpr int Q = 27;
constexpr int BS = 8;

struct Tables {
  int cx[Q], cy[Q], cz[Q], opp[Q], mir_y[Q], mir_z[Q];
  double w[Q];
};

// lattice.jl:10-60 — z outer, y middle, x inner; k = 1 + (cx+1) + 3(cy+1) + 9(cz+1)
Tables make_tables() {
  Tables t{};
  int n = 0;
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        t.cx[n] = x; t.cy[n] = y; t.cz[n] = z;
        int d2 = x * x + y * y + z * z;
        t.w[n] = d2 == 0 ? 8.0 / 27.0 : d2 == 1 ? 2.0 / 27.0 : d2 == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
        ++n;
      }
  for (int i = 0; i < Q; ++i)
    for (int j = 0; j < Q; ++j) {
      if (t.cx[j] == -t.cx[i] && t.cy[j] == -t.cy[i] && t.cz[j] == -t.cz[i]) t.opp[i] = j;
      if (t.cx[j] == t.cx[i] && t.cy[j] == -t.cy[i] && t.cz[j] == t.cz[i]) t.mir_y[i] = j;
      if (t.cx[j] == t.cx[i] && t.cy[j] == t.cy[i] && t.cz[j] == -t.cz[i]) t.mir_z[i] = j;
    }
  return t;
}
const Tables TB = make_tables();

// physics_utils.jl:5-17 (Int32 wrap-around arithmetic done in uint32)
uint32_t gpu_hash(int32_t x) {
  uint32_t h = (uint32_t)x;
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  return h ^ (h >> 16);
}
float gradient_noise(int32_t gx, int32_t gy, int32_t gz, int32_t seed) {
  uint32_t combined = (uint32_t)gx * 374761393u + (uint32_t)gy * 668265263u +
                      (uint32_t)gz * 1274126177u + (uint32_t)seed;
  uint32_t h = gpu_hash((int32_t)combined);
  return ((float)(h & 0xFFFFu) / 32768.0f) - 1.0f;
}

// physics_utils.jl:30-35
template <class T>
T feq2(T rho, T ux, T uy, T uz, T w, T cx, T cy, T cz) {
  T cu = cx * ux + cy * uy + cz * uz;
  T usq = ux * ux + uy * uy + uz * uz;
  return rho * w * (T(1) + T(3) * cu + T(4.5) * cu * cu - T(1.5) * usq);
}
// physics_utils.jl:65-95 (limiter gate off: the default build)
template <class T>
T feq4(T rho, T ux, T uy, T uz, T w, T cx, T cy, T cz) {
  T cu = cx * ux + cy * uy + cz * uz;
  T usq = ux * ux + uy * uy + uz * uz;
  T cu2 = cu * cu, cu3 = cu2 * cu, cu4 = cu2 * cu2, usq2 = usq * usq;
  T val = T(1) + T(3) * cu + T(4.5) * cu2 - T(1.5) * usq;
  T ho = (T(4.5) * cu3 - T(4.5) * cu * usq) + (T(3.375) * cu4 - T(6.75) * cu2 * usq + T(1.125) * usq2);
  val += ho;
  return rho * w * val;
}
// physics_utils.jl:97-109
template <class T>
T feq_auto(T rho, T ux, T uy, T uz, T w, T cx, T cy, T cz, int comp) {
  return comp == 1 ? feq4(rho, ux, uy, uz, w, cx, cy, cz) : feq2(rho, ux, uy, uz, w, cx, cy, cz);
}

// kernel_cumulant.jl:4-26
template <class T>
void chimera_forward(T& a, T& b, T& c, T u) {
  T m0 = a + b + c, m1 = c - a, m2 = a + c;
  a = m0;
  b = m1 - u * m0;
  c = m2 - T(2) * u * m1 + u * u * m0;
}
template <class T>
void chimera_backward(T& a, T& b, T& c, T u) {
  T kc0 = a, kc1 = b, kc2 = c;
  T m0 = kc0;
  T m1 = kc1 + u * kc0;
  T m2 = kc2 + T(2) * u * kc1 + u * u * kc0;
  T fp = (m2 + m1) * T(0.5);
  T fm = (m2 - m1) * T(0.5);
  T f0 = m0 - m2;
  a = fm; b = f0; c = fp;
}

struct Level {
  int32_t nb, nx, ny, nz;
  const int32_t* coords;   // n*3 1-based
  const int32_t* nbr;      // Julia (n,27): nbr[b + n*dir], 1-based, 0 none
  const uint8_t* obstacle; // 512*n or null
  const float* sponge;
  const float* wall_dist;
  const void* parent = nullptr;  // Parent<T> of a refined level (null on level 1)
  void* pi_neq = nullptr;        // T[6][512 * nb]: Pi_neq of variable nu_sgs mode 1 (read, then refreshed)
};

// The parent level seen from a refined level's kernel (perform_timestep_v2! arguments
// parent_f, parent_rho, parent_vel, parent_ptr, *_old, parent_dim_*, tau_parent, temporal_weight,
// use_temporal_interp). Arrays in the reference layout of the parent level.
template <class T>
struct Parent {
  const T* f_new; const T* rho_new; const T* vel_new;
  const T* f_old; const T* rho_old; const T* vel_old;
  const int32_t* ptr;  // parent_ptr (dim_x, dim_y, dim_z), Julia column-major, 1-based block, 0 = none
  int32_t dim_x, dim_y, dim_z, nb;
  T tau_parent, tau_fine, tw;
  int use_temporal, comp, level_visc_physical;
};

inline int64_t cidx(int x, int y, int z) { return (int64_t)x + 8 * y + 64 * z; }  // 0-based

template <class T>
struct Arr {
  // Reference layout accessors; x,y,z 0-based, b 0-based, k 0-based.
  int64_t nb;
  int64_t f(int x, int y, int z, int b, int k) const { return cidx(x, y, z) + 512 * (int64_t)b + 512 * nb * k; }
  int64_t s(int x, int y, int z, int b) const { return cidx(x, y, z) + 512 * (int64_t)b; }
};

// ---- parent interpolation (physics_interpolation.jl, default flags: no mirror ghost, no periodic-y
// AMR, no B-spline or quintic macros, extrapolation fallback on) --------------------------------
struct Bracket { int i0, i1; };
template <class T>
void parent_bracket(T p_cont, int n, int& i0, int& i1, T& w) {  // :128-137
  if (n <= 1) { i0 = 1; i1 = 1; w = T(0); return; }
  const T pc = std::min(std::max(p_cont, T(1)), T(n));
  i0 = std::min(std::max((int)std::floor(pc), 1), n - 1);
  i1 = i0 + 1;
  w = std::min(std::max(pc - T(i0), T(0)), T(1));
}

template <class T>
struct Node { T f, rho, ux, uy, uz, fneq; bool ok; };

// parent cell (1-based global index) -> block (0-based) and cell offset, or -1 outside / absent.
// Julia's (g - 1) ÷ 8 truncates toward zero, so g < 1 would alias block 1 with an out-of-block
// local index; such nodes count as absent here.
template <class T>
int64_t parent_cell(const Parent<T>& P, int pgx, int pgy, int pgz) {
  if (pgx < 1 || pgy < 1 || pgz < 1) return -1;
  const int pbx = (pgx - 1) / BS + 1, pby = (pgy - 1) / BS + 1, pbz = (pgz - 1) / BS + 1;
  if (pbx > P.dim_x || pby > P.dim_y || pbz > P.dim_z) return -1;
  const int32_t pb = P.ptr[(pbx - 1) + (int64_t)P.dim_x * ((pby - 1) + (int64_t)P.dim_y * (pbz - 1))];
  if (pb <= 0) return -1;
  return cidx((pgx - 1) % BS, (pgy - 1) % BS, (pgz - 1) % BS) + 512 * (int64_t)(pb - 1);
}

// get_blended (:776-859), time-blended when use_temporal and tw < 0.99
template <class T>
Node<T> get_blended(const Parent<T>& P, int pgx, int pgy, int pgz, int k, T wk, T cx, T cy, T cz) {
  const int64_t c = parent_cell(P, pgx, pgy, pgz);
  if (c < 0) return Node<T>{wk, T(1), T(0), T(0), T(0), T(0), false};
  const int64_t n = 512 * (int64_t)P.nb;
  T f = P.f_new[c + n * k], rho = P.rho_new[c], ux = P.vel_new[c], uy = P.vel_new[c + n], uz = P.vel_new[c + 2 * n];
  if (P.use_temporal == 1 && P.tw < T(0.99) && P.f_old) {
    const T tw = P.tw;
    f = P.f_old[c + n * k] * (T(1) - tw) + f * tw;
    rho = P.rho_old[c] * (T(1) - tw) + rho * tw;
    ux = P.vel_old[c] * (T(1) - tw) + ux * tw;
    uy = P.vel_old[c + n] * (T(1) - tw) + uy * tw;
    uz = P.vel_old[c + 2 * n] * (T(1) - tw) + uz * tw;
  }
  const T feqc = feq_auto<T>(rho, ux, uy, uz, wk, cx, cy, cz, P.comp);
  return Node<T>{f, rho, ux, uy, uz, f - feqc, true};
}

// get_macro (:860-923)
template <class T>
Node<T> get_macro(const Parent<T>& P, int pgx, int pgy, int pgz) {
  const int64_t c = parent_cell(P, pgx, pgy, pgz);
  if (c < 0) return Node<T>{T(0), T(1), T(0), T(0), T(0), T(0), false};
  const int64_t n = 512 * (int64_t)P.nb;
  T rho = P.rho_new[c], ux = P.vel_new[c], uy = P.vel_new[c + n], uz = P.vel_new[c + 2 * n];
  if (P.use_temporal == 1 && P.tw < T(0.99) && P.rho_old) {
    const T tw = P.tw;
    rho = P.rho_old[c] * (T(1) - tw) + rho * tw;
    ux = P.vel_old[c] * (T(1) - tw) + ux * tw;
    uy = P.vel_old[c + n] * (T(1) - tw) + uy * tw;
    uz = P.vel_old[c + 2 * n] * (T(1) - tw) + uz * tw;
  }
  return Node<T>{T(0), rho, ux, uy, uz, T(0), true};
}

// cubic Lagrange weights of the stencil node i in -1..2 (:953-960)
template <class T>
T lagrange3(int i, T w) {
  return i == -1 ? (-w * (w - T(1)) * (w - T(2)) / T(6))
       : i == 0  ? ((w + T(1)) * (w - T(1)) * (w - T(2)) / T(2))
       : i == 1  ? (-w * (w + T(1)) * (w - T(2)) / T(2))
                 : (w * (w + T(1)) * (w - T(1)) / T(6));
}

// sample_parent_macro_for_fine_cell (:188-346): trilinear macros; a missing corner is
// extrapolated linearly from its partner along x, then y, then z
template <class T>
bool sample_parent_macro(const Parent<T>& P, int fgx, int fgy, int fgz, T& r_out, T& x_out, T& y_out, T& z_out) {
  const int pnx = P.dim_x * BS, pny = P.dim_y * BS, pnz = P.dim_z * BS;
  int px0, px1, py0, py1, pz0, pz1;
  T wx, wy, wz;
  parent_bracket<T>(T(fgx) * T(0.5) + T(0.25), pnx, px0, px1, wx);
  parent_bracket<T>(T(fgy) * T(0.5) + T(0.25), pny, py0, py1, wy);
  parent_bracket<T>(T(fgz) * T(0.5) + T(0.25), pnz, pz0, pz1, wz);
  Node<T> d[8];
  const int ix[8] = {px0, px1, px0, px1, px0, px1, px0, px1};
  const int iy[8] = {py0, py0, py1, py1, py0, py0, py1, py1};
  const int iz[8] = {pz0, pz0, pz0, pz0, pz1, pz1, pz1, pz1};
  for (int c = 0; c < 8; ++c) d[c] = get_macro<T>(P, ix[c], iy[c], iz[c]);
  const T w[8] = {(T(1) - wx) * (T(1) - wy) * (T(1) - wz), wx * (T(1) - wy) * (T(1) - wz),
                  (T(1) - wx) * wy * (T(1) - wz),         wx * wy * (T(1) - wz),
                  (T(1) - wx) * (T(1) - wy) * wz,         wx * (T(1) - wy) * wz,
                  (T(1) - wx) * wy * wz,                  wx * wy * wz};
  bool all = true;
  for (int c = 0; c < 8; ++c) all = all && d[c].ok;
  auto acc = [&](T Node<T>::*m) {
    T s = w[0] * (d[0].*m);
    for (int c = 1; c < 8; ++c) s = s + w[c] * (d[c].*m);
    return s;
  };
  if (!all) {
    bool any = false;
    for (int c = 0; c < 8; ++c) any = any || d[c].ok;
    if (!any) { r_out = T(1); x_out = y_out = z_out = T(0); return false; }
    const int pxm = px0 - 1, pxp = px1 + 1, pym = py0 - 1, pyp = py1 + 1, pzm = pz0 - 1, pzp = pz1 + 1;
    // (a, b, far node of a when b is missing, far node of b when a is missing), reference order
    struct Edge { int a, b, fa[3], fb[3]; };
    const Edge edges[12] = {
        {0, 1, {pxm, py0, pz0}, {pxp, py0, pz0}}, {2, 3, {pxm, py1, pz0}, {pxp, py1, pz0}},
        {4, 5, {pxm, py0, pz1}, {pxp, py0, pz1}}, {6, 7, {pxm, py1, pz1}, {pxp, py1, pz1}},
        {0, 2, {px0, pym, pz0}, {px0, pyp, pz0}}, {1, 3, {px1, pym, pz0}, {px1, pyp, pz0}},
        {4, 6, {px0, pym, pz1}, {px0, pyp, pz1}}, {5, 7, {px1, pym, pz1}, {px1, pyp, pz1}},
        {0, 4, {px0, py0, pzm}, {px0, py0, pzp}}, {1, 5, {px1, py0, pzm}, {px1, py0, pzp}},
        {2, 6, {px0, py1, pzm}, {px0, py1, pzp}}, {3, 7, {px1, py1, pzm}, {px1, py1, pzp}}};
    for (const Edge& e : edges) {
      if (d[e.a].ok == d[e.b].ok) continue;
      const int src = d[e.a].ok ? e.a : e.b, dst = d[e.a].ok ? e.b : e.a;
      const int* far = d[e.a].ok ? e.fa : e.fb;
      const Node<T> fd = get_macro<T>(P, far[0], far[1], far[2]);
      Node<T>& o = d[dst];
      const Node<T>& s0 = d[src];
      o.rho = fd.ok ? T(2) * s0.rho - fd.rho : s0.rho;
      o.ux = fd.ok ? T(2) * s0.ux - fd.ux : s0.ux;
      o.uy = fd.ok ? T(2) * s0.uy - fd.uy : s0.uy;
      o.uz = fd.ok ? T(2) * s0.uz - fd.uz : s0.uz;
      o.ok = true;
    }
  }
  r_out = acc(&Node<T>::rho); x_out = acc(&Node<T>::ux); y_out = acc(&Node<T>::uy); z_out = acc(&Node<T>::uz);
  return true;
}

// interpolate_with_rescaling (:705-1198) at the fine cell (fgx, fgy, fgz), direction k
template <class T>
T interpolate_with_rescaling(const Parent<T>& P, int fgx, int fgy, int fgz, int k, T wk, T cx, T cy, T cz) {
  const int pnx = P.dim_x * BS, pny = P.dim_y * BS, pnz = P.dim_z * BS;
  int px0, px1, py0, py1, pz0, pz1;
  T wx, wy, wz;
  parent_bracket<T>(T(fgx) * T(0.5) + T(0.25), pnx, px0, px1, wx);
  parent_bracket<T>(T(fgy) * T(0.5) + T(0.25), pny, py0, py1, wy);
  parent_bracket<T>(T(fgz) * T(0.5) + T(0.25), pnz, pz0, pz1, wz);
  const bool use_cubic = px0 - 2 >= 1 && px0 + 2 <= pnx && py0 - 2 >= 1 && py0 + 2 <= pny && pz0 - 2 >= 1 &&
                         pz0 + 2 <= pnz;
  Node<T> d[8];
  const int ix[8] = {px0, px1, px0, px1, px0, px1, px0, px1};
  const int iy[8] = {py0, py0, py1, py1, py0, py0, py1, py1};
  const int iz[8] = {pz0, pz0, pz0, pz0, pz1, pz1, pz1, pz1};
  for (int c = 0; c < 8; ++c) d[c] = get_blended<T>(P, ix[c], iy[c], iz[c], k, wk, cx, cy, cz);
  int anchor = 7;
  for (int c = 0; c < 7; ++c)
    if (d[c].ok) { anchor = c; break; }
  Node<T> v[8];
  for (int c = 0; c < 8; ++c) v[c] = d[c].ok ? d[c] : d[anchor];
  auto trilin = [&](T Node<T>::*m) {
    const T c00 = (v[0].*m) * (T(1) - wx) + (v[1].*m) * wx;
    const T c01 = (v[4].*m) * (T(1) - wx) + (v[5].*m) * wx;
    const T c10 = (v[2].*m) * (T(1) - wx) + (v[3].*m) * wx;
    const T c11 = (v[6].*m) * (T(1) - wx) + (v[7].*m) * wx;
    const T c0 = c00 * (T(1) - wy) + c10 * wy;
    const T c1 = c01 * (T(1) - wy) + c11 * wy;
    return c0 * (T(1) - wz) + c1 * wz;
  };
  bool cubic_all_valid = use_cubic;
  if (use_cubic) {
    for (int a = -1; a <= 2 && cubic_all_valid; ++a)
      for (int bb = -1; bb <= 2 && cubic_all_valid; ++bb)
        for (int c = -1; c <= 2 && cubic_all_valid; ++c)
          if (!get_macro<T>(P, px0 + a, py0 + bb, pz0 + c).ok) cubic_all_valid = false;
  }
  T rho_int, ux_int, uy_int, uz_int;
  if (cubic_all_valid) {
    rho_int = ux_int = uy_int = uz_int = T(0);
    for (int a = -1; a <= 2; ++a)
      for (int bb = -1; bb <= 2; ++bb)
        for (int c = -1; c <= 2; ++c) {
          const Node<T> m = get_macro<T>(P, px0 + a, py0 + bb, pz0 + c);
          const T w3 = lagrange3<T>(a, wx) * lagrange3<T>(bb, wy) * lagrange3<T>(c, wz);
          rho_int += w3 * m.rho;
          ux_int += w3 * m.ux;
          uy_int += w3 * m.uy;
          uz_int += w3 * m.uz;
        }
  } else if (!sample_parent_macro<T>(P, fgx, fgy, fgz, rho_int, ux_int, uy_int, uz_int)) {
    rho_int = trilin(&Node<T>::rho); ux_int = trilin(&Node<T>::ux);
    uy_int = trilin(&Node<T>::uy); uz_int = trilin(&Node<T>::uz);
  }
  const T feq_int = feq_auto<T>(rho_int, ux_int, uy_int, uz_int, wk, cx, cy, cz, P.comp);
  T f_neq = T(0);
  if (use_cubic) {
    const T anchor_neq = d[anchor].fneq;
    for (int a = -1; a <= 2; ++a) {
      const T wxv = lagrange3<T>(a, wx);
      for (int bb = -1; bb <= 2; ++bb) {
        const T wyv = lagrange3<T>(bb, wy);
        for (int c = -1; c <= 2; ++c) {
          const T wzv = lagrange3<T>(c, wz);
          const Node<T> n = get_blended<T>(P, px0 + a, py0 + bb, pz0 + c, k, wk, cx, cy, cz);
          f_neq += wxv * wyv * wzv * (n.ok ? n.fneq : anchor_neq);
        }
      }
    }
  } else {
    f_neq = trilin(&Node<T>::fneq);
  }
  const T tau_c = P.tau_parent - T(0.5), tau_f = P.tau_fine - T(0.5);
  T scale = tau_c > T(1e-6) ? std::min(std::max(tau_f / tau_c, T(0.01)), T(100)) : T(1);
  if (P.level_visc_physical == 1)
    scale = std::min(std::max(P.tau_fine / (T(2) * std::max(P.tau_parent, T(0.500001))), T(0.01)), T(100));
  {  // _amr_fneq_postcoll_prolong_scale (:39-51), on by default
    const T omega_c = T(1) / std::max(P.tau_parent, T(0.500001));
    const T omega_f = T(1) / std::max(P.tau_fine, T(0.500001));
    const T one_m_wc = T(1) - omega_c, one_m_wf = T(1) - omega_f;
    if (std::fabs(one_m_wc) > T(1e-6)) scale = std::min(std::max(scale * (one_m_wf / one_m_wc), T(0.01)), T(100));
  }
  return feq_int + f_neq * scale;
}

// physics_utils.jl:2001-2035 get_velocity_neighbor_fluid (sym_y_plane = 0)
template <class T>
void vel_nb_fluid(const Level& L, const T* vel_in, int x, int y, int z, int b, int dx, int dy, int dz,
                  T& ux, T& uy, T& uz) {
  Arr<T> A{L.nb};
  const int64_t cs = 512 * (int64_t)L.nb;
  int64_t own = A.s(x, y, z, b);
  T ux0 = vel_in[own], uy0 = vel_in[own + cs], uz0 = vel_in[own + 2 * cs];
  int nx = x + dx, ny = y + dy, nz = z + dz;
  if (nx >= 0 && nx < BS && ny >= 0 && ny < BS && nz >= 0 && nz < BS) {
    int64_t i = A.s(nx, ny, nz, b);
    if (L.obstacle && L.obstacle[i]) { ux = ux0; uy = uy0; uz = uz0; return; }
    ux = vel_in[i]; uy = vel_in[i + cs]; uz = vel_in[i + 2 * cs];
    return;
  }
  int ox = nx < 0 ? -1 : (nx >= BS ? 1 : 0);
  int oy = ny < 0 ? -1 : (ny >= BS ? 1 : 0);
  int oz = nz < 0 ? -1 : (nz >= BS ? 1 : 0);
  int dir = (ox + 1) + (oy + 1) * 3 + (oz + 1) * 9;
  int nbi = L.nbr[b + (int64_t)L.nb * dir];
  if (nbi > 0) {
    int nnx = nx < 0 ? nx + BS : (nx >= BS ? nx - BS : nx);
    int nny = ny < 0 ? ny + BS : (ny >= BS ? ny - BS : ny);
    int nnz = nz < 0 ? nz + BS : (nz >= BS ? nz - BS : nz);
    int64_t i = A.s(nnx, nny, nnz, nbi - 1);
    if (L.obstacle && L.obstacle[i]) { ux = ux0; uy = uy0; uz = uz0; return; }
    ux = vel_in[i]; uy = vel_in[i + cs]; uz = vel_in[i + 2 * cs];
    return;
  }
  ux = ux0; uy = uy0; uz = uz0;
}

// Neighbour velocity of the dynamic test filter (kernel_dynamic_sgs.jl:57-103): the previous
// step's velocity of a fluid neighbour, else the given centre velocity (missing or solid).
template <class T>
void vel_nb_centre(const Level& L, const T* vel_in, int x, int y, int z, int b, int dx, int dy, int dz,
                   T cx, T cy, T cz, T (&o)[3]) {
  Arr<T> A{L.nb};
  const int64_t cs = 512 * (int64_t)L.nb;
  const int nx = x + dx, ny = y + dy, nz = z + dz;
  int64_t i = -1;
  if (nx >= 0 && nx < BS && ny >= 0 && ny < BS && nz >= 0 && nz < BS) {
    i = A.s(nx, ny, nz, b);
  } else {
    const int ox = nx < 0 ? -1 : (nx >= BS ? 1 : 0);
    const int oy = ny < 0 ? -1 : (ny >= BS ? 1 : 0);
    const int oz = nz < 0 ? -1 : (nz >= BS ? 1 : 0);
    const int nbi = L.nbr[b + (int64_t)L.nb * ((ox + 1) + (oy + 1) * 3 + (oz + 1) * 9)];
    if (nbi > 0) i = A.s((nx + BS) % BS, (ny + BS) % BS, (nz + BS) % BS, nbi - 1);
  }
  if (i < 0 || (L.obstacle && L.obstacle[i])) { o[0] = cx; o[1] = cy; o[2] = cz; return; }
  o[0] = vel_in[i]; o[1] = vel_in[i + cs]; o[2] = vel_in[i + 2 * cs];
}

// Germano-Lilly Cs^2 (compute_dynamic_cs2_inline, kernel_dynamic_sgs.jl:124-240), Dx = 1
template <class T>
T dynamic_cs2(const T (&c)[3], const T (&n)[6][3], T g11, T g22, T g33, T S12, T S13, T S23) {
  const T inv7 = T(1) / T(7);
  T ut[3], uu[6];
  for (int a = 0; a < 3; ++a) {
    T sum = c[a];
    for (int j = 0; j < 6; ++j) sum += n[j][a];
    ut[a] = inv7 * sum;
  }
  const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
  for (int m = 0; m < 6; ++m) {
    T sum = c[ia[m]] * c[ib[m]];
    for (int j = 0; j < 6; ++j) sum += n[j][ia[m]] * n[j][ib[m]];
    uu[m] = inv7 * sum;
  }
  const T Lxx = uu[0] - ut[0] * ut[0], Lyy = uu[1] - ut[1] * ut[1], Lzz = uu[2] - ut[2] * ut[2];
  const T Lxy = uu[3] - ut[0] * ut[1], Lxz = uu[4] - ut[0] * ut[2], Lyz = uu[5] - ut[1] * ut[2];
  const T Ltr = (Lxx + Lyy + Lzz) * (T(1) / T(3));
  const T Lxx_d = Lxx - Ltr, Lyy_d = Lyy - Ltr, Lzz_d = Lzz - Ltr;
  const T S_sq = T(2) * (g11 * g11 + g22 * g22 + g33 * g33) + T(4) * (S12 * S12 + S13 * S13 + S23 * S23);
  const T S_mag = std::sqrt(std::max(S_sq, T(1e-30)));
  const T M_coeff = T(2) * T(1) * T(1) * T(3.659306f) * S_mag;
  const T Mxx = M_coeff * g11, Myy = M_coeff * g22, Mzz = M_coeff * g33;
  const T Mxy = M_coeff * S12, Mxz = M_coeff * S13, Myz = M_coeff * S23;
  const T Mtr = (Mxx + Myy + Mzz) * (T(1) / T(3));
  const T Mxx_d = Mxx - Mtr, Myy_d = Myy - Mtr, Mzz_d = Mzz - Mtr;
  const T LM = Lxx_d * Mxx_d + Lyy_d * Myy_d + Lzz_d * Mzz_d + T(2) * (Lxy * Mxy + Lxz * Mxz + Lyz * Myz);
  const T MM = Mxx_d * Mxx_d + Myy_d * Myy_d + Mzz_d * Mzz_d + T(2) * (Mxy * Mxy + Mxz * Mxz + Myz * Myz);
  const T cd = T(0.5) * LM / (MM + T(1e-20));
  return std::min(std::max(cd, T(0)), T(0.25));
}

// Pi_neq_ab = sum_k c_a c_b (f_k - f_eq_k) (compute_pi_neq_kernel!, kernel_pi_neq.jl:61-180, D3Q27)
template <class T>
void pi_neq_cell(const T* fk, T rho, T ux, T uy, T uz, int comp, T (&pi)[6]) {
  const bool skip = !std::isfinite(rho) || rho < T(0.01) || rho > T(10) || !std::isfinite(ux) ||
                    !std::isfinite(uy) || !std::isfinite(uz);
  const T rs = skip ? T(0) : rho, us = skip ? T(0) : ux, vs = skip ? T(0) : uy, ws = skip ? T(0) : uz;
  T p[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  for (int k = 0; k < Q; ++k) {
    const T cx = T(TB.cx[k]), cy = T(TB.cy[k]), cz = T(TB.cz[k]);
    const T fe = feq_auto<T>(rs, us, vs, ws, T(TB.w[k]), cx, cy, cz, comp);
    const T fn = (skip ? T(0) : fk[k]) - fe;
    p[0] += cx * cx * fn; p[1] += cy * cy * fn; p[2] += cz * cz * fn;
    p[3] += cx * cy * fn; p[4] += cx * cz * fn; p[5] += cy * cz * fn;
  }
  const T mask = skip ? T(0) : T(1);
  for (int m = 0; m < 6; ++m) pi[m] = p[m] * mask;
}

// Source cell of the pull x - c_k: block index (0-based, -1 = none) and local coordinates.
inline int src_block(const Level& L, int b, int sx, int sy, int sz, int& lx, int& ly, int& lz) {
  if (sx >= 0 && sx < BS && sy >= 0 && sy < BS && sz >= 0 && sz < BS) { lx = sx; ly = sy; lz = sz; return b; }
  int ox = sx < 0 ? -1 : (sx >= BS ? 1 : 0);
  int oy = sy < 0 ? -1 : (sy >= BS ? 1 : 0);
  int oz = sz < 0 ? -1 : (sz >= BS ? 1 : 0);
  int dir = (ox + 1) + (oy + 1) * 3 + (oz + 1) * 9;
  int nbi = L.nbr[b + (int64_t)L.nb * dir];
  if (nbi <= 0) return -1;
  lx = sx - BS * ox; ly = sy - BS * oy; lz = sz - BS * oz;
  return nbi - 1;
}

template <class T>
void step_cell(const Level& L, const oal_step_params& P, const T* f_in, T* f_out, T* f_post, T* rho_out,
               T* vel_out, const T* vel_in, int b, int x, int y, int z, double* force_acc) {
  Arr<T> A{L.nb};
  const int64_t cs = 512 * (int64_t)L.nb;
  const int bx = L.coords[3 * b], by = L.coords[3 * b + 1], bz = L.coords[3 * b + 2];
  // 1-based global coordinates (kernel_cumulant.jl:181-183)
  const int gx = (bx - 1) * BS + x + 1, gy = (by - 1) * BS + y + 1, gz = (bz - 1) * BS + z + 1;
  const int64_t own = A.s(x, y, z, b);
  const bool is_obs = L.obstacle && L.obstacle[own];
  const bool halfway = P.solid_bc == OAL_SOLID_HALFWAY;
  const int comp = P.compressible_corr;
  const T u_inlet = T(P.u_inlet);
  const bool store_post = P.store_post_collision == 1 && f_post != nullptr;

  T* pi_neq = P.variable_nu_sgs == 1 ? static_cast<T*>(L.pi_neq) : nullptr;
  if (halfway && is_obs) {
    // Half-way mode: a solid cell holds the rest equilibrium; no fluid cell reads it.
    vel_out[own] = T(0); vel_out[own + cs] = T(0); vel_out[own + 2 * cs] = T(0);
    rho_out[own] = T(1);
    if (pi_neq)
      for (int m = 0; m < 6; ++m) pi_neq[own + m * cs] = T(0);
    for (int k = 0; k < Q; ++k) {
      f_out[A.f(x, y, z, b, k)] = T(TB.w[k]);
      if (store_post) f_post[A.f(x, y, z, b, k)] = T(TB.w[k]);
    }
    return;
  }

  // STEP 1: pull streaming (kernel_cumulant.jl:190-400)
  T rho = T(0), jx = T(0), jy = T(0), jz = T(0);
  T fs[Q];
  double mx = 0, my = 0, mz = 0;
  bool wall_cell = false;  // a pull source is solid (the reference's Bouzidi/Grad boundary-cell list)
  for (int k = 0; k < Q; ++k) {
    const int cx = TB.cx[k], cy = TB.cy[k], cz = TB.cz[k];
    const int sx = x - cx, sy = y - cy, sz = z - cz;
    T val = T(0);
    int lx, ly, lz;
    int sb = src_block(L, b, sx, sy, sz, lx, ly, lz);
    if (sb >= 0) {
      const bool src_solid = L.obstacle && L.obstacle[A.s(lx, ly, lz, sb)];
      wall_cell = wall_cell || src_solid;
      if (halfway && src_solid) {
        // link opp(k) of this cell is cut: the population this cell sent toward the wall
        // returns (octree_q19/src/stream.jl:229-233, half-way rule, wall at rest)
        const int i = TB.opp[k];
        val = f_in[A.f(x, y, z, b, i)];
        if (P.collect_forces) {
          // momentum exchange (f_i* + f_j(t+1)) c_i with j = k, i toward the wall
          // (stream.jl:248-256), accumulated in Float64
          const double mom = (double)f_in[A.f(x, y, z, b, i)] + (double)val;
          mx += mom * TB.cx[i]; my += mom * TB.cy[i]; mz += mom * TB.cz[i];
        }
      } else {
        val = f_in[A.f(lx, ly, lz, sb, k)];
      }
    } else {
      const int src_gx = gx - cx;
      const int src_gy = gy - cy;  // _pwrap_y: identity (periodic-Y AMR gate off)
      const int src_gz = gz - cz;
      const bool is_inlet = src_gx < 1, is_outlet = src_gx > L.nx;
      const bool is_y_min = src_gy < 1, is_y_max = src_gy > L.ny;
      const bool is_z_min = src_gz < 1, is_z_max = src_gz > L.nz;
      if (is_inlet) {
        float noise = P.inlet_turbulence > 0.0f
                          ? gradient_noise(gy, gz, P.time_step_seed, 1234) * P.inlet_turbulence * P.u_inlet
                          : 0.0f;
        T u_inst = u_inlet + T(noise);
        val = feq_auto<T>(T(1), u_inst, T(0), T(0), T(TB.w[k]), T(cx), T(cy), T(cz), comp);
      } else if (is_outlet) {
        val = f_in[A.f(x, y, z, b, k)];
      } else if (P.zwall_bc != 0 && (is_z_min || is_z_max)) {
        if (P.zwall_bc == 2) {
          val = f_in[A.f(x, y, z, b, TB.opp[k])];
        } else {
          const int zw_k = TB.mir_z[k];
          const int zw_ix = x - cx, zw_iy = y - cy;
          if (zw_ix >= 0 && zw_ix < BS && zw_iy >= 0 && zw_iy < BS) {
            val = f_in[A.f(zw_ix, zw_iy, z, b, zw_k)];
          } else {
            const int zw_ox = zw_ix < 0 ? -1 : (zw_ix >= BS ? 1 : 0);
            const int zw_oy = zw_iy < 0 ? -1 : (zw_iy >= BS ? 1 : 0);
            const int dir = (zw_ox + 1) + (zw_oy + 1) * 3 + 9;
            const int zw_nb = L.nbr[b + (int64_t)L.nb * dir];
            if (zw_nb > 0) {
              const int zw_lx = zw_ix < 0 ? zw_ix + BS : (zw_ix >= BS ? zw_ix - BS : zw_ix);
              const int zw_ly = zw_iy < 0 ? zw_iy + BS : (zw_iy >= BS ? zw_iy - BS : zw_iy);
              val = f_in[A.f(zw_lx, zw_ly, z, zw_nb - 1, zw_k)];
            } else if (L.parent && gy - cy >= 1 && gy - cy <= L.ny) {
              // refined level: the image cell comes from the parent (kernel_cumulant.jl:286-312)
              val = interpolate_with_rescaling<T>(*static_cast<const Parent<T>*>(L.parent), gx - cx, gy - cy, gz, zw_k,
                                                  T(TB.w[zw_k]), T(cx), T(cy), T(-cz));
            } else {
              // level 1: no parent image; the cell's own mirror_z population
              val = f_in[A.f(x, y, z, b, zw_k)];
            }
          }
        }
      } else if (P.transverse_freestream == 1 && (is_y_min || is_y_max || is_z_min || is_z_max)) {
        const T beta_t = T(P.transverse_freestream_blend);
        const T donor = f_in[A.f(x, y, z, b, k)];
        const T feq_fs = feq_auto<T>(T(1), u_inlet, T(0), T(0), T(TB.w[k]), T(cx), T(cy), T(cz), comp);
        val = (T(1) - beta_t) * donor + beta_t * feq_fs;
      } else if (is_y_min && P.ymin_wall_bc == 1) {
        val = f_in[A.f(x, y, z, b, TB.opp[k])];
      } else if (is_y_min || is_y_max) {
        val = f_in[A.f(x, y, z, b, TB.mir_y[k])];
      } else if (is_z_min || is_z_max) {
        val = f_in[A.f(x, y, z, b, TB.mir_z[k])];
      } else if (L.parent) {
        // refined level: interpolated from the parent (kernel_cumulant.jl:346-388)
        val = interpolate_with_rescaling<T>(*static_cast<const Parent<T>*>(L.parent), src_gx, src_gy, src_gz, k,
                                            T(TB.w[k]), T(cx), T(cy), T(cz));
      } else {
        // level 1 (no parent): lattice weight (kernel_cumulant.jl:389-391)
        val = T(TB.w[k]);
      }
    }
    fs[k] = val;
    rho += val;
    jx += val * T(cx);
    jy += val * T(cy);
    jz += val * T(cz);
  }
  if (P.collect_forces && (mx != 0 || my != 0 || mz != 0)) {
    force_acc[0] += mx; force_acc[1] += my; force_acc[2] += mz;
  }

  // Obstacle: simple bounce-back (kernel_cumulant.jl:402-417)
  if (is_obs) {
    vel_out[own] = T(0); vel_out[own + cs] = T(0); vel_out[own + 2 * cs] = T(0);
    rho_out[own] = T(1);
    if (pi_neq)
      for (int m = 0; m < 6; ++m) pi_neq[own + m * cs] = T(0);
    for (int k = 0; k < Q; ++k) {
      T fc = fs[TB.opp[k]];
      f_out[A.f(x, y, z, b, k)] = fc;
      if (store_post) f_post[A.f(x, y, z, b, k)] = fc;
    }
    return;
  }

  // STEP 2: macros + sponge + wall model (kernel_cumulant.jl:420-491)
  rho = std::max(rho, T(0.01));
  T inv_rho = T(1) / rho;
  T ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  const T sp = L.sponge ? T(L.sponge[own]) : T(0);
  if (sp > T(0)) {
    const T rho_target = T(1), ux_target = u_inlet;
    rho = rho * (T(1) - sp) + rho_target * sp;
    ux = ux * (T(1) - sp) + ux_target * sp;
    uy = uy * (T(1) - sp);
    uz = uz * (T(1) - sp);
    if (P.sponge_blend_distributions == 1) {
      for (int k = 0; k < Q; ++k) {
        T fe = feq_auto<T>(rho_target, ux_target, T(0), T(0), T(TB.w[k]), T(TB.cx[k]), T(TB.cy[k]), T(TB.cz[k]), comp);
        fs[k] = fs[k] * (T(1) - sp) + fe * sp;
      }
    }
  }
  T Fx = T(0), Fy = T(0), Fz = T(0);
  if (P.wall_model_active == 1 && L.wall_dist) {
    const T dist_wall = T(L.wall_dist[own]);
    if (dist_wall > T(0) && dist_wall < T(P.wall_model_max_distance)) {
      T u_mag = std::sqrt(ux * ux + uy * uy + uz * uz);
      T nu_visc = (T(P.tau) - T(0.5)) / T(3);
      if (u_mag > T(1e-6) && nu_visc > T(1e-10)) {
        T u_tau = u_mag * std::pow(nu_visc / (dist_wall * u_mag + T(1e-10)), T(1) / T(7)) *
                  std::pow(T(2) * T(8.3), -T(1) / T(7));
        u_tau = std::max(u_tau, T(1e-6));
        T y_p = u_tau * dist_wall / nu_visc;
        if (y_p > T(11.81)) {
          T u_plus_law = (T(1) / T(0.41)) * std::log(y_p) + T(5.2);
          if (u_plus_law > T(0.1)) {
            u_tau = u_tau * ((u_mag / u_tau) / u_plus_law);
            u_tau = std::max(u_tau, T(1e-6));
          }
        }
        T tau_wall = rho * u_tau * u_tau;
        T tau_res = rho * nu_visc * (u_mag / dist_wall);
        if (tau_wall > tau_res) {
          T force_mag = (tau_wall - tau_res) / dist_wall;
          Fx = -force_mag * ux / u_mag;
          Fy = -force_mag * uy / u_mag;
          Fz = -force_mag * uz / u_mag;
        }
      }
    }
  }
  const T ux_eq = ux + T(0.5) * Fx * inv_rho;
  const T uy_eq = uy + T(0.5) * Fy * inv_rho;
  const T uz_eq = uz + T(0.5) * Fz * inv_rho;
  vel_out[own] = ux; vel_out[own + cs] = uy; vel_out[own + 2 * cs] = uz;
  rho_out[own] = rho;

  // STEP 3: WALE (kernel_cumulant.jl:496-595), background path (variable_nu_sgs off)
  T uE[3], uW[3], uN[3], uS[3], uT[3], uB[3];
  vel_nb_fluid(L, vel_in, x, y, z, b, 1, 0, 0, uE[0], uE[1], uE[2]);
  vel_nb_fluid(L, vel_in, x, y, z, b, -1, 0, 0, uW[0], uW[1], uW[2]);
  vel_nb_fluid(L, vel_in, x, y, z, b, 0, 1, 0, uN[0], uN[1], uN[2]);
  vel_nb_fluid(L, vel_in, x, y, z, b, 0, -1, 0, uS[0], uS[1], uS[2]);
  vel_nb_fluid(L, vel_in, x, y, z, b, 0, 0, 1, uT[0], uT[1], uT[2]);
  vel_nb_fluid(L, vel_in, x, y, z, b, 0, 0, -1, uB[0], uB[1], uB[2]);
  const T h = T(0.5);
  const T g11 = h * (uE[0] - uW[0]), g12 = h * (uN[0] - uS[0]), g13 = h * (uT[0] - uB[0]);
  const T g21 = h * (uE[1] - uW[1]), g22 = h * (uN[1] - uS[1]), g23 = h * (uT[1] - uB[1]);
  const T g31 = h * (uE[2] - uW[2]), g32 = h * (uN[2] - uS[2]), g33 = h * (uT[2] - uB[2]);
  const T gsq11 = g11 * g11 + g12 * g21 + g13 * g31;
  const T gsq12 = g11 * g12 + g12 * g22 + g13 * g32;
  const T gsq13 = g11 * g13 + g12 * g23 + g13 * g33;
  const T gsq21 = g21 * g11 + g22 * g21 + g23 * g31;
  const T gsq22 = g21 * g12 + g22 * g22 + g23 * g32;
  const T gsq23 = g21 * g13 + g22 * g23 + g23 * g33;
  const T gsq31 = g31 * g11 + g32 * g21 + g33 * g31;
  const T gsq32 = g31 * g12 + g32 * g22 + g33 * g32;
  const T gsq33 = g31 * g13 + g32 * g23 + g33 * g33;
  const T tr_term = (gsq11 + gsq22 + gsq33) / T(3);
  const T Sd11 = gsq11 - tr_term, Sd22 = gsq22 - tr_term, Sd33 = gsq33 - tr_term;
  const T Sd12 = T(0.5) * (gsq12 + gsq21), Sd13 = T(0.5) * (gsq13 + gsq31), Sd23 = T(0.5) * (gsq23 + gsq32);
  const T S12 = T(0.5) * (g12 + g21), S13 = T(0.5) * (g13 + g31), S23 = T(0.5) * (g23 + g32);
  const T OP1 = Sd11 * Sd11 + Sd22 * Sd22 + Sd33 * Sd33 + T(2) * (Sd12 * Sd12 + Sd13 * Sd13 + Sd23 * Sd23);
  const T OP2 = g11 * g11 + g22 * g22 + g33 * g33 + T(2) * (S12 * S12 + S13 * S13 + S23 * S23);
  T nu_eddy = T(0);
  if (OP1 > T(1e-12)) {
    T OP1_32 = OP1 * std::sqrt(OP1);
    T OP2_52 = OP2 * OP2 * std::sqrt(std::max(OP2, T(1e-12)));
    T denom = OP2_52 + OP1 * std::sqrt(std::sqrt(std::max(OP1, T(1e-12))));
    if (denom > T(1e-12)) nu_eddy = (T(P.c_wale) * T(P.c_wale)) * OP1_32 / denom;
  }
  nu_eddy = nu_eddy * T(P.amr_sgs_scale);
  if (P.variable_nu_sgs == 2) {
    // Germano-Lilly dynamic coefficient (kernel_cumulant.jl:553-565)
    const T c[3] = {ux, uy, uz};
    T n[6][3];
    vel_nb_centre(L, vel_in, x, y, z, b, 1, 0, 0, ux, uy, uz, n[0]);
    vel_nb_centre(L, vel_in, x, y, z, b, -1, 0, 0, ux, uy, uz, n[1]);
    vel_nb_centre(L, vel_in, x, y, z, b, 0, 1, 0, ux, uy, uz, n[2]);
    vel_nb_centre(L, vel_in, x, y, z, b, 0, -1, 0, ux, uy, uz, n[3]);
    vel_nb_centre(L, vel_in, x, y, z, b, 0, 0, 1, ux, uy, uz, n[4]);
    vel_nb_centre(L, vel_in, x, y, z, b, 0, 0, -1, ux, uy, uz, n[5]);
    const T c_d = dynamic_cs2<T>(c, n, g11, g22, g33, S12, S13, S23);
    const T S_mag = std::sqrt(std::max(T(2) * (g11 * g11 + g22 * g22 + g33 * g33) +
                                       T(4) * (S12 * S12 + S13 * S13 + S23 * S23), T(1e-30)));
    const T stress = std::min(c_d * S_mag * T(P.amr_sgs_scale), T(0.1));
    nu_eddy = std::max(std::max(nu_eddy, stress), T(P.nu_sgs_floor) * T(P.amr_sgs_scale));
  } else if (P.variable_nu_sgs == 1) {
    // nu_sgs from the previous step's post-collision Pi_neq (kernel_cumulant.jl:566-586)
    const T* pn = static_cast<const T*>(L.pi_neq);
    const T pxx = pn[own], pyy = pn[own + cs], pzz = pn[own + 2 * cs];
    const T pxy = pn[own + 3 * cs], pxz = pn[own + 4 * cs], pyz = pn[own + 5 * cs];
    const T mag = std::sqrt(pxx * pxx + pyy * pyy + pzz * pzz + T(2) * (pxy * pxy + pxz * pxz + pyz * pyz));
    const T denom_tau = T(P.tau) - T(1);
    const T tau_corr = std::fabs(denom_tau) < T(1e-3) ? T(1) : T(P.tau) / denom_tau;
    const T pre = std::fabs(tau_corr) * mag;
    const T rho_cell = (!std::isfinite(rho) || rho < T(0.01)) ? T(1) : rho;
    const T stress = std::min(T(P.c_pi) * pre / (rho_cell * (T(1) / T(3)) + T(1e-10)) * T(P.amr_sgs_scale), T(0.1));
    nu_eddy = std::max(std::max(nu_eddy, stress), T(P.nu_sgs_floor) * T(P.amr_sgs_scale));
  } else {
    nu_eddy = std::max(nu_eddy, T(P.nu_sgs_background) * T(P.amr_sgs_scale));
  }
  const T nu_mol = (T(P.tau) - T(0.5)) / T(3);
  const T nu_eff = nu_mol + nu_eddy;
  const T tau_eff = T(0.5) + T(3) * nu_eff;
  const T omega1 = T(1) / std::max(tau_eff, T(0.500001));
  const T omega_bulk = T(P.omega_bulk), omega3 = T(P.omega3), omega4 = T(P.omega4);
  T omega4_diag = omega4;
  if (P.adaptive_omega4 == 1) {
    T om1_m2 = omega1 - T(2);
    T denom_adaptive = T(P.lambda_param) * omega1 + T(1e-10);
    T A_val = -(om1_m2 * om1_m2) / denom_adaptive;
    omega4_diag = std::min(std::max(A_val, T(0.01)), T(2));
  }

  // STEP 4: chimera forward (kernel_cumulant.jl:612-656); A index = (cx+1)+3(cy+1)+9(cz+1)
  T Am[Q];
  for (int k = 0; k < Q; ++k) Am[k] = fs[k];
  for (int iz = 0; iz < 3; ++iz)
    for (int iy = 0; iy < 3; ++iy) {
      int base = iy * 3 + iz * 9;
      chimera_forward(Am[base], Am[base + 1], Am[base + 2], ux_eq);
    }
  for (int iz = 0; iz < 3; ++iz)
    for (int ma = 0; ma < 3; ++ma)
      chimera_forward(Am[ma + iz * 9], Am[ma + 3 + iz * 9], Am[ma + 6 + iz * 9], uy_eq);
  for (int mb = 0; mb < 3; ++mb)
    for (int ma = 0; ma < 3; ++ma)
      chimera_forward(Am[ma + mb * 3], Am[ma + mb * 3 + 9], Am[ma + mb * 3 + 18], uz_eq);

  // STEP 5: central moments -> cumulants (kernel_cumulant.jl:661-699); 1-based A[n] = Am[n-1]
  const T k_000 = Am[0];
  const T k_200 = Am[2], k_020 = Am[6], k_002 = Am[18];
  const T k_110 = Am[4], k_101 = Am[10], k_011 = Am[12];
  const T k_210 = Am[5], k_120 = Am[7], k_201 = Am[11];
  const T k_021 = Am[15], k_102 = Am[19], k_012 = Am[21];
  const T k_111 = Am[13];
  const T k_220 = Am[8], k_202 = Am[20], k_022 = Am[24];
  const T k_211 = Am[14], k_121 = Am[16], k_112 = Am[22];
  const T inv_r = T(1) / std::max(k_000, T(0.01));
  const T c200 = k_200 * inv_r, c020 = k_020 * inv_r, c002 = k_002 * inv_r;
  const T c110 = k_110 * inv_r, c101 = k_101 * inv_r, c011 = k_011 * inv_r;
  const T c210 = k_210 * inv_r, c120 = k_120 * inv_r, c201 = k_201 * inv_r;
  const T c021 = k_021 * inv_r, c102 = k_102 * inv_r, c012 = k_012 * inv_r;
  const T c111 = k_111 * inv_r;
  const T c220n = k_220 * inv_r, c202n = k_202 * inv_r, c022n = k_022 * inv_r;
  const T c211n = k_211 * inv_r, c121n = k_121 * inv_r, c112n = k_112 * inv_r;
  const T C_220 = c220n - c200 * c020 - T(2) * c110 * c110;
  const T C_202 = c202n - c200 * c002 - T(2) * c101 * c101;
  const T C_022 = c022n - c020 * c002 - T(2) * c011 * c011;
  const T C_211 = c211n - c200 * c011 - T(2) * c110 * c101;
  const T C_121 = c121n - c020 * c101 - T(2) * c110 * c011;
  const T C_112 = c112n - c002 * c110 - T(2) * c101 * c011;

  // STEP 6: relaxation (kernel_cumulant.jl:705-754)
  // the reference's literal 0.333333333f0 rounds to the float nearest 1/3; 1/3 keeps that value in
  // float and is the intended constant in double
  const T cs2 = T(1) / T(3);
  const T D_trace = c200 + c020 + c002;
  const T D_trace_eq = T(3) * cs2;
  const T D_trace_s = (T(1) - omega_bulk) * D_trace + omega_bulk * D_trace_eq;
  const T D1 = c200 - c020, D2 = c200 - c002;
  const T D1_s = (T(1) - omega1) * D1, D2_s = (T(1) - omega1) * D2;
  const T c200_s = (D_trace_s + D1_s + D2_s) / T(3);
  const T c020_s = (D_trace_s - T(2) * D1_s + D2_s) / T(3);
  const T c002_s = (D_trace_s + D1_s - T(2) * D2_s) / T(3);
  T c110_s = (T(1) - omega1) * c110;
  T c101_s = (T(1) - omega1) * c101;
  T c011_s = (T(1) - omega1) * c011;
  if (P.limiter_type == 1) {
    T b110 = std::sqrt(std::max(c200_s * c020_s, T(0)));
    T b101 = std::sqrt(std::max(c200_s * c002_s, T(0)));
    T b011 = std::sqrt(std::max(c020_s * c002_s, T(0)));
    c110_s = std::min(std::max(c110_s, -b110), b110);
    c101_s = std::min(std::max(c101_s, -b101), b101);
    c011_s = std::min(std::max(c011_s, -b011), b011);
  }
  const T c210_s = (T(1) - omega3) * c210, c120_s = (T(1) - omega3) * c120;
  const T c201_s = (T(1) - omega3) * c201, c021_s = (T(1) - omega3) * c021;
  const T c102_s = (T(1) - omega3) * c102, c012_s = (T(1) - omega3) * c012;
  const T c111_s = (T(1) - omega3) * c111;
  const T C_220_s = (T(1) - omega4_diag) * C_220;
  const T C_202_s = (T(1) - omega4_diag) * C_202;
  const T C_022_s = (T(1) - omega4_diag) * C_022;
  const T C_211_s = (T(1) - omega4) * C_211;
  const T C_121_s = (T(1) - omega4) * C_121;
  const T C_112_s = (T(1) - omega4) * C_112;

  // STEP 7: reconstruction (kernel_cumulant.jl:759-781)
  const T c220_s = C_220_s + c200_s * c020_s + T(2) * c110_s * c110_s;
  const T c202_s = C_202_s + c200_s * c002_s + T(2) * c101_s * c101_s;
  const T c022_s = C_022_s + c020_s * c002_s + T(2) * c011_s * c011_s;
  const T c211_s = C_211_s + c200_s * c011_s + T(2) * c110_s * c101_s;
  const T c121_s = C_121_s + c020_s * c101_s + T(2) * c110_s * c011_s;
  const T c112_s = C_112_s + c002_s * c110_s + T(2) * c101_s * c011_s;
  const T c221_s = c200_s * c021_s + c020_s * c201_s + T(4) * c110_s * c111_s + T(2) * c101_s * c120_s +
                   T(2) * c011_s * c210_s;
  const T c212_s = c200_s * c012_s + c002_s * c210_s + T(2) * c110_s * c102_s + T(4) * c101_s * c111_s +
                   T(2) * c011_s * c201_s;
  const T c122_s = c020_s * c102_s + c002_s * c120_s + T(2) * c110_s * c012_s + T(4) * c011_s * c111_s +
                   T(2) * c101_s * c021_s;
  T c222_s = c200_s * C_022_s + c020_s * C_202_s + c002_s * C_220_s +
             T(4) * (c110_s * C_112_s + c101_s * C_121_s + c011_s * C_211_s);
  c222_s += T(2) * (c210_s * c012_s + c201_s * c021_s + c120_s * c102_s) + T(4) * c111_s * c111_s;
  c222_s += c200_s * c020_s * c002_s +
            T(2) * (c200_s * c011_s * c011_s + c020_s * c101_s * c101_s + c002_s * c110_s * c110_s) +
            T(8) * c110_s * c101_s * c011_s;

  // STEP 8: write back (kernel_cumulant.jl:786-804)
  const T r = k_000;
  Am[0] = r;
  Am[1] = T(0); Am[3] = T(0); Am[9] = T(0);
  Am[2] = r * c200_s; Am[6] = r * c020_s; Am[18] = r * c002_s;
  Am[4] = r * c110_s; Am[10] = r * c101_s; Am[12] = r * c011_s;
  Am[5] = r * c210_s; Am[7] = r * c120_s; Am[11] = r * c201_s;
  Am[15] = r * c021_s; Am[19] = r * c102_s; Am[21] = r * c012_s;
  Am[13] = r * c111_s;
  Am[8] = r * c220_s; Am[20] = r * c202_s; Am[24] = r * c022_s;
  Am[14] = r * c211_s; Am[16] = r * c121_s; Am[22] = r * c112_s;
  Am[17] = r * c221_s; Am[23] = r * c212_s; Am[25] = r * c122_s;
  Am[26] = r * c222_s;

  // STEP 9: chimera backward z, y, x (kernel_cumulant.jl:810-844)
  for (int mb = 0; mb < 3; ++mb)
    for (int ma = 0; ma < 3; ++ma)
      chimera_backward(Am[ma + mb * 3], Am[ma + mb * 3 + 9], Am[ma + mb * 3 + 18], uz_eq);
  for (int iz = 0; iz < 3; ++iz)
    for (int ma = 0; ma < 3; ++ma)
      chimera_backward(Am[ma + iz * 9], Am[ma + 3 + iz * 9], Am[ma + 6 + iz * 9], uy_eq);
  for (int iz = 0; iz < 3; ++iz)
    for (int iy = 0; iy < 3; ++iy) {
      int base = iy * 3 + iz * 9;
      chimera_backward(Am[base], Am[base + 1], Am[base + 2], ux_eq);
    }

  // positivity limiter (kernel_cumulant.jl:849-884)
  if (P.limiter_type == 2) {
    T fmin = Am[0];
    for (int k = 1; k < Q; ++k) fmin = std::min(fmin, Am[k]);
    if (fmin < T(0)) {
      T alpha = T(1);
      for (int k = 0; k < Q; ++k) {
        T fe = feq_auto<T>(rho, ux_eq, uy_eq, uz_eq, T(TB.w[k]), T(TB.cx[k]), T(TB.cy[k]), T(TB.cz[k]), comp);
        T fneq = Am[k] - fe;
        if (fneq < T(0) && fe > T(1e-15)) alpha = std::min(alpha, fe / (fe - fneq + T(1e-15)));
      }
      alpha = std::max(alpha, T(0));
      for (int k = 0; k < Q; ++k) {
        T fe = feq_auto<T>(rho, ux_eq, uy_eq, uz_eq, T(TB.w[k]), T(TB.cx[k]), T(TB.cy[k]), T(TB.cz[k]), comp);
        Am[k] = fe + alpha * (Am[k] - fe);
      }
    }
  }

  // STEP 10: Guo forcing + store (kernel_cumulant.jl:889-908)
  T fcs[Q];
  for (int k = 0; k < Q; ++k) {
    const T cxf = T(TB.cx[k]), cyf = T(TB.cy[k]), czf = T(TB.cz[k]);
    const T cu = cxf * ux_eq + cyf * uy_eq + czf * uz_eq;
    const T force_term = T(TB.w[k]) * T(3) *
                         ((cxf - ux + T(3) * cu * cxf) * Fx + (cyf - uy + T(3) * cu * cyf) * Fy +
                          (czf - uz + T(3) * cu * czf) * Fz);
    fcs[k] = Am[k] + (T(1) - T(0.5) * omega1) * force_term;
  }
  if (P.solid_bc == OAL_SOLID_GRAD && wall_cell) {
    // Grad-reconstruction wall (geometry/grad_wall_kernel.jl:62-144 with grad_vel_mode 0, called
    // from collision/timestep.jl:1738-1751 with omega_wall = 1/tau): rebuild every population of
    // a fluid cell with a wall-crossing link from (rho_out, u_wall = 0, Pi_neq of the
    // post-collision populations); the velocity output becomes the wall velocity.
    const T uw = T(0);
    T pxx = T(0), pyy = T(0), pzz = T(0), pxy = T(0), pyz = T(0), pzx = T(0);
    for (int k = 0; k < Q; ++k) {
      const T cxf = T(TB.cx[k]), cyf = T(TB.cy[k]), czf = T(TB.cz[k]);
      const T fe = feq2<T>(rho, uw, uw, uw, T(TB.w[k]), cxf, cyf, czf);
      const T fneq = fcs[k] - fe;
      pxx += fneq * cxf * cxf; pyy += fneq * cyf * cyf; pzz += fneq * czf * czf;
      pxy += fneq * cxf * cyf; pyz += fneq * cyf * czf; pzx += fneq * czf * cxf;
    }
    const T sc = T(P.grad_pineq_scale);
    pxx *= sc; pyy *= sc; pzz *= sc; pxy *= sc; pyz *= sc; pzx *= sc;
    const T cs2 = T(1) / T(3), inv_2cs4 = T(0.5) / (cs2 * cs2);
    const T one_m_w = T(1) - T(1) / T(P.tau);
    for (int k = 0; k < Q; ++k) {
      const T cxf = T(TB.cx[k]), cyf = T(TB.cy[k]), czf = T(TB.cz[k]), wk = T(TB.w[k]);
      const T fe = feq2<T>(rho, uw, uw, uw, wk, cxf, cyf, czf);
      const T qxx = cxf * cxf - cs2, qyy = cyf * cyf - cs2, qzz = czf * czf - cs2;
      const T reg = wk * inv_2cs4 *
                    (pxx * qxx + pyy * qyy + pzz * qzz + T(2) * (pxy * cxf * cyf + pyz * cyf * czf + pzx * czf * cxf));
      const T fc = fe + one_m_w * reg;
      fcs[k] = fc < T(1e-12) ? T(1e-12) : fc;  // max(fc, 1e-12), NaN passes
    }
    vel_out[own] = uw; vel_out[own + cs] = uw; vel_out[own + 2 * cs] = uw;
  }
  for (int k = 0; k < Q; ++k) {
    if (store_post) f_post[A.f(x, y, z, b, k)] = fcs[k];
    f_out[A.f(x, y, z, b, k)] = fcs[k];
  }
  if (pi_neq) {
    // refresh_pi_neq! after the step (timestep.jl:1828, solver_control.jl:152): the stored
    // populations against the stored macros
    T pv[6];
    pi_neq_cell<T>(fcs, rho_out[own], vel_out[own], vel_out[own + cs], vel_out[own + 2 * cs], comp, pv);
    for (int m = 0; m < 6; ++m) pi_neq[own + m * cs] = pv[m];
  }
}

template <class T>
int step_level(const Level& L, const oal_step_params& P, const T* f_in, T* f_out, T* f_post, T* rho_out,
               T* vel_out, const T* vel_in, double* force_out) {
  std::vector<double> part((size_t)L.nb * 3, 0.0);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < L.nb; ++b) {
    double acc[3] = {0, 0, 0};
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x)
          step_cell<T>(L, P, f_in, f_out, f_post, rho_out, vel_out, vel_in, b, x, y, z, acc);
    part[3 * b] = acc[0]; part[3 * b + 1] = acc[1]; part[3 * b + 2] = acc[2];
  }
  if (force_out && P.collect_forces) {
    double s[3] = {0, 0, 0};
    for (int b = 0; b < L.nb; ++b) { s[0] += part[3 * b]; s[1] += part[3 * b + 1]; s[2] += part[3 * b + 2]; }
    force_out[0] = s[0]; force_out[1] = s[1]; force_out[2] = s[2];
  }
  return 0;
}

// ---- restriction (amr_coupling.jl, default flags) --------------------------------------------
// solve_shell_moment4 (:130-176): 4x4 Gaussian elimination without pivoting
template <class T>
bool solve_shell_moment4(T m00, T m01, T m02, T m03, T m11, T m12, T m13, T m22, T m23, T m33, T r0, T r1, T r2,
                         T r3, T& x0, T& x1, T& x2, T& x3) {
  const T eps = T(1e-12);
  T a00 = m00 + eps, a01 = m01, a02 = m02, a03 = m03, b0 = r0;
  T a10 = m01, a11 = m11 + eps, a12 = m12, a13 = m13, b1 = r1;
  T a20 = m02, a21 = m12, a22 = m22 + eps, a23 = m23, b2 = r2;
  T a30 = m03, a31 = m13, a32 = m23, a33 = m33 + eps, b3 = r3;
  const T p0 = a00;
  const bool ok0 = std::fabs(p0) > eps;
  const T inv0 = ok0 ? T(1) / p0 : T(0);
  const T f10 = a10 * inv0, f20 = a20 * inv0, f30 = a30 * inv0;
  a11 -= f10 * a01; a12 -= f10 * a02; a13 -= f10 * a03; b1 -= f10 * b0;
  a21 -= f20 * a01; a22 -= f20 * a02; a23 -= f20 * a03; b2 -= f20 * b0;
  a31 -= f30 * a01; a32 -= f30 * a02; a33 -= f30 * a03; b3 -= f30 * b0;
  const T p1 = a11;
  const bool ok1 = std::fabs(p1) > eps;
  const T inv1 = ok1 ? T(1) / p1 : T(0);
  const T f21 = a21 * inv1, f31 = a31 * inv1;
  a22 -= f21 * a12; a23 -= f21 * a13; b2 -= f21 * b1;
  a32 -= f31 * a12; a33 -= f31 * a13; b3 -= f31 * b1;
  const T p2 = a22;
  const bool ok2 = std::fabs(p2) > eps;
  const T inv2 = ok2 ? T(1) / p2 : T(0);
  const T f32 = a32 * inv2;
  a33 -= f32 * a23; b3 -= f32 * b2;
  const T p3 = a33;
  const bool ok3 = std::fabs(p3) > eps;
  const T inv3 = ok3 ? T(1) / p3 : T(0);
  x3 = b3 * inv3;
  x2 = (b2 - a23 * x3) * inv2;
  x1 = (b1 - a12 * x2 - a13 * x3) * inv1;
  x0 = (b0 - a01 * x1 - a02 * x2 - a03 * x3) * inv0;
  return ok0 && ok1 && ok2 && ok3;
}

// tau_ratio_flow of restrict_fine_to_parent! (:7596-7615): (tau_p - 1/2)/(tau_c - 1/2), or the
// physical rule, times the post-collision factor (1 - omega_p)/(1 - omega_c)
template <class T>
T restrict_tau_ratio(T tau_p, T tau_c, int level_visc_physical) {
  const T tpc = std::max(tau_p - T(0.5), T(1e-6)), tcc = std::max(tau_c - T(0.5), T(1e-6));
  T r = std::min(std::max(tpc / tcc, T(0.01)), T(100));
  if (level_visc_physical == 1) r = std::min(std::max(T(2) * tau_p / std::max(tau_c, T(0.500001)), T(0.01)), T(100));
  const T omega_p = T(1) / std::max(tau_p, T(0.500001)), omega_c = T(1) / std::max(tau_c, T(0.500001));
  const T one_m_wp = T(1) - omega_p, one_m_wc = T(1) - omega_c;
  if (std::fabs(one_m_wc) > T(1e-6)) r = std::min(std::max(r * (one_m_wp / one_m_wc), T(0.01)), T(100));
  return r;
}

// restrict_child_state_to_parent_kernel! (:1900-3242) for one parent cell whose 8 children exist:
// children average, f = feq + ratio (avg - feq), two moment-correction passes, shell macros
template <class T>
void restrict_cell(int32_t pnb, const int32_t* pcoords, T* pf, T* prho, T* pvel, int32_t cnb, const int32_t* cptr,
                   int32_t cdx, int32_t cdy, int32_t cdz, const uint8_t* cobst, const T* cf, T ratio, int comp, int pb,
                   int lx, int ly, int lz) {
  const int64_t pn = 512 * (int64_t)pnb, cn = 512 * (int64_t)cnb;
  const int cbase_x = 2 * pcoords[3 * pb] - 1, cbase_y = 2 * pcoords[3 * pb + 1] - 1, cbase_z = 2 * pcoords[3 * pb + 2] - 1;
  int64_t ccell[8];
  int n = 0;
  for (int sx = 0; sx <= 1; ++sx)
    for (int sy = 0; sy <= 1; ++sy)
      for (int sz = 0; sz <= 1; ++sz) {
        const int fx = 2 * (lx - 1) + 1 + sx, fy = 2 * (ly - 1) + 1 + sy, fz = 2 * (lz - 1) + 1 + sz;
        const int cbx = cbase_x + (fx - 1) / BS, cby = cbase_y + (fy - 1) / BS, cbz = cbase_z + (fz - 1) / BS;
        if (cbx < 1 || cby < 1 || cbz < 1 || cbx > cdx || cby > cdy || cbz > cdz) return;
        const int32_t cb = cptr[(cbx - 1) + (int64_t)cdx * ((cby - 1) + (int64_t)cdy * (cbz - 1))];
        if (cb == 0) return;
        ccell[n++] = cidx((fx - 1) % BS, (fy - 1) % BS, (fz - 1) % BS) + 512 * (int64_t)(cb - 1);
      }
  T avg[Q];
  for (int k = 0; k < Q; ++k) avg[k] = T(0);
  int fluid = 0;
  for (int c = 0; c < 8; ++c) {
    if (cobst && cobst[ccell[c]]) continue;
    ++fluid;
    for (int k = 0; k < Q; ++k) avg[k] += cf[ccell[c] + cn * k];
  }
  if (fluid == 0) return;
  const T inv_children = T(1) / T(fluid);
  T rho_raw = T(0), jx = T(0), jy = T(0), jz = T(0);
  for (int k = 0; k < Q; ++k) {
    const T favg = avg[k] * inv_children;
    avg[k] = favg;
    rho_raw += favg;
    jx += favg * T(TB.cx[k]);
    jy += favg * T(TB.cy[k]);
    jz += favg * T(TB.cz[k]);
  }
  const T rho_p = std::max(rho_raw, T(0.01));
  const T inv_rho = T(1) / rho_p;
  const T ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  const int64_t pc = cidx(lx - 1, ly - 1, lz - 1) + 512 * (int64_t)pb;
  const T frac = T(1), one_m_frac = T(0);
  for (int k = 0; k < Q; ++k) {
    const T feq = feq_auto<T>(rho_p, ux, uy, uz, T(TB.w[k]), T(TB.cx[k]), T(TB.cy[k]), T(TB.cz[k]), comp);
    const T prior = pf[pc + pn * k];
    const T fr = feq + ratio * (avg[k] - feq);
    pf[pc + pn * k] = std::max(frac * fr + one_m_frac * prior, T(1e-10));
  }
  T m00 = 0, m01 = 0, m02 = 0, m03 = 0, m11 = 0, m12 = 0, m13 = 0, m22 = 0, m23 = 0, m33 = 0;
  for (int k = 0; k < Q; ++k) {
    const T cx = T(TB.cx[k]), cy = T(TB.cy[k]), cz = T(TB.cz[k]), w = T(TB.w[k]);
    m00 += w; m01 += w * cx; m02 += w * cy; m03 += w * cz;
    m11 += w * cx * cx; m12 += w * cx * cy; m13 += w * cx * cz;
    m22 += w * cy * cy; m23 += w * cy * cz; m33 += w * cz * cz;
  }
  const T inv_cs2 = T(1) / std::max(T(1.0 / 3.0), T(1e-6));
  for (int pass = 0; pass < 2; ++pass) {  // AMR_RESTRICTION_CORRECTION_PASSES = 2
    T rr = T(0), rx = T(0), ry = T(0), rz = T(0);
    for (int k = 0; k < Q; ++k) {
      const T v = pf[pc + pn * k];
      rr += v; rx += v * T(TB.cx[k]); ry += v * T(TB.cy[k]); rz += v * T(TB.cz[k]);
    }
    const T dr = rho_p - rr, dx = jx - rx, dy = jy - ry, dz = jz - rz;
    if (std::fabs(dr) > T(1e-12) || std::fabs(dx) > T(1e-12) || std::fabs(dy) > T(1e-12) || std::fabs(dz) > T(1e-12)) {
      T c0, c1, c2, c3;
      const bool ok = solve_shell_moment4<T>(m00, m01, m02, m03, m11, m12, m13, m22, m23, m33, dr, dx, dy, dz, c0, c1, c2, c3);
      for (int k = 0; k < Q; ++k) {
        const T cx = T(TB.cx[k]), cy = T(TB.cy[k]), cz = T(TB.cz[k]), w = T(TB.w[k]);
        const T delta = ok ? w * (c0 + c1 * cx + c2 * cy + c3 * cz) : w * (dr + inv_cs2 * (cx * dx + cy * dy + cz * dz));
        pf[pc + pn * k] = std::max(pf[pc + pn * k] + delta, T(1e-10));
      }
    }
  }
  T rs = T(0), sx = T(0), sy = T(0), sz = T(0);
  for (int k = 0; k < Q; ++k) {
    const T v = pf[pc + pn * k];
    rs += v; sx += v * T(TB.cx[k]); sy += v * T(TB.cy[k]); sz += v * T(TB.cz[k]);
  }
  const T rho_s = std::max(rs, T(0.01));
  const T inv_s = T(1) / rho_s;
  prho[pc] = rho_s;
  pvel[pc] = sx * inv_s; pvel[pc + pn] = sy * inv_s; pvel[pc + 2 * pn] = sz * inv_s;
}

template <class T>
void restrict_level(int32_t pnb, const int32_t* pcoords, T* pf, T* prho, T* pvel, int32_t cnb, const int32_t* cptr,
                    int32_t cdx, int32_t cdy, int32_t cdz, const uint8_t* cobst, const T* cf, T tau_p, T tau_c, int comp,
                    int level_visc_physical) {
  const T ratio = restrict_tau_ratio<T>(tau_p, tau_c, level_visc_physical);
#pragma omp parallel for schedule(static)
  for (int pb = 0; pb < pnb; ++pb)
    for (int lz = 1; lz <= BS; ++lz)
      for (int ly = 1; ly <= BS; ++ly)
        for (int lx = 1; lx <= BS; ++lx)
          restrict_cell<T>(pnb, pcoords, pf, prho, pvel, cnb, cptr, cdx, cdy, cdz, cobst, cf, ratio, comp, pb, lx, ly, lz);
}

Level make_level(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords, const int32_t* nbr,
                 const uint8_t* obstacle, const float* sponge, const float* wall_dist) {
  return Level{nb, nx, ny, nz, coords, nbr, obstacle, sponge, wall_dist};
}

// Characteristic outlet (apply_nscbc_outlet_kernel!, kernel_nscbc_outlet.jl:80-340; driver
// apply_nscbc_outlet!, :343-393), athermal (T = 1): for every face cell x = 8 (1-based) of the
// blocks on the +x face (or of every block, the range the reference's driver launches) whose
// cell and interior neighbour x = 7 are fluid, in the reference's operation order.
template <class T>
void nscbc_outlet(const Level& L, int all_blocks, float p_target, float sigma, float blend, T* f, T* rho, T* vel) {
  Arr<T> A{L.nb};
  const int64_t cs = 512 * (int64_t)L.nb;
  int bxmax = 0;
  for (int b = 0; b < L.nb; ++b) bxmax = std::max(bxmax, L.coords[3 * b]);
  const float c_ref = std::sqrt(1.0f * float(2.0 / 3.0));
  const float k_relax = sigma * c_ref / std::max(float(L.nx), 1.0f);
  for (int b = 0; b < L.nb; ++b) {
    if (!all_blocks && L.coords[3 * b] != bxmax) continue;
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y) {
        const int64_t of = A.s(7, y, z, b), oi = A.s(6, y, z, b);
        if (L.obstacle && (L.obstacle[of] || L.obstacle[oi])) continue;
        const int gy = (L.coords[3 * b + 1] - 1) * BS + y + 1, gz = (L.coords[3 * b + 2] - 1) * BS + z + 1;
        const bool corner = gy == 1 || gy == L.ny || gz == 1 || gz == L.nz;
        const T rf = rho[of], uf = vel[of], vf = vel[of + cs], wf = vel[of + 2 * cs];
        const T ri = rho[oi], ui = vel[oi], vi = vel[oi + cs], wi = vel[oi + 2 * cs];
        const T Ru = T(1) / T(3), Tt = T(1);
        const T pf = rf * Ru * Tt, pi = ri * Ru * Tt;
        const T c = std::sqrt(std::max(T(1) * Ru * Tt, T(1e-12)));
        const T drho = rf - ri, du = uf - ui, dv = vf - vi, dw = wf - wi, dp = pf - pi;
        const T un = uf;
        const T mach = un / std::max(c, T(1e-6));
        T L1 = (un - c) * (dp - rf * c * du);
        const T L2 = un * (c * c * drho - dp);
        const T L3 = corner ? T(0) : un * dv;
        const T L4 = corner ? T(0) : un * dw;
        const T L5 = (un + c) * (dp + rf * c * du);
        if (mach < T(1) && un > T(0)) {
          const T mc = std::min(std::max(mach, T(0.05f)), T(0.95f));
          L1 = T(k_relax) * (T(1) - mc * mc) * (pf - T(p_target));
        }
        const T d1 = (T(1) / (c * c)) * (L2 + T(0.5) * (L5 + L1));
        const T d2 = T(0.5) * (L5 + L1);
        const T d3 = (L5 - L1) / (T(2) * rf * c + T(1e-12));
        auto cl = [](T x, T lo, T hi) { return x > hi ? hi : (x < lo ? lo : x); };
        const T cap = corner ? T(0.10f) : T(0.20f);
        const T d1c = cl(d1, -cap * rf, cap * rf), d2c = cl(d2, T(-0.10f) * pf, T(0.10f) * pf);
        const T d3c = cl(d3, T(-0.10f) * c, T(0.10f) * c);
        const T L3c = cl(L3, T(-0.10f) * c, T(0.10f) * c), L4c = cl(L4, T(-0.10f) * c, T(0.10f) * c);
        T rn = rf - d1c;
        const T un2 = uf - d3c;
        const T vn = corner ? vi : vf - L3c;
        const T wn = corner ? wi : wf - L4c;
        T pn = pf - d2c;
        rn = cl(rn, T(0.1f), T(10));
        pn = std::max(pn, T(1e-6));
        const T Tn = cl(pn / (rn * Ru + T(1e-12)), T(0.1f), T(10));
        rho[of] = rn;
        vel[of] = un2; vel[of + cs] = vn; vel[of + 2 * cs] = wn;
        const T inv_n = T(1) / std::max(Ru * Tn, T(1e-12)), inv_i = T(1) / std::max(Ru * Tt, T(1e-12));
        const T usq_n = un2 * un2 + vn * vn + wn * wn, usq_i = ui * ui + vi * vi + wi * wi;
        for (int k = 0; k < Q; ++k) {
          const T cx = T(TB.cx[k]), cy = T(TB.cy[k]), cz = T(TB.cz[k]), w = T(TB.w[k]);
          const T cun = cx * un2 + cy * vn + cz * wn;
          const T fen = std::max(rn * w * (T(1) + cun * inv_n + T(0.5) * cun * cun * inv_n * inv_n - T(0.5) * usq_n * inv_n), T(1e-15));
          const T cui = cx * ui + cy * vi + cz * wi;
          const T fei = std::max(ri * w * (T(1) + cui * inv_i + T(0.5) * cui * cui * inv_i * inv_i - T(0.5) * usq_i * inv_i), T(1e-15));
          f[A.f(7, y, z, b, k)] = fen + T(blend) * (f[A.f(6, y, z, b, k)] - fei);
        }
      }
  }
}

// Spectral vanishing viscosity post-pass (apply_svv_d3q19_postcollision!, kernel_svv_yz_d3q39.jl:
// 426-458, with apply_svv_d3q19_inline!, :301-375, and the tap helpers get_pop_neighbor_x/_yz,
// :225-250 and :78-116): for every fluid cell, each post-collision population f_k is filtered by
// the 5-point bi-Laplacian of the step's INPUT populations along x (eps_x) and along y and z
// (eps_yz), the centre tap being f_k itself; a tap in a solid cell or past a missing neighbour
// block reads the cell's own input population. The 4-moment correction
// f_k -= w_k (drho + c_k . dj / cs2) restores the cell's mass and momentum, then every population
// is floored at 1e-12. f_out is filtered in place; f_post2, when given, receives the same values
// (the reference's write of f_post_collision on a level with boundary cells).
template <class T>
void svv_post(const Level& L, float eps_x, float eps_yz, const T* f_in, T* f_out, T* f_post2) {
  if (eps_x == 0.0f && eps_yz == 0.0f) return;
  Arr<T> A{L.nb};
  const T ex = T(eps_x), eyz = T(eps_yz);
  const T inv_cs2 = T(1) / T(1.0 / 3.0);  // CS2_LATTICE
  auto solid = [&](int x, int y, int z, int b) { return L.obstacle && L.obstacle[A.s(x, y, z, b)]; };
  // the input population k at (x, y, z) + d (one axis), with the fall-backs of the tap helpers
  auto tap = [&](int x, int y, int z, int b, int dx, int dy, int dz, int k) -> T {
    const int nx = x + dx, ny = y + dy, nz = z + dz;
    const int ox = nx < 0 ? -1 : (nx >= BS ? 1 : 0), oy = ny < 0 ? -1 : (ny >= BS ? 1 : 0),
              oz = nz < 0 ? -1 : (nz >= BS ? 1 : 0);
    if (ox == 0 && oy == 0 && oz == 0)
      return solid(nx, ny, nz, b) ? f_in[A.f(x, y, z, b, k)] : f_in[A.f(nx, ny, nz, b, k)];
    const int nbb = L.nbr[b + (int64_t)L.nb * ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))];
    if (nbb == 0) return f_in[A.f(x, y, z, b, k)];
    const int lx = nx - BS * ox, ly = ny - BS * oy, lz = nz - BS * oz;
    if (solid(lx, ly, lz, nbb - 1)) return f_in[A.f(x, y, z, b, k)];
    return f_in[A.f(lx, ly, lz, nbb - 1, k)];
  };
#pragma omp parallel for schedule(static)
  for (int b = 0; b < L.nb; ++b)
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) {
          if (solid(x, y, z, b)) continue;
          T fl[Q];
          T d_rho = T(0), d_jx = T(0), d_jy = T(0), d_jz = T(0);
          for (int k = 0; k < Q; ++k) {
            const T fc = f_out[A.f(x, y, z, b, k)];
            T bilap = T(0);
            if (eps_x > 0.0f)
              bilap += ex * (tap(x, y, z, b, -2, 0, 0, k) - T(4) * tap(x, y, z, b, -1, 0, 0, k) + T(6) * fc -
                             T(4) * tap(x, y, z, b, 1, 0, 0, k) + tap(x, y, z, b, 2, 0, 0, k));
            if (eps_yz > 0.0f) {
              bilap += eyz * (tap(x, y, z, b, 0, -2, 0, k) - T(4) * tap(x, y, z, b, 0, -1, 0, k) + T(6) * fc -
                              T(4) * tap(x, y, z, b, 0, 1, 0, k) + tap(x, y, z, b, 0, 2, 0, k));
              bilap += eyz * (tap(x, y, z, b, 0, 0, -2, k) - T(4) * tap(x, y, z, b, 0, 0, -1, k) + T(6) * fc -
                              T(4) * tap(x, y, z, b, 0, 0, 1, k) + tap(x, y, z, b, 0, 0, 2, k));
            }
            const T ff = fc - bilap;
            const T diff = ff - fc;
            d_rho += diff;
            d_jx += diff * T(TB.cx[k]);
            d_jy += diff * T(TB.cy[k]);
            d_jz += diff * T(TB.cz[k]);
            fl[k] = ff;
          }
          for (int k = 0; k < Q; ++k) {
            const T cu = T(TB.cx[k]) * d_jx + T(TB.cy[k]) * d_jy + T(TB.cz[k]) * d_jz;
            fl[k] -= T(TB.w[k]) * (d_rho + inv_cs2 * cu);
            const T fc = fl[k] < T(1e-12f) ? T(1e-12f) : fl[k];
            f_out[A.f(x, y, z, b, k)] = fc;
            if (f_post2) f_post2[A.f(x, y, z, b, k)] = fc;
          }
        }
}

}  // namespace

// ---- linear Bouzidi wall (geometry/bouzidi_kernel.jl:150-380, default D3Q27 options) ---------
// bouzidi_correction_kernel_fixed! on the unshifted lattice (out_k = opp k, shifted-wall scale 0):
// for every listed fluid cell x and link k with q_min < q <= 1, from the post-collision
// populations f* of the step, f_out[x, opp k] =
//   q < 1/2:  2q f*_k(x) + (1-2q) f*_k(x_ff), x_ff = x + c_{opp k} when it exists and is fluid,
//             else (ff_fallback) 0: f*_k(x), 1: w_k rho_f, 2: f*_{opp k}(x)        (:223-287)
//   q >= 1/2: f*_k(x)/(2q) + (2q-1)/(2q) f*_{opp k}(x)                             (:320-328)
// then, with a limiter cap > 0, clamp to w_{opp k} rho_f +- max(abs, rel max(|.|, 1e-12)) and
// floor at 1e-12 (_limit_wall_population, :65-87); rho_f = sum of f*(x) in direction order.
// cells: n x 4 int32 (block, x, y, z), 1-based like the reference's bouzidi_cell_* arrays.
template <class T>
void bouzidi_linear(const Level& L, int32_t n, const int32_t* cells, const float* q, float q_min, int ff,
                    float rel_cap, float abs_cap, const T* fpost, T* fout) {
  Arr<T> A{L.nb};
  for (int32_t i = 0; i < n; ++i) {
    const int b = cells[4 * i] - 1, x = cells[4 * i + 1] - 1, y = cells[4 * i + 2] - 1, z = cells[4 * i + 3] - 1;
    bool rho_valid = false;
    T rho_f = T(0);
    auto density = [&]() {
      if (!rho_valid) {
        T s = T(0);
        for (int kk = 0; kk < Q; ++kk) s += fpost[A.f(x, y, z, b, kk)];
        rho_f = s;
        rho_valid = true;
      }
      return rho_f;
    };
    for (int k = 0; k < Q; ++k) {
      const float qf = q[(size_t)i * Q + k];
      if (!(qf > q_min && qf <= 1.0f)) continue;
      const int ok = TB.opp[k];
      const T qq = T(qf);
      const T fk = fpost[A.f(x, y, z, b, k)];
      T raw;
      if (qq < T(0.5)) {
        const int nx = x + TB.cx[ok], ny = y + TB.cy[ok], nz = z + TB.cz[ok];
        T fff = fk;
        bool have = false;
        if (nx >= 0 && nx < BS && ny >= 0 && ny < BS && nz >= 0 && nz < BS) {
          if (!(L.obstacle && L.obstacle[A.s(nx, ny, nz, b)])) { fff = fpost[A.f(nx, ny, nz, b, k)]; have = true; }
        } else {
          const int ox = nx < 0 ? -1 : (nx >= BS ? 1 : 0), oy = ny < 0 ? -1 : (ny >= BS ? 1 : 0),
                    oz = nz < 0 ? -1 : (nz >= BS ? 1 : 0);
          const int dir = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1);
          const int nbb = L.nbr[b + (int64_t)L.nb * dir];
          if (nbb > 0) {
            const int lx = nx - BS * ox, ly = ny - BS * oy, lz = nz - BS * oz;
            if (!(L.obstacle && L.obstacle[A.s(lx, ly, lz, nbb - 1)])) {
              fff = fpost[A.f(lx, ly, lz, nbb - 1, k)];
              have = true;
            }
          }
        }
        if (!have && ff == 1) fff = density() * T(TB.w[k]);
        else if (!have && ff == 2) fff = fpost[A.f(x, y, z, b, ok)];
        const T c1 = T(2) * qq;
        raw = c1 * fk + (T(1) - c1) * fff;
      } else {
        const T fo = fpost[A.f(x, y, z, b, ok)];
        const T inv_2q = T(1) / (T(2) * qq);
        const T c2 = (T(2) * qq - T(1)) * inv_2q;
        raw = inv_2q * fk + c2 * fo;
      }
      if (rel_cap > 0.0f || abs_cap > 0.0f) {
        const T target = density() * T(TB.w[ok]);
        const T scale = std::max(std::fabs(target), T(1e-12f));
        const T cap = std::max(T(abs_cap), T(rel_cap) * scale);
        const T lo = target - cap, hi = target + cap;
        raw = raw > hi ? hi : (raw < lo ? lo : raw);
        raw = raw < T(1e-12f) ? T(1e-12f) : raw;
      }
      fout[A.f(x, y, z, b, ok)] = raw;
    }
  }
}

extern "C" {

// Configuration defaults of the cumulant level step (src/io/config_loader.jl:1305-1380,
// src/collision/timestep.jl:1127), so that CPU-only callers need nothing from the product library.
void ora_default_step_params(oal_step_params* p) {
  std::memset(p, 0, sizeof *p);
  p->abi_version = OAL_ABI_VERSION;
  p->operator_id = OAL_OP_CUMULANT_D3Q27;
  p->tau = 0.6f;
  p->tau_parent = 0.6f;
  p->c_wale = 0.20f;                 // config_loader.jl:1305
  p->amr_sgs_scale = 1.0f;           // timestep.jl:1127
  p->omega_bulk = 1.0f;              // config_loader.jl:1373
  p->omega3 = 1.0f;                  // :1374
  p->omega4 = 1.0f;                  // :1375
  p->adaptive_omega4 = 1;            // :1376
  p->lambda_param = 1.0f / 6.0f;     // :1377
  p->limiter_type = OAL_LIMITER_FACTORED;  // :1379
  p->u_inlet = 0.05f;
  p->wall_model_max_distance = 10.0f;
  p->transverse_freestream_blend = 1.0f;
  p->solid_bc = OAL_SOLID_FULLWAY;
  p->temporal_weight = 1.0f;
  p->hrr_sigma = 1.0f;
  p->grad_pineq_scale = 1.0f;        // config_loader.jl:898
  p->variable_nu_sgs = 0;            // VARIABLE_NU_SGS, config_loader.jl:237
  p->c_pi = 0.2f;                    // :238
  p->nu_sgs_floor = 0.002f;          // :239
}

// D3Q27 tables in the reference order (0-based indices for opp/mirrors).
void ora_d3q27_tables(int32_t* cx, int32_t* cy, int32_t* cz, double* w, int32_t* opp, int32_t* mir_y,
                      int32_t* mir_z) {
  for (int k = 0; k < Q; ++k) {
    cx[k] = TB.cx[k]; cy[k] = TB.cy[k]; cz[k] = TB.cz[k]; w[k] = TB.w[k];
    opp[k] = TB.opp[k]; mir_y[k] = TB.mir_y[k]; mir_z[k] = TB.mir_z[k];
  }
}

// domain.jl:785 sorted tuples (bx most significant) + domain_topology.jl:919-953 with a wrap
// on each axis whose bit is set in periodic_mask (the reference wraps y only; a full wrap makes
// the same kernel a periodic box).
int ora_build_box(int32_t bxm, int32_t bym, int32_t bzm, int32_t periodic_mask, int32_t* coords, int32_t* nbr) {
  const int64_t n = (int64_t)bxm * bym * bzm;
  std::vector<int32_t> ptr((size_t)n, 0);
  int64_t i = 0;
  for (int bx = 1; bx <= bxm; ++bx)
    for (int by = 1; by <= bym; ++by)
      for (int bz = 1; bz <= bzm; ++bz) {
        coords[3 * i] = bx; coords[3 * i + 1] = by; coords[3 * i + 2] = bz;
        ptr[((size_t)(bx - 1) * bym + (by - 1)) * bzm + (bz - 1)] = (int32_t)(i + 1);
        ++i;
      }
  auto wrap = [](int v, int m, bool p) { return p ? (v < 1 ? m : (v > m ? 1 : v)) : v; };
  for (int64_t b = 0; b < n; ++b) {
    int bx = coords[3 * b], by = coords[3 * b + 1], bz = coords[3 * b + 2];
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int dir = (dx + 1) + (dy + 1) * 3 + (dz + 1) * 9;
          int nx = wrap(bx + dx, bxm, periodic_mask & 1);
          int ny = wrap(by + dy, bym, periodic_mask & 2);
          int nz = wrap(bz + dz, bzm, periodic_mask & 4);
          int32_t v = 0;
          if (nx >= 1 && nx <= bxm && ny >= 1 && ny <= bym && nz >= 1 && nz <= bzm)
            v = ptr[((size_t)(nx - 1) * bym + (ny - 1)) * bzm + (nz - 1)];
          nbr[b + n * dir] = v;
        }
  }
  return 0;
}

// domain_generation.jl:140-150 with dx = 1 (cell units)
int64_t ora_sphere(int32_t nb, const int32_t* coords, double cx, double cy, double cz, double radius,
                   uint8_t* obstacle) {
  const double r2 = radius * radius;
  int64_t count = 0;
  for (int b = 0; b < nb; ++b) {
    int bx = coords[3 * b], by = coords[3 * b + 1], bz = coords[3 * b + 2];
    for (int lz = 1; lz <= BS; ++lz)
      for (int ly = 1; ly <= BS; ++ly)
        for (int lx = 1; lx <= BS; ++lx) {
          double px = ((bx - 1) * BS + lx - 0.5), py = ((by - 1) * BS + ly - 0.5), pz = ((bz - 1) * BS + lz - 0.5);
          double d = (px - cx) * (px - cx) + (py - cy) * (py - cy) + (pz - cz) * (pz - cz);
          uint8_t s = d <= r2 ? 1 : 0;
          obstacle[(lx - 1) + 8 * (ly - 1) + 64 * (lz - 1) + 512 * (int64_t)b] = s;
          count += s;
        }
  }
  return count;
}

// Equilibrium start f = feq(rho, u) (physics_utils.jl:30-35 / :65-95).
void ora_init_feq_f64(int32_t nb, const double* rho, const double* vel, int32_t comp, double* f) {
  const int64_t n = 512 * (int64_t)nb;
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < Q; ++k)
      f[i + n * k] = feq_auto<double>(rho[i], vel[i], vel[i + n], vel[i + 2 * n], TB.w[k], TB.cx[k], TB.cy[k],
                                       TB.cz[k], comp);
}

int ora_step_d3q27_f64(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords, const int32_t* nbr,
                       const uint8_t* obstacle, const float* sponge, const float* wall_dist,
                       const oal_step_params* P, const double* f_in, double* f_out, double* f_post,
                       double* rho_out, double* vel_out, const double* vel_in, double* force_out) {
  Level L = make_level(nb, nx, ny, nz, coords, nbr, obstacle, sponge, wall_dist);
  return step_level<double>(L, *P, f_in, f_out, f_post, rho_out, vel_out, vel_in, force_out);
}

int ora_step_d3q27_f32(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords, const int32_t* nbr,
                       const uint8_t* obstacle, const float* sponge, const float* wall_dist,
                       const oal_step_params* P, const float* f_in, float* f_out, float* f_post,
                       float* rho_out, float* vel_out, const float* vel_in, double* force_out) {
  Level L = make_level(nb, nx, ny, nz, coords, nbr, obstacle, sponge, wall_dist);
  return step_level<float>(L, *P, f_in, f_out, f_post, rho_out, vel_out, vel_in, force_out);
}

// The level step with variable nu_sgs: pi_neq (T[6][512 * nb], xx yy zz xy xz yz; mode 1) holds
// the previous step's Pi_neq on entry and this step's on return; f_post may be null.
int ora_step_d3q27_pi_f64(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords, const int32_t* nbr,
                          const uint8_t* obstacle, const float* sponge, const float* wall_dist,
                          const oal_step_params* P, const double* f_in, double* f_out, double* f_post, double* rho_out,
                          double* vel_out, const double* vel_in, double* pi_neq, double* force_out) {
  Level L = make_level(nb, nx, ny, nz, coords, nbr, obstacle, sponge, wall_dist);
  L.pi_neq = pi_neq;
  if (P->variable_nu_sgs == 1 && !pi_neq) return -1;
  return step_level<double>(L, *P, f_in, f_out, f_post, rho_out, vel_out, vel_in, force_out);
}

int ora_step_d3q27_pi_f32(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords, const int32_t* nbr,
                          const uint8_t* obstacle, const float* sponge, const float* wall_dist,
                          const oal_step_params* P, const float* f_in, float* f_out, float* f_post, float* rho_out,
                          float* vel_out, const float* vel_in, float* pi_neq, double* force_out) {
  Level L = make_level(nb, nx, ny, nz, coords, nbr, obstacle, sponge, wall_dist);
  L.pi_neq = pi_neq;
  if (P->variable_nu_sgs == 1 && !pi_neq) return -1;
  return step_level<float>(L, *P, f_in, f_out, f_post, rho_out, vel_out, vel_in, force_out);
}

void ora_nscbc_outlet_f64(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords, const uint8_t* obstacle,
                          int32_t all_blocks, float p_target, float sigma, float blend, double* f, double* rho, double* vel) {
  Level L = make_level(nb, nx, ny, nz, coords, nullptr, obstacle, nullptr, nullptr);
  nscbc_outlet<double>(L, all_blocks, p_target, sigma, blend, f, rho, vel);
}

void ora_nscbc_outlet_f32(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords, const uint8_t* obstacle,
                          int32_t all_blocks, float p_target, float sigma, float blend, float* f, float* rho, float* vel) {
  Level L = make_level(nb, nx, ny, nz, coords, nullptr, obstacle, nullptr, nullptr);
  nscbc_outlet<float>(L, all_blocks, p_target, sigma, blend, f, rho, vel);
}

// The spectral vanishing viscosity post-pass on a stepped level: f_in the step's input, f_out its
// output (filtered in place), f_post2 null or a second array to receive the filtered values.
void ora_svv_d3q27_f64(int32_t nb, const int32_t* nbr, const uint8_t* obstacle, float eps_x, float eps_yz,
                       const double* f_in, double* f_out, double* f_post2) {
  Level L = make_level(nb, 0, 0, 0, nullptr, nbr, obstacle, nullptr, nullptr);
  svv_post<double>(L, eps_x, eps_yz, f_in, f_out, f_post2);
}

void ora_svv_d3q27_f32(int32_t nb, const int32_t* nbr, const uint8_t* obstacle, float eps_x, float eps_yz,
                       const float* f_in, float* f_out, float* f_post2) {
  Level L = make_level(nb, 0, 0, 0, nullptr, nbr, obstacle, nullptr, nullptr);
  svv_post<float>(L, eps_x, eps_yz, f_in, f_out, f_post2);
}

// Pi_neq of a stored state (compute_pi_neq_kernel!, kernel_pi_neq.jl:39-180, D3Q27): out
// double[6][512 * nb]; a solid cell enters with a non-finite density, which the unphysical-state
// test zeroes.
void ora_pi_neq_f64(int32_t nb, const uint8_t* obstacle, const double* f, const double* rho, const double* vel,
                    int32_t comp, double* out) {
  const int64_t n = 512 * (int64_t)nb;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double fk[Q], pv[6];
    for (int k = 0; k < Q; ++k) fk[k] = f[i + n * k];
    const bool obs = obstacle && obstacle[i];
    pi_neq_cell<double>(fk, obs ? std::nan("") : rho[i], vel[i], vel[i + n], vel[i + 2 * n], comp, pv);
    for (int m = 0; m < 6; ++m) out[i + m * n] = pv[m];
  }
}

// A refined level's step: the level step with its pulls from outside its blocks interpolated from
// the parent. parent_ptr: (pdx, pdy, pdz) Julia column-major, 1-based parent block or 0;
// parent arrays in the parent level's reference layout (pnb blocks); the *_old arrays may be null.
int ora_step_d3q27_refined_f64(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords,
                               const int32_t* nbr, const uint8_t* obstacle, const oal_step_params* P,
                               const double* f_in, double* f_out, double* rho_out, double* vel_out,
                               const double* vel_in, double* force_out, int32_t pnb, const int32_t* pptr, int32_t pdx,
                               int32_t pdy, int32_t pdz, const double* pf_new, const double* prho_new,
                               const double* pvel_new, const double* pf_old, const double* prho_old,
                               const double* pvel_old, double tau_parent, double tw, int32_t use_temporal) {
  Parent<double> PP{pf_new, prho_new, pvel_new, pf_old, prho_old, pvel_old, pptr, pdx, pdy, pdz, pnb,
                    (double)tau_parent, (double)P->tau, tw, use_temporal, P->compressible_corr, P->level_visc_physical};
  Level L = make_level(nb, nx, ny, nz, coords, nbr, obstacle, nullptr, nullptr);
  L.parent = &PP;
  return step_level<double>(L, *P, f_in, f_out, nullptr, rho_out, vel_out, vel_in, force_out);
}

int ora_step_d3q27_refined_f32(int32_t nb, int32_t nx, int32_t ny, int32_t nz, const int32_t* coords,
                               const int32_t* nbr, const uint8_t* obstacle, const oal_step_params* P,
                               const float* f_in, float* f_out, float* rho_out, float* vel_out, const float* vel_in,
                               double* force_out, int32_t pnb, const int32_t* pptr, int32_t pdx, int32_t pdy,
                               int32_t pdz, const float* pf_new, const float* prho_new, const float* pvel_new,
                               const float* pf_old, const float* prho_old, const float* pvel_old, double tau_parent,
                               double tw, int32_t use_temporal) {
  Parent<float> PP{pf_new, prho_new, pvel_new, pf_old, prho_old, pvel_old, pptr, pdx, pdy, pdz, pnb,
                   (float)tau_parent, P->tau, (float)tw, use_temporal, P->compressible_corr, P->level_visc_physical};
  Level L = make_level(nb, nx, ny, nz, coords, nbr, obstacle, nullptr, nullptr);
  L.parent = &PP;
  return step_level<float>(L, *P, f_in, f_out, nullptr, rho_out, vel_out, vel_in, force_out);
}

// restrict_fine_to_parent! on the parent's current arrays (reference layout): every parent cell
// whose 8 children exist. child_ptr: (cdx, cdy, cdz) Julia column-major, 1-based child block or 0.
void ora_restrict_d3q27_f64(int32_t pnb, const int32_t* pcoords, double* pf, double* prho, double* pvel,
                            int32_t cnb, const int32_t* cptr, int32_t cdx, int32_t cdy, int32_t cdz,
                            const uint8_t* cobst, const double* cf, double tau_p, double tau_c, int32_t comp,
                            int32_t level_visc_physical) {
  restrict_level<double>(pnb, pcoords, pf, prho, pvel, cnb, cptr, cdx, cdy, cdz, cobst, cf, tau_p, tau_c, comp,
                         level_visc_physical);
}

void ora_restrict_d3q27_f32(int32_t pnb, const int32_t* pcoords, float* pf, float* prho, float* pvel, int32_t cnb,
                            const int32_t* cptr, int32_t cdx, int32_t cdy, int32_t cdz, const uint8_t* cobst,
                            const float* cf, double tau_p, double tau_c, int32_t comp, int32_t level_visc_physical) {
  restrict_level<float>(pnb, pcoords, pf, prho, pvel, cnb, cptr, cdx, cdy, cdz, cobst, cf, (float)tau_p, (float)tau_c,
                        comp, level_visc_physical);
}

// Float64 totals over fluid cells (state.jl:614-637): out = {mass, px, py, pz} from f.
void ora_mass_momentum_f64(int32_t nb, const uint8_t* obstacle, const double* f, double* out) {
  const int64_t n = 512 * (int64_t)nb;
  double m = 0, px = 0, py = 0, pz = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (obstacle && obstacle[i]) continue;
    for (int k = 0; k < Q; ++k) {
      double v = f[i + n * k];
      m += v; px += v * TB.cx[k]; py += v * TB.cy[k]; pz += v * TB.cz[k];
    }
  }
  out[0] = m; out[1] = px; out[2] = py; out[3] = pz;
}

// Bouzidi correction of one step's output: f_post = the step's post-collision populations,
// f_out = its output (overwritten on the corrected links). Arrays in the reference layout.
int ora_bouzidi_linear_f64(int32_t nb, const int32_t* nbr, const uint8_t* obstacle, int32_t n, const int32_t* cells,
                           const float* q, float q_min, int32_t ff, float rel_cap, float abs_cap,
                           const double* f_post, double* f_out) {
  Level L = make_level(nb, 0, 0, 0, nullptr, nbr, obstacle, nullptr, nullptr);
  bouzidi_linear<double>(L, n, cells, q, q_min, ff, rel_cap, abs_cap, f_post, f_out);
  return 0;
}
int ora_bouzidi_linear_f32(int32_t nb, const int32_t* nbr, const uint8_t* obstacle, int32_t n, const int32_t* cells,
                           const float* q, float q_min, int32_t ff, float rel_cap, float abs_cap,
                           const float* f_post, float* f_out) {
  Level L = make_level(nb, 0, 0, 0, nullptr, nbr, obstacle, nullptr, nullptr);
  bouzidi_linear<float>(L, n, cells, q, q_min, ff, rel_cap, abs_cap, f_post, f_out);
  return 0;
}

}  // extern "C"
