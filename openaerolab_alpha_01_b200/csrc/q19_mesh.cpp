// q19_mesh.cpp — host-side octree mesh of one level with a body: the D3Q19 solver's mesh generator
// for a single level (no refinement), from placed triangles and a box domain.
//
// Reference (OpenAeroLab src/octree_q19, Julia):
//   triangle queries: BVH, nearest point, first crossing of a segment, axis-ray parity
//                                               src/octree_q19/src/geometry.jl:71-280
//   periodic replication of the surface ....... src/octree_q19/src/generator.jl:116-140
//   root grid (even counts) ................... generator.jl:168-178
//   octs, boundary octs, kinds, face masks,
//   Morton order, neighbour table ............. generator.jl:270-350, octree.jl:16-48
//   near-surface slots ........................ generator.jl:851-870
//   crossings of the near slots' links ........ generator.jl:352-378
//   flood fill from the -x face over uncut links, unreached -> solid, leak check
//                                               generator.jl:410-540
//   cut links (Bouzidi q, triangle, partner) .. generator.jl:543-600
//   special-direction masks ................... generator.jl:794-816
// The arithmetic of the geometric predicates (Moller-Trumbore with the reference's tolerances,
// Ericson's closest point) is the reference's, so crossings and parities agree with it up to
// ties between triangles of equal hit distance.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <array>
#include <cstdarg>
#include <vector>
#include <functional>
#include <mutex>

#include "../../include/oal.h"

oal_status oal_internal_set_error(oal_status s, const char* msg);

namespace {

struct V3 {
  double x, y, z;
  double operator[](int a) const { return a == 0 ? x : a == 1 ? y : z; }
  double& operator[](int a) { return a == 0 ? x : a == 1 ? y : z; }
};
inline V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 vmul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 vcross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 vmin(V3 a, V3 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }

struct Tri {
  V3 v[3];
};

// D3Q19 (lattice.jl:8-11), 0-based
const int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
const int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
const int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
inline int opp(int i) { return i == 0 ? 0 : (i & 1) ? i + 1 : i - 1; }

enum : uint8_t { K_NONE = 0, K_FLUID = 1, K_SOLID = 2, K_COVERED = 3, K_GHOST = 4, K_BOUNDARY = 5 };

inline int nbr_index(int dx, int dy, int dz) { return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); }
inline void slot_offset(int k, int& x, int& y, int& z) { x = k & 1; y = (k >> 1) & 1; z = (k >> 2) & 1; }
inline int slot_index(int x, int y, int z) { return x + 2 * y + 4 * z; }
inline int clamp1(int v) { return v < 0 ? -1 : (v > 1 ? 1 : 0); }

uint64_t spread(uint64_t v) {
  v &= 0x1fffff;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}
uint64_t morton(int64_t ix, int64_t iy, int64_t iz) {
  return spread((uint64_t)ix) | (spread((uint64_t)iy) << 1) | (spread((uint64_t)iz) << 2);
}

// ---- bounding-volume hierarchy (geometry.jl:71-113) ---------------------------------------------
struct BVH {
  std::vector<V3> lo, hi;
  std::vector<int32_t> left, right, first, count, order;
  const std::vector<Tri>* tri = nullptr;

  static void tri_box(const Tri& t, V3& lo, V3& hi) {
    lo = vmin(vmin(t.v[0], t.v[1]), t.v[2]);
    hi = vmax(vmax(t.v[0], t.v[1]), t.v[2]);
  }

  void build(const std::vector<Tri>& tris, int leaf = 8) {
    tri = &tris;
    const int n = (int)tris.size();
    std::vector<V3> cen(n);
    for (int i = 0; i < n; ++i) cen[i] = vmul(vadd(vadd(tris[i].v[0], tris[i].v[1]), tris[i].v[2]), 1.0 / 3.0);
    order.resize(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    node(0, n - 1, cen, leaf);
  }

  int node(int a, int b, const std::vector<V3>& cen, int leaf) {
    const int id = (int)lo.size();
    lo.push_back({INFINITY, INFINITY, INFINITY});
    hi.push_back({-INFINITY, -INFINITY, -INFINITY});
    left.push_back(-1);
    right.push_back(-1);
    first.push_back(0);
    count.push_back(0);
    V3 blo{INFINITY, INFINITY, INFINITY}, bhi{-INFINITY, -INFINITY, -INFINITY};
    V3 clo = blo, chi = bhi;
    for (int k = a; k <= b; ++k) {
      V3 tl, th;
      tri_box((*tri)[order[k]], tl, th);
      blo = vmin(blo, tl);
      bhi = vmax(bhi, th);
      clo = vmin(clo, cen[order[k]]);
      chi = vmax(chi, cen[order[k]]);
    }
    lo[id] = blo;
    hi[id] = bhi;
    if (b - a + 1 <= leaf) {
      first[id] = a;
      count[id] = b - a + 1;
      return id;
    }
    const V3 ext = vsub(chi, clo);
    const int axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);
    const int mid = (a + b) / 2;
    std::nth_element(order.begin() + a, order.begin() + mid, order.begin() + b + 1,
                     [&](int32_t p, int32_t q) { return cen[p][axis] < cen[q][axis]; });
    const int l = node(a, mid, cen, leaf);
    const int r = node(mid + 1, b, cen, leaf);
    left[id] = l;
    right[id] = r;
    return id;
  }

  static double box_dist2(V3 p, V3 lo, V3 hi) {
    double d = 0;
    for (int a = 0; a < 3; ++a) {
      const double t = p[a] < lo[a] ? lo[a] - p[a] : (p[a] > hi[a] ? p[a] - hi[a] : 0.0);
      d += t * t;
    }
    return d;
  }

  // Ericson, Real-Time Collision Detection 5.1.5 (geometry.jl:125-152)
  static V3 tri_closest(V3 p, V3 a, V3 b, V3 c) {
    const V3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
    const double d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return a;
    const V3 bp = vsub(p, b);
    const double d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return b;
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) return vadd(a, vmul(ab, d1 / (d1 - d3)));
    const V3 cp = vsub(p, c);
    const double d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return c;
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return vadd(a, vmul(ac, d2 / (d2 - d6)));
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0)
      return vadd(b, vmul(vsub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
    const double den = 1 / (va + vb + vc), v = vb * den, w = vc * den;
    return vadd(a, vadd(vmul(ab, v), vmul(ac, w)));
  }

  // nearest surface distance to p; `bound` when nothing is closer (geometry.jl:154-181)
  double nearest(V3 p, double bound, std::vector<int32_t>& stack, int* tri_out = nullptr) const {
    double best = bound * bound;
    int besttri = -1;
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const int id = stack[--sp];
      if (box_dist2(p, lo[id], hi[id]) >= best) continue;
      if (left[id] < 0) {
        for (int k = first[id]; k < first[id] + count[id]; ++k) {
          const int ti = order[k];
          const Tri& t = (*tri)[ti];
          const V3 q = tri_closest(p, t.v[0], t.v[1], t.v[2]);
          const V3 d = vsub(p, q);
          const double dd = vdot(d, d);
          if (dd < best) {
            best = dd;
            besttri = ti;
          }
        }
      } else {
        const int l = left[id], r = right[id];
        const double dl = box_dist2(p, lo[l], hi[l]), dr = box_dist2(p, lo[r], hi[r]);
        if (dl < dr) {
          if (dr < best) stack[sp++] = r;
          if (dl < best) stack[sp++] = l;
        } else {
          if (dl < best) stack[sp++] = l;
          if (dr < best) stack[sp++] = r;
        }
      }
    }
    if (tri_out) *tri_out = besttri;
    return std::sqrt(best);
  }

  static bool segment_box_overlap(V3 a, V3 b, V3 lo, V3 hi) {
    double tmin = 0.0, tmax = 1.0;
    for (int k = 0; k < 3; ++k) {
      const double d = b[k] - a[k];
      if (std::fabs(d) < 1e-300) {
        if (a[k] < lo[k] || a[k] > hi[k]) return false;
      } else {
        double t1 = (lo[k] - a[k]) / d, t2 = (hi[k] - a[k]) / d;
        if (t1 > t2) std::swap(t1, t2);
        tmin = std::max(tmin, t1);
        tmax = std::min(tmax, t2);
        if (tmin > tmax) return false;
      }
    }
    return true;
  }

  // first crossing of a -> b: q in (0, 1] and the triangle, or (1, -1) (geometry.jl:204-232)
  double first_crossing(V3 a, V3 b, std::vector<int32_t>& stack, int* tri_out) const {
    const V3 dir = vsub(b, a);
    double best = INFINITY;
    int besttri = -1;
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const int id = stack[--sp];
      if (!segment_box_overlap(a, b, lo[id], hi[id])) continue;
      if (left[id] < 0) {
        for (int k = first[id]; k < first[id] + count[id]; ++k) {
          const int ti = order[k];
          const Tri& t = (*tri)[ti];
          const V3 e1 = vsub(t.v[1], t.v[0]), e2 = vsub(t.v[2], t.v[0]);
          const V3 h = vcross(dir, e2);
          const double det = vdot(e1, h);
          if (std::fabs(det) < 1e-300) continue;
          const double inv = 1 / det;
          const V3 s = vsub(a, t.v[0]);
          const double u = inv * vdot(s, h);
          if (u < -1e-12 || u > 1 + 1e-12) continue;
          const V3 qv = vcross(s, e1);
          const double v = inv * vdot(dir, qv);
          if (v < -1e-12 || u + v > 1 + 1e-12) continue;
          const double tt = inv * vdot(e2, qv);
          if (tt >= 1e-12 && tt <= 1 + 1e-12 && tt < best) {
            best = std::max(tt, 0.0);
            besttri = ti;
          }
        }
      } else {
        stack[sp++] = left[id];
        stack[sp++] = right[id];
      }
    }
    *tri_out = besttri;
    return std::min(best, 1.0);
  }

  // crossings of the ray from p along +axis (dirn 1) or -axis (dirn -1) (geometry.jl:235-268). Hits
  // at the same ray parameter (a ray through an edge or vertex shared by several triangles) count
  // once; the reference counts each triangle, which miscounts a ray through a shared edge.
  int ray_crossings(V3 p, int axis, std::vector<int32_t>& stack, int dirn = 1) const {
    thread_local std::vector<double> hits;
    hits.clear();
    int sp = 0;
    stack[sp++] = 0;
    const int b1 = axis == 0 ? 1 : 0, b2 = axis == 2 ? 1 : 2;
    V3 dir{0, 0, 0};
    dir[axis] = dirn > 0 ? 1.0 : -1.0;
    while (sp > 0) {
      const int id = stack[--sp];
      const V3 l = lo[id], h = hi[id];
      if ((dirn > 0 ? h[axis] < p[axis] : l[axis] > p[axis]) || p[b1] < l[b1] || p[b1] > h[b1] || p[b2] < l[b2] || p[b2] > h[b2]) continue;
      if (left[id] < 0) {
        for (int k = first[id]; k < first[id] + count[id]; ++k) {
          const Tri& t = (*tri)[order[k]];
          const V3 e1 = vsub(t.v[1], t.v[0]), e2 = vsub(t.v[2], t.v[0]);
          const V3 hh = vcross(dir, e2);
          const double det = vdot(e1, hh);
          if (std::fabs(det) < 1e-300) continue;
          const double inv = 1 / det;
          const V3 s = vsub(p, t.v[0]);
          const double u = inv * vdot(s, hh);
          if (u < 0 || u > 1) continue;
          const V3 q = vcross(s, e1);
          const double v = inv * vdot(dir, q);
          if (v < 0 || u + v > 1) continue;
          const double tt = inv * vdot(e2, q);
          if (tt > 1e-12) hits.push_back(tt);
        }
      } else {
        stack[sp++] = left[id];
        stack[sp++] = right[id];
      }
    }
    std::sort(hits.begin(), hits.end());
    int n = 0;
    for (size_t h = 0; h < hits.size(); ++h)
      if (h == 0 || hits[h] - hits[h - 1] > 1e-9 * std::max(1.0, std::fabs(hits[h]))) ++n;
    return n;
  }

  bool is_inside(V3 p, std::vector<int32_t>& stack) const {
    return (ray_crossings(p, 0, stack) & 1) + (ray_crossings(p, 1, stack) & 1) + (ray_crossings(p, 2, stack) & 1) >= 2;
  }

  // cavity sealing (cavity_seal_decision, geometry.jl:275-295): 0 outside by the majority of the
  // +axis parities; 1 inside (near the surface the majority suffices, farther away two axes must
  // also have odd -axis parity); 2 majority inside but not bracketed on two axes
  uint8_t seal_decision(V3 p, std::vector<int32_t>& stack, bool near_surface) const {
    bool pos[3];
    int npos = 0;
    for (int a = 0; a < 3; ++a) npos += (pos[a] = (ray_crossings(p, a, stack) & 1) != 0);
    if (npos < 2) return 0;
    if (near_surface) return 1;
    int pairs = 0;
    for (int a = 0; a < 3; ++a)
      if (pos[a] && (ray_crossings(p, a, stack, -1) & 1) && ++pairs >= 2) return 1;
    return 2;
  }
};

// run f(t, begin, end) over [0, n) on up to `nt` threads
template <class F>
void parallel_for(int64_t n, F f) {
  int nt = (int)std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()), 32);
  if (n < 4096) nt = 1;
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    const int64_t b = n * t / nt, e = n * (t + 1) / nt;
    if (nt == 1) {
      f(t, b, e);
      return;
    }
    th.emplace_back([=] { f(t, b, e); });
  }
  for (auto& x : th) x.join();
}

}  // namespace


namespace {

// one level of the mesh (octree.jl:50-71)
struct LevelMesh {
  int level = 1;  // 1-based
  double dx = 1.0;
  int n[3] = {0, 0, 0};
  int32_t nocts = 0;
  std::vector<int32_t> origin;    // (3, nocts)
  std::vector<uint8_t> real;      // (nocts)
  std::vector<uint8_t> kind;      // (8, nocts)
  std::vector<uint8_t> face;      // (8, nocts)
  std::vector<int32_t> onbr;      // (27, nocts) 1-based
  std::vector<int32_t> cutidx;    // (8, nocts) 1-based, 0 none
  std::vector<uint32_t> special;  // (8, nocts)
  std::vector<int32_t> cut_slot;  // (ncut) 1-based slot id k + 8 (o - 1)
  std::vector<int32_t> cut_off;   // (ncut + 1) 1-based
  std::vector<uint8_t> cut_dir;   // (nlinks) 2..19
  std::vector<float> cut_q;
  std::vector<int32_t> cut_tri;   // 1-based original triangle, 0 none
  std::vector<uint8_t> cut_partner;
  std::vector<int32_t> ghost_slot, ghost_donor;  // 1-based slot ids; donors (64, nghost) of level - 1
  std::vector<float> ghost_w;
  std::vector<int32_t> restrict_slot, restrict_src;  // sources (64, nrestrict) of level + 1
  std::vector<uint8_t> restrict_cubic;
  std::map<int64_t, int32_t> octmap;  // origin key -> 0-based oct
  int64_t counts[16] = {};

  int64_t key(int x, int y, int z) const {
    return (((int64_t)(x + 2) / 2) * ((n[1] + 4) / 2) + (y + 2) / 2) * ((n[2] + 4) / 2) + (z + 2) / 2;
  }
  // oct whose origin is (ox, oy, oz) (even), or -1
  int32_t find_origin(int ox, int oy, int oz) const {
    if (ox < -2 || oy < -2 || oz < -2 || ox > n[0] || oy > n[1] || oz > n[2]) return -1;
    auto it = octmap.find(key(ox, oy, oz));
    return it == octmap.end() ? -1 : it->second;
  }
  // 0-based slot s = k + 8 o of level cell (i, j, k), or -1 (octree.jl:98-106)
  int64_t find_slot(int i, int j, int k) const {
    const int32_t o = find_origin(i & ~1, j & ~1, k & ~1);
    return o < 0 ? -1 : 8 * (int64_t)o + ((i & 1) + 2 * (j & 1) + 4 * (k & 1));
  }
  void cell(int64_t s, int c[3]) const {
    const int64_t o = s / 8;
    const int k = (int)(s % 8);
    c[0] = origin[3 * o] + (k & 1);
    c[1] = origin[3 * o + 1] + ((k >> 1) & 1);
    c[2] = origin[3 * o + 2] + ((k >> 2) & 1);
  }
  V3 centre(int64_t s) const {
    int c[3];
    cell(s, c);
    return {(c[0] + 0.5) * dx, (c[1] + 0.5) * dx, (c[2] + 0.5) * dx};
  }
  // same-level neighbour slot of slot s along e (octree.jl:152-159), -1 when the oct is missing
  int64_t neighbour(int64_t s, int ex, int ey, int ez) const {
    const int64_t o = s / 8;
    int x, y, z;
    slot_offset((int)(s % 8), x, y, z);
    const int nx = x + ex, ny = y + ey, nz = z + ez;
    const int ox = clamp1(nx), oy = clamp1(ny), oz = clamp1(nz);
    const int32_t no = onbr[27 * o + nbr_index(ox, oy, oz)] - 1;
    return no < 0 ? -1 : 8 * (int64_t)no + slot_index(nx - 2 * ox, ny - 2 * oy, nz - 2 * oz);
  }
};

// cubic Lagrange weights of a point at t in [0, 1) between the 2nd and 3rd of 4 nodes (octree.jl:84)
inline void cubic_weights(double t, double w[4]) {
  w[0] = -t * (1 - t) * (2 - t) / 6;
  w[1] = (1 + t) * (1 - t) * (2 - t) / 2;
  w[2] = (1 + t) * t * (2 - t) / 2;
  w[3] = -(1 + t) * t * (1 - t) / 6;
}
// the 8 inner nodes (children) of a 4x4x4 stencil, 0-based node index di + 4 dj + 16 dk (octree.jl:82)
inline int stencil_inner(int m) { return (1 + (m & 1)) + 4 * (1 + ((m >> 1) & 1)) + 16 * (1 + ((m >> 2) & 1)); }
inline bool is_inner(int nidx) {
  const int di = nidx & 3, dj = (nidx >> 2) & 3, dk = nidx >> 4;
  return di >= 1 && di <= 2 && dj >= 1 && dj <= 2 && dk >= 1 && dk <= 2;
}

// dense bit masks of level cells (Julia BitArray{3}, x fastest)
struct Mask {
  int n[3] = {0, 0, 0};
  std::vector<uint8_t> b;
  Mask() = default;
  Mask(int nx, int ny, int nz, bool v) : b((size_t)nx * ny * nz, v ? 1 : 0) {
    n[0] = nx;
    n[1] = ny;
    n[2] = nz;
  }
  size_t idx(int i, int j, int k) const { return (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * k); }
  uint8_t& at(int i, int j, int k) { return b[idx(i, j, k)]; }
  uint8_t at(int i, int j, int k) const { return b[idx(i, j, k)]; }
};

Mask parent_mask(const Mask& R) {
  Mask P(R.n[0] / 2, R.n[1] / 2, R.n[2] / 2, false);
  for (int k = 0; k < R.n[2]; ++k)
    for (int j = 0; j < R.n[1]; ++j)
      for (int i = 0; i < R.n[0]; ++i)
        if (R.at(i, j, k)) P.at(i / 2, j / 2, k / 2) = 1;
  return P;
}
Mask children_mask(const Mask& P) {
  Mask R(2 * P.n[0], 2 * P.n[1], 2 * P.n[2], false);
  for (int k = 0; k < P.n[2]; ++k)
    for (int j = 0; j < P.n[1]; ++j)
      for (int i = 0; i < P.n[0]; ++i)
        if (P.at(i, j, k))
          for (int dk = 0; dk < 2; ++dk)
            for (int dj = 0; dj < 2; ++dj)
              for (int di = 0; di < 2; ++di) R.at(2 * i + di, 2 * j + dj, 2 * k + dk) = 1;
  return R;
}
// separable Chebyshev dilation by r cells, periodic axes wrap (generator.jl:47-70)
void dilate(Mask& M, int r, const int periodic[3]) {
  for (int axis = 0; axis < 3; ++axis) {
    std::vector<std::array<int, 3>> idx;
    for (int k = 0; k < M.n[2]; ++k)
      for (int j = 0; j < M.n[1]; ++j)
        for (int i = 0; i < M.n[0]; ++i)
          if (M.at(i, j, k)) idx.push_back({i, j, k});
    const int na = M.n[axis];
    for (auto& I : idx)
      for (int s = -r; s <= r; ++s) {
        if (!s) continue;
        int v = I[axis] + s;
        if (periodic[axis]) v = ((v % na) + na) % na;
        else if (v < 0 || v >= na) continue;
        std::array<int, 3> J = I;
        J[axis] = v;
        M.at(J[0], J[1], J[2]) = 1;
      }
  }
}
// coarse-row buffer at non-periodic faces except symmetry (generator.jl:838-850)
Mask face_margin(const int n[3], int l, const int periodic[3], const int faces[6]) {
  Mask M(n[0], n[1], n[2], false);
  const int m = 1 << (l - 1);
  for (int a = 0; a < 3; ++a) {
    if (periodic[a]) continue;
    for (int side = 0; side < 2; ++side) {
      if (faces[2 * a + side] == OAL_Q19_FACE_SYMMETRY) continue;
      const int lo = side == 0 ? 0 : n[a] - m, hi = side == 0 ? std::min(m, n[a]) : n[a];
      for (int v = std::max(lo, 0); v < hi; ++v)
        for (int p = 0; p < n[(a + 1) % 3]; ++p)
          for (int q = 0; q < n[(a + 2) % 3]; ++q) {
            int c[3];
            c[a] = v;
            c[(a + 1) % 3] = p;
            c[(a + 2) % 3] = q;
            M.at(c[0], c[1], c[2]) = 1;
          }
    }
  }
  return M;
}
void and_not(Mask& R, const Mask& M) {
  for (size_t i = 0; i < R.b.size(); ++i) R.b[i] = R.b[i] && !M.b[i];
}

bool in_region(V3 p, const oal_q19_region& r) {
  if (r.kind == 0)
    return r.lo[0] <= p.x && p.x <= r.hi[0] && r.lo[1] <= p.y && p.y <= r.hi[1] && r.lo[2] <= p.z && p.z <= r.hi[2];
  const V3 c{r.centre[0], r.centre[1], r.centre[2]};
  if (r.kind == 1) {
    const V3 d = vsub(p, c);
    return vdot(d, d) <= r.radius * r.radius;
  }
  const V3 lo{r.lo[0], r.lo[1], r.lo[2]}, hi{r.hi[0], r.hi[1], r.hi[2]};
  const V3 a = vsub(hi, lo);
  const double l2 = vdot(a, a);
  if (l2 == 0) return false;
  const double t = vdot(vsub(p, lo), a) / l2;
  if (t < 0 || t > 1) return false;
  const V3 d = vsub(vsub(p, lo), vmul(a, t));
  return vdot(d, d) <= r.radius * r.radius;
}

}  // namespace

struct oal_q19_mesh {
  int L = 1;
  int periodic[3] = {0, 0, 0};
  int faces[6] = {0, 0, 0, 0, 0, 0};
  int32_t ntri = 0;
  std::vector<LevelMesh> levels;
  int64_t counts[16] = {};
  int64_t sealed = 0, unbracketed = 0;  // cavity-sealing report
};

namespace {

oal_status fail(oal_status s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
oal_status fail(oal_status s, const char* fmt, ...) {
  char buf[400];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return oal_internal_set_error(s, buf);
}

oal_status generate(const double* tri_in, int32_t ntri_in, const oal_q19_mesh_spec* spec, oal_q19_mesh* M) {
  const int L = spec->levels;
  const int Ls0 = spec->surface_level > 0 ? spec->surface_level : L;
  if (L < 1 || L > 12) return fail(OAL_E_INVALID_ARG, "levels must lie in 1..12 (got %d)", L);
  if (Ls0 > L) return fail(OAL_E_INVALID_ARG, "surface_level must be in 1..levels");
  if (spec->nsurface_levels < 0 || (spec->nsurface_levels > 0 && !spec->surface_levels))
    return fail(OAL_E_INVALID_ARG, "surface_levels: %d boxes without an array", spec->nsurface_levels);
  for (int i = 0; i < spec->nsurface_levels; ++i)
    if (spec->surface_levels[i].level < 1 || spec->surface_levels[i].level > L)
      return fail(OAL_E_INVALID_ARG, "surface_levels[%d].level must be in 1..levels", i);
  std::vector<double> dxs(L + 1);
  for (int l = 1; l <= L; ++l) dxs[l] = spec->dx * std::ldexp(1.0, L - l);
  const double domain_in[3] = {spec->domain[0], spec->domain[1], spec->domain[2]};
  const bool no_geometry = ntri_in == 0;
  M->L = L;
  M->ntri = ntri_in;
  for (int a = 0; a < 3; ++a) M->periodic[a] = spec->periodic[a] != 0;
  for (int f = 0; f < 6; ++f) M->faces[f] = spec->faces[f];
  const int* periodic = M->periodic;
  // ---- the surface, replicated across periodic faces (generator.jl:112-140)
  std::vector<Tri> tri_orig, tri;
  std::vector<int32_t> tri_src;
  if (no_geometry) {
    const double far = 1e6 * (1 + std::max(domain_in[0], std::max(domain_in[1], domain_in[2])));
    tri_orig.push_back({{{far, far, far}, {far + 1, far, far}, {far, far + 1, far}}});
  } else {
    for (int t = 0; t < ntri_in; ++t) {
      Tri T;
      for (int v = 0; v < 3; ++v) T.v[v] = {tri_in[9 * t + 3 * v], tri_in[9 * t + 3 * v + 1], tri_in[9 * t + 3 * v + 2]};
      tri_orig.push_back(T);
    }
  }
  tri = tri_orig;
  for (size_t t = 0; t < tri.size(); ++t) tri_src.push_back((int32_t)t);
  if (!no_geometry) {
    double margin = spec->band_fine * dxs[L] + 4 * dxs[1];
    for (int m = 2; m <= L - 1; ++m) margin += spec->band * dxs[m];
    for (int a = 0; a < 3; ++a) {
      if (!periodic[a]) continue;
      double blo = INFINITY, bhi = -INFINITY;
      for (const Tri& T : tri)
        for (int v = 0; v < 3; ++v) {
          blo = std::min(blo, T.v[v][a]);
          bhi = std::max(bhi, T.v[v][a]);
        }
      if (bhi - blo >= domain_in[a] - 1e-9) {
        std::vector<Tri> keep;
        std::vector<int32_t> ksrc;
        for (size_t t = 0; t < tri.size(); ++t) {
          const double mx = std::max(tri[t].v[0][a], std::max(tri[t].v[1][a], tri[t].v[2][a]));
          const double mn = std::min(tri[t].v[0][a], std::min(tri[t].v[1][a], tri[t].v[2][a]));
          if (mx > 0 && mn < domain_in[a]) {
            keep.push_back(tri[t]);
            ksrc.push_back(tri_src[t]);
          }
        }
        tri.swap(keep);
        tri_src.swap(ksrc);
      }
      std::vector<Tri> extra;
      std::vector<int32_t> esrc;
      for (size_t t = 0; t < tri.size(); ++t) {
        const double lo = std::min(tri[t].v[0][a], std::min(tri[t].v[1][a], tri[t].v[2][a]));
        const double hi = std::max(tri[t].v[0][a], std::max(tri[t].v[1][a], tri[t].v[2][a]));
        V3 sh{0, 0, 0};
        sh[a] = domain_in[a];
        if (lo < margin) {
          extra.push_back({{vadd(tri[t].v[0], sh), vadd(tri[t].v[1], sh), vadd(tri[t].v[2], sh)}});
          esrc.push_back(tri_src[t]);
        }
        if (hi > domain_in[a] - margin) {
          extra.push_back({{vsub(tri[t].v[0], sh), vsub(tri[t].v[1], sh), vsub(tri[t].v[2], sh)}});
          esrc.push_back(tri_src[t]);
        }
      }
      tri.insert(tri.end(), extra.begin(), extra.end());
      tri_src.insert(tri_src.end(), esrc.begin(), esrc.end());
    }
    if (tri.empty()) return fail(OAL_E_INVALID_ARG, "no triangle lies in the domain");
  }
  BVH bvh;
  bvh.build(tri);
  const size_t stack_size = 4096 + 4 * bvh.lo.size();
  V3 blo{INFINITY, INFINITY, INFINITY}, bhi{-INFINITY, -INFINITY, -INFINITY};
  for (const Tri& T : tri_orig)
    for (int v = 0; v < 3; ++v) {
      blo = vmin(blo, T.v[v]);
      bhi = vmax(bhi, T.v[v]);
    }
  std::vector<V3> normals(tri.size());
  for (size_t t = 0; t < tri.size(); ++t) {
    const V3 nn = vcross(vsub(tri[t].v[1], tri[t].v[0]), vsub(tri[t].v[2], tri[t].v[0]));
    normals[t] = vmul(nn, 1 / std::sqrt(vdot(nn, nn)));
  }
  // surface orientation (generator.jl:145-166): +1 normals into the fluid, -1 into the body, 0 open
  int orient = 0;
  if (!no_geometry && L > 1) {
    std::vector<int32_t> st(stack_size);
    const int n = std::min<int>((int)tri_orig.size(), 2000), step = std::max<int>(1, (int)tri_orig.size() / n);
    int pos = 0, neg = 0, open = 0;
    for (size_t t = 0; t < tri_orig.size(); t += step) {
      const V3 c = vmul(vadd(vadd(tri_orig[t].v[0], tri_orig[t].v[1]), tri_orig[t].v[2]), 1.0 / 3.0);
      const V3 nn = vcross(vsub(tri_orig[t].v[1], tri_orig[t].v[0]), vsub(tri_orig[t].v[2], tri_orig[t].v[0]));
      const V3 nrm = vmul(nn, 1 / std::sqrt(vdot(nn, nn)));
      const bool a = bvh.is_inside(vadd(c, vmul(nrm, spec->dx)), st), b = bvh.is_inside(vsub(c, vmul(nrm, spec->dx)), st);
      if (a && !b) ++neg;
      else if (b && !a) ++pos;
      else ++open;
    }
    const int total = std::max(pos + neg + open, 1);
    orient = (double)open / total > 0.5 ? 0 : (pos >= neg ? 1 : -1);
  }
  // ---- root grid: even counts, periodic axes exact (generator.jl:168-178)
  int n1[3];
  for (int a = 0; a < 3; ++a) {
    const double c = domain_in[a] / dxs[1];
    if (periodic[a]) {
      const long r = std::lround(c);
      if (std::fabs((double)r - c) > 1e-9 * std::max(1.0, std::fabs(c)) || (r & 1) || r < 2)
        return fail(OAL_E_INVALID_ARG, "periodic axis %d: the domain must be an even number of coarse cells", a);
      n1[a] = (int)r;
    } else {
      int v = (int)std::ceil(c - 1e-9);
      v += v % 2;
      if (v < 2) return fail(OAL_E_INVALID_ARG, "axis %d: domain smaller than two coarse cells", a);
      n1[a] = v;
    }
  }
  double domain[3];
  for (int a = 0; a < 3; ++a) domain[a] = n1[a] * dxs[1];
  std::vector<std::array<int, 3>> sizes(L + 1);
  for (int l = 1; l <= L; ++l)
    for (int a = 0; a < 3; ++a) sizes[l][a] = n1[a] << (l - 1);
  if ((int64_t)sizes[L][0] * sizes[L][1] * sizes[L][2] > (int64_t)1 << 36) return fail(OAL_E_TOO_LARGE, "finest grid too large");

  // ---- 1. refinement marks (generator.jl:186-252)
  auto band_distance = [&](int l, int Ls) {
    if (l > Ls) return -1.0;
    double d = spec->band_fine * dxs[Ls];
    for (int m = l; m <= Ls - 1; ++m) d += spec->band * dxs[m];
    return d;
  };
  // the surface level at a point: the global one, raised inside per-box surface levels
  // (local_surface_level, generator.jl:185)
  auto local_surface_level = [&](const V3& p) {
    int ls = Ls0;
    for (int i = 0; i < spec->nsurface_levels; ++i) {
      const oal_q19_surface_level& b = spec->surface_levels[i];
      if (p.x >= b.lo[0] && p.x <= b.hi[0] && p.y >= b.lo[1] && p.y <= b.hi[1] && p.z >= b.lo[2] && p.z <= b.hi[2])
        ls = std::max(ls, b.level);
    }
    return ls;
  };
  const double inner_band = 1.0;
  std::vector<Mask> R(L + 1);
  R[1] = Mask(sizes[1][0], sizes[1][1], sizes[1][2], true);
  const V3 ex = vsub(bhi, blo);
  const int wake_level = spec->wake_length > 0 ? Ls0 - spec->wake_level_offset : 0;
  for (int l = 2; l <= L; ++l) {
    R[l] = Mask(sizes[l][0], sizes[l][1], sizes[l][2], false);
    const double dxp = dxs[l - 1], dxc = dxs[l], hdc = std::sqrt(3.0) * dxc / 2;
    const double dmax = band_distance(l, L);
    std::vector<std::array<int, 3>> cand;
    for (int k = 0; k < sizes[l - 1][2]; ++k)
      for (int j = 0; j < sizes[l - 1][1]; ++j)
        for (int i = 0; i < sizes[l - 1][0]; ++i)
          if (R[l - 1].at(i, j, k)) cand.push_back({i, j, k});
    if (!no_geometry && dmax >= 0) {
      std::vector<std::vector<size_t>> lists(64);
      std::vector<int> nts(1, 0);
      std::mutex mu;
      parallel_for((int64_t)cand.size(), [&](int, int64_t b, int64_t e) {
        std::vector<int32_t> st(stack_size);
        std::vector<size_t> lst;
        for (int64_t ci = b; ci < e; ++ci) {
          const int i = cand[ci][0], j = cand[ci][1], k = cand[ci][2];
          const V3 pc{(i + 0.5) * dxp, (j + 0.5) * dxp, (k + 0.5) * dxp};
          const double dp = bvh.nearest(pc, dmax + 2 * hdc + dxp, st);
          if (dp > dmax + 2 * hdc) continue;
          for (int ck = 0; ck < 2; ++ck)
            for (int cj = 0; cj < 2; ++cj)
              for (int cci = 0; cci < 2; ++cci) {
                const int ii = 2 * i + cci, jj = 2 * j + cj, kk = 2 * k + ck;
                const V3 cc{(ii + 0.5) * dxc, (jj + 0.5) * dxc, (kk + 0.5) * dxc};
                const double dl = band_distance(l, local_surface_level(cc));
                if (dl < 0) continue;
                int ti = -1;
                const double dc = bvh.nearest(cc, dl + hdc + dxc, st, &ti);
                if (!(dc - hdc <= dl)) continue;
                if (orient != 0 && ti >= 0) {
                  // one-sided band: deeper than `inner_band` cells inside the body, nothing is refined
                  const Tri& T = tri[ti];
                  const V3 qn = BVH::tri_closest(cc, T.v[0], T.v[1], T.v[2]);
                  const double side = orient * vdot(vsub(cc, qn), normals[ti]);
                  if (side < -(inner_band * dxc + hdc)) continue;
                }
                lst.push_back(R[l].idx(ii, jj, kk));
              }
        }
        std::lock_guard<std::mutex> g(mu);
        lists.push_back(std::move(lst));
      });
      for (auto& lst : lists)
        for (size_t idx : lst) R[l].b[idx] = 1;
    }
    if (wake_level >= l && !no_geometry) {
      const double x0 = bhi.x, x1 = std::min(domain[0], bhi.x + spec->wake_length * ex.x);
      const double y0 = std::max(0.0, blo.y - spec->wake_margin * ex.y), y1 = std::min(domain[1], bhi.y + spec->wake_margin * ex.y);
      const double z0 = std::max(0.0, blo.z - spec->wake_margin * ex.z), z1 = std::min(domain[2], bhi.z + spec->wake_margin * ex.z);
      for (int k = std::max(0, (int)std::floor(z0 / dxc)); k < std::min(sizes[l][2], (int)std::ceil(z1 / dxc)); ++k)
        for (int j = std::max(0, (int)std::floor(y0 / dxc)); j < std::min(sizes[l][1], (int)std::ceil(y1 / dxc)); ++j)
          for (int i = std::max(0, (int)std::floor(x0 / dxc)); i < std::min(sizes[l][0], (int)std::ceil(x1 / dxc)); ++i)
            R[l].at(i, j, k) = 1;
    }
    for (int r = 0; r < spec->nregions; ++r) {
      const oal_q19_region& g = spec->regions[r];
      if (g.level < l) continue;
      double lo[3], hi[3];
      for (int a = 0; a < 3; ++a) {
        if (g.kind == 0) { lo[a] = g.lo[a]; hi[a] = g.hi[a]; }
        else if (g.kind == 1) { lo[a] = g.centre[a] - g.radius; hi[a] = g.centre[a] + g.radius; }
        else { lo[a] = std::min(g.lo[a], g.hi[a]) - g.radius; hi[a] = std::max(g.lo[a], g.hi[a]) + g.radius; }
      }
      for (int k = std::max(0, (int)std::floor(lo[2] / dxc)); k < std::min(sizes[l][2], (int)std::ceil(hi[2] / dxc)); ++k)
        for (int j = std::max(0, (int)std::floor(lo[1] / dxc)); j < std::min(sizes[l][1], (int)std::ceil(hi[1] / dxc)); ++j)
          for (int i = std::max(0, (int)std::floor(lo[0] / dxc)); i < std::min(sizes[l][0], (int)std::ceil(hi[0] / dxc)); ++i)
            if (in_region({(i + 0.5) * dxc, (j + 0.5) * dxc, (k + 0.5) * dxc}, g)) R[l].at(i, j, k) = 1;
    }
  }
  // ---- 2. balance, buffers, domain-face margin, sibling closure (generator.jl:254-268)
  for (int l = L; l >= 2; --l) {
    and_not(R[l], face_margin(sizes[l].data(), l, periodic, M->faces));
    Mask P = parent_mask(R[l]);
    dilate(P, 2, periodic);
    and_not(P, face_margin(sizes[l - 1].data(), l - 1, periodic, M->faces));
    for (size_t i = 0; i < P.b.size(); ++i) R[l - 1].b[i] |= P.b[i];
    R[l] = children_mask(parent_mask(R[l]));
    and_not(R[l], face_margin(sizes[l].data(), l, periodic, M->faces));
    R[l] = children_mask(parent_mask(R[l]));
  }
  for (int l = L; l >= 2; --l) {
    Mask P = parent_mask(R[l]);
    dilate(P, 2, periodic);
    and_not(P, face_margin(sizes[l - 1].data(), l - 1, periodic, M->faces));
    for (size_t i = 0; i < P.b.size(); ++i) R[l - 1].b[i] |= P.b[i];
  }
  std::vector<Mask> refined(L + 1);
  for (int l = 1; l < L; ++l) refined[l] = parent_mask(R[l + 1]);

  // ---- 3. octs, ghost octs, boundary octs, neighbour tables (generator.jl:270-350)
  M->levels.resize(L);
  for (int l = 1; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    Lv.level = l;
    Lv.dx = dxs[l];
    for (int a = 0; a < 3; ++a) Lv.n[a] = sizes[l][a];
    const int* n = Lv.n;
    std::vector<std::array<int, 3>> origins;
    if (l == 1) {
      for (int k = 0; k < n[2]; k += 2)
        for (int j = 0; j < n[1]; j += 2)
          for (int i = 0; i < n[0]; i += 2) origins.push_back({i, j, k});
    } else {
      const Mask& Pm = refined[l - 1];
      for (int k = 0; k < Pm.n[2]; ++k)
        for (int j = 0; j < Pm.n[1]; ++j)
          for (int i = 0; i < Pm.n[0]; ++i)
            if (Pm.at(i, j, k)) origins.push_back({2 * i, 2 * j, 2 * k});
    }
    auto wrap = [&](int p[3]) {
      bool inside = true;
      for (int a = 0; a < 3; ++a)
        if (p[a] < 0 || p[a] >= n[a]) {
          if (periodic[a]) p[a] = ((p[a] % n[a]) + n[a]) % n[a];
          else inside = false;
        }
      return inside;
    };
    const size_t nreal = origins.size();
    std::map<int64_t, std::array<int, 3>> realset, ghosts, bounds;
    for (auto& o : origins) realset[Lv.key(o[0], o[1], o[2])] = o;
    for (size_t r = 0; r < nreal; ++r)
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dxo = -1; dxo <= 1; ++dxo) {
            if (!dxo && !dy && !dz) continue;
            int p[3] = {origins[r][0] + 2 * dxo, origins[r][1] + 2 * dy, origins[r][2] + 2 * dz};
            const bool inside = wrap(p);
            const int64_t kk = Lv.key(p[0], p[1], p[2]);
            if (!inside) {
              bounds[kk] = {p[0], p[1], p[2]};
              continue;
            }
            if (realset.count(kk) || l == 1) continue;
            ghosts[kk] = {p[0], p[1], p[2]};
          }
    std::vector<uint8_t> okind(nreal, 0);
    for (auto& kv : ghosts) {
      origins.push_back(kv.second);
      okind.push_back(K_GHOST);
    }
    for (auto& kv : bounds) {
      origins.push_back(kv.second);
      okind.push_back(K_BOUNDARY);
    }
    const int64_t nocts = (int64_t)origins.size();
    if (nocts * 27 > INT32_MAX) return fail(OAL_E_TOO_LARGE, "too many octs on level %d", l);
    std::vector<std::pair<uint64_t, int32_t>> order(nocts);
    for (int64_t o = 0; o < nocts; ++o)
      order[o] = {morton((origins[o][0] >> 1) + 1, (origins[o][1] >> 1) + 1, (origins[o][2] >> 1) + 1), (int32_t)o};
    std::sort(order.begin(), order.end());
    Lv.nocts = (int32_t)nocts;
    Lv.origin.assign(3 * nocts, 0);
    Lv.real.assign(nocts, 0);
    Lv.kind.assign(8 * nocts, K_NONE);
    Lv.face.assign(8 * nocts, 0);
    Lv.onbr.assign(27 * nocts, 0);
    Lv.cutidx.assign(8 * nocts, 0);
    Lv.special.assign(8 * nocts, 0);
    for (int64_t o = 0; o < nocts; ++o) {
      const int src = order[o].second;
      const auto& og = origins[src];
      for (int a = 0; a < 3; ++a) Lv.origin[3 * o + a] = og[a];
      Lv.octmap[Lv.key(og[0], og[1], og[2])] = (int32_t)o;
      const uint8_t ok = okind[src];
      Lv.real[o] = ok == 0;
      for (int k = 0; k < 8; ++k) {
        int x, y, z;
        slot_offset(k, x, y, z);
        const int c[3] = {og[0] + x, og[1] + y, og[2] + z};
        if (ok == K_BOUNDARY) {
          uint8_t m = 0;
          if (c[0] < 0) m |= 1;
          if (c[0] >= n[0]) m |= 2;
          if (c[1] < 0) m |= 4;
          if (c[1] >= n[1]) m |= 8;
          if (c[2] < 0) m |= 16;
          if (c[2] >= n[2]) m |= 32;
          Lv.kind[8 * o + k] = K_BOUNDARY;
          Lv.face[8 * o + k] = m;
        } else if (ok == K_GHOST) {
          Lv.kind[8 * o + k] = K_GHOST;
        } else {
          Lv.kind[8 * o + k] = (l < L && refined[l].at(c[0], c[1], c[2])) ? K_COVERED : K_FLUID;
        }
      }
    }
    for (int64_t o = 0; o < nocts; ++o)
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dxo = -1; dxo <= 1; ++dxo) {
            int p[3] = {Lv.origin[3 * o] + 2 * dxo, Lv.origin[3 * o + 1] + 2 * dy, Lv.origin[3 * o + 2] + 2 * dz};
            wrap(p);
            Lv.onbr[27 * o + nbr_index(dxo, dy, dz)] = Lv.find_origin(p[0], p[1], p[2]) + 1;
          }
    Lv.counts[13] = (int64_t)nreal;
  }
  auto wrap_cell = [&](const LevelMesh& Lv, int c[3]) {  // -1 components outside non-periodic faces
    for (int a = 0; a < 3; ++a)
      if (c[a] < 0 || c[a] >= Lv.n[a]) c[a] = periodic[a] ? ((c[a] % Lv.n[a]) + Lv.n[a]) % Lv.n[a] : -1;
  };

  // ---- 4. classification (generator.jl:350-540)
  std::vector<std::vector<uint8_t>> near(L + 1), reached(L + 1), covered_solid(L + 1);
  std::vector<std::vector<int32_t>> nearrow(L + 1), ct(L + 1);
  std::vector<std::vector<float>> cq(L + 1);
  for (int l = 1; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    const int64_t ns = 8 * (int64_t)Lv.nocts;
    near[l].assign(ns, 0);
    const double dx = Lv.dx, bound = 2.0 * std::sqrt(3.0) * dx;
    if (!no_geometry) {
      parallel_for(Lv.nocts, [&](int, int64_t b, int64_t e) {
        std::vector<int32_t> st(stack_size);
        for (int64_t o = b; o < e; ++o) {
          const V3 oc{(Lv.origin[3 * o] + 1.0) * dx, (Lv.origin[3 * o + 1] + 1.0) * dx, (Lv.origin[3 * o + 2] + 1.0) * dx};
          const double d = bvh.nearest(oc, bound + std::sqrt(3.0) * dx, st);
          if (d >= bound + std::sqrt(3.0) * dx) continue;
          for (int k = 0; k < 8; ++k) {
            if (Lv.kind[8 * o + k] == K_BOUNDARY) continue;
            near[l][8 * o + k] = bvh.nearest(Lv.centre(8 * o + k), bound, st) < bound;
          }
        }
      });
    }
    nearrow[l].assign(ns, 0);
    std::vector<int64_t> slots;
    for (int64_t s = 0; s < ns; ++s)
      if (near[l][s] && Lv.kind[s] != K_BOUNDARY && Lv.kind[s] != K_COVERED) {
        slots.push_back(s);
        nearrow[l][s] = (int32_t)slots.size();
      }
    cq[l].assign(18 * slots.size(), 1.0f);
    ct[l].assign(18 * slots.size(), -1);
    parallel_for((int64_t)slots.size(), [&](int, int64_t b, int64_t e) {
      std::vector<int32_t> st(stack_size);
      for (int64_t r = b; r < e; ++r) {
        const V3 pc = Lv.centre(slots[r]);
        for (int i = 1; i < 19; ++i) {
          const V3 target{pc.x + CX[i] * dx, pc.y + CY[i] * dx, pc.z + CZ[i] * dx};
          int ti;
          const double q = bvh.first_crossing(pc, target, st, &ti);
          cq[l][18 * r + i - 1] = (float)q;
          ct[l][18 * r + i - 1] = ti;
        }
      }
    });
    reached[l].assign(ns, 0);
    covered_solid[l].assign(ns, 0);
  }
  auto crossq = [&](int l, int64_t s, int i) -> float {
    const int32_t row = nearrow[l][s];
    return row ? cq[l][18 * (int64_t)(row - 1) + i - 1] : 1.0f;
  };
  // ---- 4b. sealed cavities (generator.jl:383-414): fluid slots inside the body's bounding box
  // (one coarsest cell of margin) that parity puts inside the surface stay out of the fill
  std::vector<std::vector<uint8_t>> sealed(L + 1);
  for (int l = 1; l <= L; ++l) sealed[l].assign(8 * (int64_t)M->levels[l - 1].nocts, 0);
  if (spec->seal_cavities && !no_geometry) {
    const V3 mlo{blo.x - dxs[1], blo.y - dxs[1], blo.z - dxs[1]}, mhi{bhi.x + dxs[1], bhi.y + dxs[1], bhi.z + dxs[1]};
    for (int l = 1; l <= L; ++l) {
      const LevelMesh& Lv = M->levels[l - 1];
      std::vector<int64_t> cand;
      for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s) {
        if (Lv.kind[s] != K_FLUID) continue;
        const V3 c = Lv.centre(s);
        if (c.x >= mlo.x && c.x <= mhi.x && c.y >= mlo.y && c.y <= mhi.y && c.z >= mlo.z && c.z <= mhi.z) cand.push_back(s);
      }
      std::vector<uint8_t> flags(cand.size(), 0);
      parallel_for((int64_t)cand.size(), [&](int, int64_t b, int64_t e) {
        std::vector<int32_t> st(stack_size);
        for (int64_t i = b; i < e; ++i) flags[i] = bvh.seal_decision(Lv.centre(cand[i]), st, near[l][cand[i]] != 0);
      });
      for (size_t i = 0; i < cand.size(); ++i) {
        if (flags[i] == 1) {
          sealed[l][cand[i]] = 1;
          ++M->sealed;
        } else if (flags[i] == 2) {
          ++M->unbracketed;
        }
      }
    }
  }
  std::vector<std::pair<int, int64_t>> queue;
  {
    std::vector<int32_t> st(stack_size);
    for (int l = 1; l <= L; ++l) {
      LevelMesh& Lv = M->levels[l - 1];
      for (int64_t o = 0; o < Lv.nocts; ++o) {
        if (!Lv.real[o] || Lv.origin[3 * o] != 0) continue;
        for (int k = 0; k < 8; ++k) {
          const int64_t s = 8 * o + k;
          if ((k & 1) || Lv.kind[s] != K_FLUID) continue;
          if (!no_geometry && bvh.is_inside(Lv.centre(s), st)) continue;
          if (!reached[l][s]) {
            reached[l][s] = 1;
            queue.push_back({l, s});
          }
        }
      }
    }
  }
  if (queue.empty()) return fail(OAL_E_INVALID_ARG, "no fluid cell on the inlet face: the geometry covers the -x face");
  // push the fluid children of covered cell c (level l) on the face toward -e (generator.jl:896-918)
  std::function<void(int, const int*, const int*)> push_near_children = [&](int l, const int* c, const int* e) {
    if (l >= L) return;
    const LevelMesh& Lf = M->levels[l];
    for (int dk = 0; dk < 2; ++dk)
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          if (e[0] != 0 && di != (e[0] > 0 ? 0 : 1)) continue;
          if (e[1] != 0 && dj != (e[1] > 0 ? 0 : 1)) continue;
          if (e[2] != 0 && dk != (e[2] > 0 ? 0 : 1)) continue;
          const int cc[3] = {2 * c[0] + di, 2 * c[1] + dj, 2 * c[2] + dk};
          const int64_t cs = Lf.find_slot(cc[0], cc[1], cc[2]);
          if (cs < 0) continue;
          const uint8_t ck = Lf.kind[cs];
          if (ck == K_FLUID) {
            if (!reached[l + 1][cs] && !sealed[l + 1][cs]) {
              reached[l + 1][cs] = 1;
              queue.push_back({l + 1, cs});
            }
          } else if (ck == K_COVERED) {
            push_near_children(l + 1, cc, e);
          }
        }
  };
  while (!queue.empty()) {
    const auto [l, s] = queue.back();
    queue.pop_back();
    const LevelMesh& Lv = M->levels[l - 1];
    int c[3];
    Lv.cell(s, c);
    for (int i = 1; i <= 6; ++i) {
      const int e[3] = {CX[i], CY[i], CZ[i]};
      const int64_t ns = Lv.neighbour(s, e[0], e[1], e[2]);
      if (ns < 0) continue;
      if (crossq(l, s, i) < 1.0f || crossq(l, ns, opp(i)) < 1.0f) continue;
      const uint8_t nk = Lv.kind[ns];
      if (nk == K_FLUID) {
        if (!reached[l][ns] && !sealed[l][ns]) {
          reached[l][ns] = 1;
          queue.push_back({l, ns});
        }
      } else if (nk == K_COVERED) {
        int nc[3];
        Lv.cell(ns, nc);
        push_near_children(l, nc, e);
      } else if (nk == K_GHOST && l > 1) {
        const LevelMesh& Lp = M->levels[l - 2];
        const int nc[3] = {c[0] + e[0], c[1] + e[1], c[2] + e[2]};
        const int64_t ps = Lp.find_slot(nc[0] >> 1, nc[1] >> 1, nc[2] >> 1);
        if (ps < 0) continue;
        if (Lp.kind[ps] == K_FLUID && !reached[l - 1][ps] && !sealed[l - 1][ps]) {
          reached[l - 1][ps] = 1;
          queue.push_back({l - 1, ps});
        }
      }
    }
  }
  int64_t nsolid_total = 0;
  for (int l = 1; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s)
      if (Lv.kind[s] == K_FLUID && !reached[l][s]) {
        Lv.kind[s] = K_SOLID;
        ++Lv.counts[5];
        ++nsolid_total;
      }
  }
  // ghost slots: solid when their parent leaf is solid, else by parity (generator.jl:481-500)
  for (int l = 2; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    const LevelMesh& Lp = M->levels[l - 2];
    std::vector<int64_t> gl;
    for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s)
      if (Lv.kind[s] == K_GHOST) gl.push_back(s);
    std::vector<uint8_t> flags(gl.size(), 0);
    parallel_for((int64_t)gl.size(), [&](int, int64_t b, int64_t e) {
      std::vector<int32_t> st(stack_size);
      for (int64_t g = b; g < e; ++g) {
        int c[3];
        Lv.cell(gl[g], c);
        const int64_t ps = Lp.find_slot(c[0] >> 1, c[1] >> 1, c[2] >> 1);
        if (ps >= 0 && Lp.kind[ps] == K_SOLID) flags[g] = 1;
        else flags[g] = !no_geometry && bvh.is_inside(Lv.centre(gl[g]), st);
      }
    });
    for (size_t g = 0; g < gl.size(); ++g)
      if (flags[g]) Lv.kind[gl[g]] = K_SOLID;
  }
  // covered slots whose children are all solid (generator.jl:503-518)
  for (int l = L - 1; l >= 1; --l) {
    LevelMesh& Lv = M->levels[l - 1];
    const LevelMesh& Lf = M->levels[l];
    for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s) {
      if (Lv.kind[s] != K_COVERED) continue;
      int c[3];
      Lv.cell(s, c);
      bool allsolid = true;
      for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
          for (int di = 0; di < 2; ++di) {
            const int64_t cs = Lf.find_slot(2 * c[0] + di, 2 * c[1] + dj, 2 * c[2] + dk);
            if (cs < 0) continue;
            const uint8_t ck = Lf.kind[cs];
            if (!(ck == K_SOLID || (ck == K_COVERED && covered_solid[l + 1][cs]))) allsolid = false;
          }
      covered_solid[l][s] = allsolid;
    }
  }
  // leak check (generator.jl:520-537)
  int64_t leaks = 0;
  if (!no_geometry) {
    std::vector<int32_t> st(stack_size);
    for (int l = 1; l <= L; ++l) {
      LevelMesh& Lv = M->levels[l - 1];
      for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s)
        if (Lv.kind[s] == K_FLUID && near[l][s] && bvh.is_inside(Lv.centre(s), st)) {
          ++leaks;
          ++Lv.counts[9];
        }
    }
  }

  // ---- 5. cut links (generator.jl:543-600)
  std::vector<uint8_t> tri_hit(std::max(ntri_in, 1), 0);
  for (int l = 1; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    struct Link {
      int64_t slot;
      uint8_t dir;
      float q;
      int32_t tri;
      uint8_t ok;
    };
    std::vector<Link> links;
    for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s) {
      if (Lv.kind[s] != K_FLUID || !near[l][s]) continue;
      const int32_t row = nearrow[l][s];
      for (int i = 1; i < 19; ++i) {
        const int64_t ns = Lv.neighbour(s, CX[i], CY[i], CZ[i]);
        double q = cq[l][18 * (int64_t)(row - 1) + i - 1];
        int ti = ct[l][18 * (int64_t)(row - 1) + i - 1];
        bool cut = q < 1.0;
        if (!cut && ns >= 0) {
          const uint8_t nk = Lv.kind[ns];
          if (nk == K_SOLID || (nk == K_COVERED && covered_solid[l][ns])) {
            cut = true;
            q = 0.5;
            ti = -1;
          }
        } else if (!cut && ns < 0) {
          cut = true;
          q = 0.5;
          ti = -1;
        }
        if (!cut) continue;
        const int64_t ps = Lv.neighbour(s, -CX[i], -CY[i], -CZ[i]);
        bool ok = false;
        if (ps >= 0) {
          const uint8_t pk = Lv.kind[ps];
          if (pk == K_FLUID || pk == K_GHOST || (pk == K_COVERED && !covered_solid[l][ps]))
            ok = cq[l][18 * (int64_t)(row - 1) + opp(i) - 1] >= 1.0f;
        }
        links.push_back({s, (uint8_t)(i + 1), (float)std::max(q, 1e-6), ti >= 0 ? tri_src[ti] + 1 : 0, (uint8_t)ok});
      }
    }
    for (size_t li = 0; li < links.size(); ++li) {
      const Link& x = links[li];
      if (li == 0 || x.slot != links[li - 1].slot) {
        Lv.cut_slot.push_back((int32_t)(x.slot + 1));
        Lv.cut_off.push_back((int32_t)li + 1);
        Lv.cutidx[x.slot] = (int32_t)Lv.cut_slot.size();
      }
      Lv.cut_dir.push_back(x.dir);
      Lv.cut_q.push_back(x.q);
      Lv.cut_tri.push_back(no_geometry ? 0 : x.tri);
      Lv.cut_partner.push_back(x.ok);
      if (x.tri > 0 && !no_geometry) tri_hit[x.tri - 1] = 1;
      if (!x.ok) ++Lv.counts[10];
    }
    Lv.cut_off.push_back((int32_t)links.size() + 1);
  }
  // ---- 5a. transfers between levels (generator.jl:600-790)
  std::vector<std::vector<uint8_t>> restricted(L + 1), depth1(L + 1), inner(L + 1), referenced(L + 1), listed(L + 1);
  for (int l = 1; l <= L; ++l) {
    const int64_t ns = 8 * (int64_t)M->levels[l - 1].nocts;
    restricted[l].assign(ns, 0);
    depth1[l].assign(ns, 0);
    inner[l].assign(ns, 0);
    referenced[l].assign(ns, 0);
  }
  // (1) covered slots with a fluid leaf within 2 cells may carry a restricted state
  for (int l = 1; l < L; ++l) {
    const LevelMesh& Lv = M->levels[l - 1];
    for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s) {
      if (!(Lv.kind[s] == K_COVERED && !covered_solid[l][s])) continue;
      int c[3];
      Lv.cell(s, c);
      bool found = false, near1 = false;
      for (int dk = -2; dk <= 2; ++dk)
        for (int dj = -2; dj <= 2; ++dj)
          for (int di = -2; di <= 2; ++di) {
            int cc[3] = {c[0] + di, c[1] + dj, c[2] + dk};
            wrap_cell(Lv, cc);
            if (cc[0] < 0 || cc[1] < 0 || cc[2] < 0) continue;
            const int64_t ns = Lv.find_slot(cc[0], cc[1], cc[2]);
            if (ns >= 0 && Lv.kind[ns] == K_FLUID) {
              found = true;
              if (std::max(std::abs(di), std::max(std::abs(dj), std::abs(dk))) <= 1) near1 = true;
            }
          }
      restricted[l][s] = found;
      depth1[l][s] = near1;
    }
  }
  // inner ghosts: within one link of a fluid slot of their level
  for (int l = 2; l <= L; ++l) {
    const LevelMesh& Lv = M->levels[l - 1];
    for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s) {
      if (Lv.kind[s] != K_GHOST) continue;
      for (int j = 1; j < 19; ++j) {
        const int64_t ns = Lv.neighbour(s, -CX[j], -CY[j], -CZ[j]);
        if (ns >= 0 && Lv.kind[ns] == K_FLUID) {
          inner[l][s] = 1;
          break;
        }
      }
    }
  }
  // (2) restriction lists from the finest level down
  for (int l = L - 1; l >= 1; --l) {
    LevelMesh& Lv = M->levels[l - 1];
    const LevelMesh& Lf = M->levels[l];
    std::vector<int64_t> rs;
    for (int k = 0; k < 8; ++k)  // the reference's comprehension order: oct fastest, then slot
      for (int64_t o = 0; o < Lv.nocts; ++o)
        if (restricted[l][8 * o + k]) rs.push_back(8 * o + k);
    std::vector<int32_t> src(64 * rs.size(), 0);
    std::vector<uint8_t> cubic(rs.size(), 0);
    for (size_t ri = 0; ri < rs.size(); ++ri) {
      int c[3];
      Lv.cell(rs[ri], c);
      bool complete = true;
      for (int dk = 0; dk < 4; ++dk)
        for (int dj = 0; dj < 4; ++dj)
          for (int di = 0; di < 4; ++di) {
            int cc[3] = {2 * c[0] - 1 + di, 2 * c[1] - 1 + dj, 2 * c[2] - 1 + dk};
            wrap_cell(Lf, cc);
            const int64_t cs = (cc[0] < 0 || cc[1] < 0 || cc[2] < 0) ? -1 : Lf.find_slot(cc[0], cc[1], cc[2]);
            bool ok = false;
            if (cs >= 0) {
              const uint8_t ck = Lf.kind[cs];
              ok = ck == K_FLUID || ck == K_GHOST || (ck == K_COVERED && restricted[l + 1][cs]);
            }
            if (ok) src[64 * ri + di + 4 * dj + 16 * dk] = (int32_t)(cs + 1);
            else complete = false;
          }
      cubic[ri] = complete && depth1[l][rs[ri]];
      if (!cubic[ri])
        for (int nidx = 0; nidx < 64; ++nidx)
          if (!is_inner(nidx)) src[64 * ri + nidx] = 0;
    }
    std::vector<uint8_t> keep(rs.size(), 0);
    for (size_t ri = 0; ri < rs.size(); ++ri) {
      for (int m = 0; m < 8; ++m) keep[ri] |= src[64 * ri + stencil_inner(m)] != 0;
      if (!keep[ri]) restricted[l][rs[ri]] = 0;
    }
    for (size_t ri = 0; ri < rs.size(); ++ri) {
      if (!(keep[ri] && cubic[ri])) continue;
      for (int nidx = 0; nidx < 64; ++nidx) {
        const int32_t cs = src[64 * ri + nidx];
        if (cs && Lf.kind[cs - 1] == K_GHOST) referenced[l + 1][cs - 1] = 1;
      }
    }
    for (size_t ri = 0; ri < rs.size(); ++ri) {
      if (!keep[ri]) continue;
      Lv.restrict_slot.push_back((int32_t)(rs[ri] + 1));
      Lv.restrict_src.insert(Lv.restrict_src.end(), src.begin() + 64 * ri, src.begin() + 64 * (ri + 1));
      Lv.restrict_cubic.push_back(cubic[ri]);
    }
  }
  for (int l = 1; l <= L; ++l) {
    listed[l].resize(inner[l].size());
    for (size_t s = 0; s < inner[l].size(); ++s) listed[l][s] = inner[l][s] | referenced[l][s];
  }
  // (3) ghost donors: cubic over 4x4x4 coarse cells, else trilinear over the admissible subset, else solid
  auto donor_slot = [&](const LevelMesh& Lp, int lp, int ci, int cj, int ck, bool allow_ghost, bool isnear, V3 pc,
                        std::vector<int32_t>& st) -> int64_t {
    int c[3] = {ci, cj, ck};
    wrap_cell(Lp, c);
    if (c[0] < 0 || c[1] < 0 || c[2] < 0) return -1;
    const int64_t ds = Lp.find_slot(c[0], c[1], c[2]);
    if (ds < 0) return -1;
    const uint8_t kd = Lp.kind[ds];
    if (!(kd == K_FLUID || (kd == K_COVERED && restricted[lp][ds]) || (allow_ghost && kd == K_GHOST && listed[lp][ds])))
      return -1;
    if (isnear) {
      int ti;
      if (bvh.first_crossing(pc, Lp.centre(ds), st, &ti) < 1.0) return -1;
    }
    return ds;
  };
  // returns 2 cubic, 1 trilinear, 0 none
  auto set_ghost_donors = [&](LevelMesh& Lv, int l, size_t gi, int64_t s, std::vector<int32_t>& st) -> int {
    const LevelMesh& Lp = M->levels[l - 2];
    const V3 pc = Lv.centre(s);
    const bool isnear = near[l][s];
    const double fx = pc.x / Lp.dx - 0.5, fy = pc.y / Lp.dx - 0.5, fz = pc.z / Lp.dx - 0.5;
    const int i0 = (int)std::floor(fx), j0 = (int)std::floor(fy), k0 = (int)std::floor(fz);
    const double tx = fx - i0, ty = fy - j0, tz = fz - k0;
    double wx[4], wy[4], wz[4];
    cubic_weights(tx, wx);
    cubic_weights(ty, wy);
    cubic_weights(tz, wz);
    int32_t* don = &Lv.ghost_donor[64 * gi];
    float* w = &Lv.ghost_w[64 * gi];
    std::fill(don, don + 64, 0);
    std::fill(w, w + 64, 0.0f);
    bool complete = true;
    for (int dk = 0; dk < 4 && complete; ++dk)
      for (int dj = 0; dj < 4 && complete; ++dj)
        for (int di = 0; di < 4 && complete; ++di) {
          const int64_t ds = donor_slot(Lp, l - 1, i0 - 1 + di, j0 - 1 + dj, k0 - 1 + dk, false, isnear, pc, st);
          if (ds < 0) {
            complete = false;
            break;
          }
          don[di + 4 * dj + 16 * dk] = (int32_t)(ds + 1);
          w[di + 4 * dj + 16 * dk] = (float)(wx[di] * wy[dj] * wz[dk]);
        }
    if (complete) return 2;
    std::fill(don, don + 64, 0);
    std::fill(w, w + 64, 0.0f);
    double wsum = 0;
    for (int dk = 0; dk < 2; ++dk)
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          const int64_t ds = donor_slot(Lp, l - 1, i0 + di, j0 + dj, k0 + dk, true, isnear, pc, st);
          if (ds < 0) continue;
          const double ww = (di == 1 ? tx : 1 - tx) * (dj == 1 ? ty : 1 - ty) * (dk == 1 ? tz : 1 - tz);
          const int nidx = (di + 1) + 4 * (dj + 1) + 16 * (dk + 1);
          don[nidx] = (int32_t)(ds + 1);
          w[nidx] = (float)ww;
          wsum += ww;
        }
    if (!(wsum > 0)) return 0;
    for (int nidx = 0; nidx < 64; ++nidx) w[nidx] = (float)(w[nidx] / wsum);
    return 1;
  };
  for (int l = 2; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    std::vector<int64_t> gl;
    for (int k = 0; k < 8; ++k)
      for (int64_t o = 0; o < Lv.nocts; ++o)
        if (Lv.kind[8 * o + k] == K_GHOST && listed[l][8 * o + k]) gl.push_back(8 * o + k);
    Lv.ghost_donor.assign(64 * gl.size(), 0);
    Lv.ghost_w.assign(64 * gl.size(), 0.0f);
    std::vector<int> modes(gl.size(), 0);
    parallel_for((int64_t)gl.size(), [&](int, int64_t b, int64_t e) {
      std::vector<int32_t> st(stack_size);
      for (int64_t gi = b; gi < e; ++gi) modes[gi] = set_ghost_donors(Lv, l, (size_t)gi, gl[gi], st);
    });
    std::vector<int32_t> donors2;
    std::vector<float> w2;
    for (size_t gi = 0; gi < gl.size(); ++gi) {
      if (modes[gi] == 0) {
        Lv.kind[gl[gi]] = K_SOLID;
        listed[l][gl[gi]] = 0;
        continue;
      }
      Lv.ghost_slot.push_back((int32_t)(gl[gi] + 1));
      donors2.insert(donors2.end(), Lv.ghost_donor.begin() + 64 * gi, Lv.ghost_donor.begin() + 64 * (gi + 1));
      w2.insert(w2.end(), Lv.ghost_w.begin() + 64 * gi, Lv.ghost_w.begin() + 64 * (gi + 1));
    }
    Lv.ghost_donor.swap(donors2);
    Lv.ghost_w.swap(w2);
  }
  // (4a) a cubic restriction whose ghost source lost its donors averages its children instead
  for (int l = 1; l < L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    const LevelMesh& Lf = M->levels[l];
    for (size_t ri = 0; ri < Lv.restrict_slot.size(); ++ri) {
      if (!Lv.restrict_cubic[ri]) continue;
      bool bad = false;
      for (int nidx = 0; nidx < 64 && !bad; ++nidx) {
        const int32_t cs = Lv.restrict_src[64 * ri + nidx];
        if (!cs) continue;
        const uint8_t ck = Lf.kind[cs - 1];
        bad = ck == K_SOLID || (ck == K_GHOST && !listed[l + 1][cs - 1]);
      }
      if (!bad) continue;
      Lv.restrict_cubic[ri] = 0;
      for (int nidx = 0; nidx < 64; ++nidx)
        if (!is_inner(nidx)) Lv.restrict_src[64 * ri + nidx] = 0;
    }
  }
  // (4) a covered ghost donor must be restricted
  for (int l = 2; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    const LevelMesh& Lp = M->levels[l - 2];
    std::vector<int32_t> st(stack_size);
    for (size_t gi = 0; gi < Lv.ghost_slot.size(); ++gi)
      for (int nidx = 0; nidx < 64; ++nidx) {
        const int32_t ds = Lv.ghost_donor[64 * gi + nidx];
        if (!ds || !(Lp.kind[ds - 1] == K_COVERED && !restricted[l - 1][ds - 1])) continue;
        if (set_ghost_donors(Lv, l, gi, Lv.ghost_slot[gi] - 1, st) == 0)
          return fail(OAL_E_INVALID_ARG, "a ghost of level %d lost its donors to the restriction filter", l);
        break;
      }
  }
  // ---- 5b. special-direction masks (generator.jl:794-816)
  for (int l = 1; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    for (int64_t o = 0; o < Lv.nocts; ++o) {
      if (!Lv.real[o]) continue;
      for (int k = 0; k < 8; ++k) {
        const int64_t s = 8 * o + k;
        if (Lv.kind[s] != K_FLUID) continue;
        uint32_t m = 0;
        for (int j = 1; j < 19; ++j) {
          const int64_t ss = Lv.neighbour(s, -CX[j], -CY[j], -CZ[j]);
          if (ss < 0 || Lv.kind[ss] == K_BOUNDARY) m |= 1u << j;
        }
        const int ci = Lv.cutidx[s];
        if (ci)
          for (int li = Lv.cut_off[ci - 1] - 1; li < Lv.cut_off[ci] - 1; ++li) m |= 1u << opp(Lv.cut_dir[li] - 1);
        Lv.special[s] = m;
      }
    }
  }
  // ---- 6. counts
  int64_t unreached = 0;
  if (!no_geometry)
    for (int t = 0; t < ntri_in; ++t) unreached += !tri_hit[t];
  for (int l = 1; l <= L; ++l) {
    LevelMesh& Lv = M->levels[l - 1];
    int64_t* c = Lv.counts;
    c[0] = Lv.nocts;
    for (int a = 0; a < 3; ++a) c[1 + a] = Lv.n[a];
    for (int64_t s = 0; s < 8 * (int64_t)Lv.nocts; ++s) {
      c[4] += Lv.kind[s] == K_FLUID;
      c[6] += Lv.kind[s] == K_BOUNDARY;
      c[12] += Lv.special[s] != 0;
    }
    c[7] = (int64_t)Lv.cut_slot.size();
    c[8] = (int64_t)Lv.cut_dir.size();
    c[14] = (int64_t)Lv.ghost_slot.size();
    c[15] = (int64_t)Lv.restrict_slot.size();
    for (int i = 0; i < 16; ++i)
      if (i < 1 || i > 3) M->counts[i] += c[i];
  }
  for (int a = 0; a < 3; ++a) M->counts[1 + a] = M->levels[L - 1].n[a];
  M->counts[9] = leaks;
  M->counts[11] = unreached;
  (void)nsolid_total;
  return OAL_OK;
}

}  // namespace

extern "C" {

oal_status oal_q19_mesh_seal_counts(const oal_q19_mesh* mesh, int64_t* out) {
  if (!mesh || !out) return fail(OAL_E_INVALID_ARG, "null argument");
  out[0] = mesh->sealed;
  out[1] = mesh->unbracketed;
  return OAL_OK;
}

oal_status oal_q19_default_mesh_spec(oal_q19_mesh_spec* s) {
  if (!s) return fail(OAL_E_INVALID_ARG, "null argument");
  std::memset(s, 0, sizeof *s);
  s->dx = 1.0;
  s->levels = 1;
  s->band_fine = 8;
  s->band = 6;
  s->wake_level_offset = 1;
  s->wake_margin = 0.1;
  const int32_t faces[6] = {OAL_Q19_FACE_INLET, OAL_Q19_FACE_OUTLET, OAL_Q19_FACE_SLIP,
                            OAL_Q19_FACE_SLIP, OAL_Q19_FACE_SLIP, OAL_Q19_FACE_SLIP};
  std::memcpy(s->faces, faces, sizeof faces);
  return OAL_OK;
}

oal_status oal_q19_mesh_generate(const double* tri, int32_t ntri, const oal_q19_mesh_spec* spec, oal_q19_mesh** out) {
  if (!spec || !out || (ntri > 0 && !tri) || ntri < 0) return fail(OAL_E_INVALID_ARG, "bad arguments");
  *out = nullptr;
  if (!(spec->dx > 0)) return fail(OAL_E_INVALID_ARG, "dx must be positive");
  for (int a = 0; a < 3; ++a)
    if (!(spec->domain[a] > 0)) return fail(OAL_E_INVALID_ARG, "domain must be positive");
  for (int f = 0; f < 6; ++f) {
    const bool per = spec->periodic[f / 2] != 0;
    if (per != (spec->faces[f] == OAL_Q19_FACE_PERIODIC))
      return fail(OAL_E_INVALID_ARG, "face %d: periodic faces must be exactly those of the periodic axes", f);
    if (spec->faces[f] < OAL_Q19_FACE_PERIODIC || spec->faces[f] > OAL_Q19_FACE_FREESTREAM)
      return fail(OAL_E_INVALID_ARG, "face %d: unknown condition %d", f, spec->faces[f]);
  }
  if (spec->nregions < 0 || (spec->nregions > 0 && !spec->regions)) return fail(OAL_E_INVALID_ARG, "regions");
  if (spec->band_fine < 0 || spec->band < 0) return fail(OAL_E_INVALID_ARG, "bands must be non-negative");
  oal_q19_mesh* M = new oal_q19_mesh();
  oal_status s;
  try {
    s = generate(tri, ntri, spec, M);
  } catch (const std::bad_alloc&) {
    s = fail(OAL_E_OUT_OF_MEMORY, "mesh generation: host memory exhausted");
  }
  if (s != OAL_OK) {
    delete M;
    return s;
  }
  *out = M;
  return OAL_OK;
}

oal_status oal_q19_mesh_destroy(oal_q19_mesh* m) {
  delete m;
  return OAL_OK;
}

int32_t oal_q19_mesh_levels(const oal_q19_mesh* m) { return m ? m->L : 0; }

oal_status oal_q19_mesh_counts(const oal_q19_mesh* m, int32_t level, int64_t* out) {
  if (!m || !out) return fail(OAL_E_INVALID_ARG, "null argument");
  if (level < 0 || level > m->L) return fail(OAL_E_INVALID_ARG, "level %d of %d", level, m->L);
  std::memcpy(out, level == 0 ? m->counts : m->levels[level - 1].counts, 16 * sizeof(int64_t));
  return OAL_OK;
}

oal_status oal_q19_mesh_level_desc(const oal_q19_mesh* m, int32_t level, oal_q19_level_desc* d) {
  if (!m || !d) return fail(OAL_E_INVALID_ARG, "null argument");
  if (level < 1 || level > m->L) return fail(OAL_E_INVALID_ARG, "level %d of %d", level, m->L);
  const LevelMesh& Lv = m->levels[level - 1];
  std::memset(d, 0, sizeof *d);
  d->nocts = Lv.nocts;
  d->origin = Lv.origin.data();
  d->real = Lv.real.data();
  d->onbr = Lv.onbr.data();
  d->kind = Lv.kind.data();
  d->face = Lv.face.data();
  d->special = Lv.special.data();
  d->cutidx = Lv.cutidx.data();
  d->ncut = (int32_t)Lv.cut_slot.size();
  d->cut_slot = Lv.cut_slot.data();
  d->cut_off = Lv.cut_off.data();
  d->nlinks = (int32_t)Lv.cut_dir.size();
  d->cut_dir = Lv.cut_dir.data();
  d->cut_q = Lv.cut_q.data();
  d->cut_tri = Lv.cut_tri.data();
  d->cut_partner = Lv.cut_partner.data();
  d->ntri = m->ntri;
  for (int f = 0; f < 6; ++f) d->faces[f] = m->faces[f];
  d->nghost = (int32_t)Lv.ghost_slot.size();
  d->ghost_slot = Lv.ghost_slot.data();
  d->ghost_donor = Lv.ghost_donor.data();
  d->ghost_w = Lv.ghost_w.data();
  d->nrestrict = (int32_t)Lv.restrict_slot.size();
  d->restrict_slot = Lv.restrict_slot.data();
  d->restrict_src = Lv.restrict_src.data();
  d->restrict_cubic = Lv.restrict_cubic.data();
  return OAL_OK;
}

}  // extern "C"
