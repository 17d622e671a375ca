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

  // crossings of the +axis ray from p (geometry.jl:235-262). Hits at the same ray parameter (a ray
  // through an edge or vertex shared by several triangles) count once; the reference counts each
  // triangle, which miscounts a ray through a shared edge.
  int ray_crossings(V3 p, int axis, std::vector<int32_t>& stack) const {
    thread_local std::vector<double> hits;
    hits.clear();
    int sp = 0;
    stack[sp++] = 0;
    const int b1 = axis == 0 ? 1 : 0, b2 = axis == 2 ? 1 : 2;
    V3 dir{0, 0, 0};
    dir[axis] = 1.0;
    while (sp > 0) {
      const int id = stack[--sp];
      const V3 l = lo[id], h = hi[id];
      if (h[axis] < p[axis] || p[b1] < l[b1] || p[b1] > h[b1] || p[b2] < l[b2] || p[b2] > h[b2]) continue;
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

struct oal_q19_mesh {
  int n[3] = {0, 0, 0};
  double dx = 1.0;
  int periodic[3] = {0, 0, 0};
  int faces[6] = {0, 0, 0, 0, 0, 0};
  int32_t nocts = 0;
  std::vector<int32_t> origin;   // (3, nocts)
  std::vector<uint8_t> real;     // (nocts)
  std::vector<uint8_t> kind;     // (8, nocts)
  std::vector<uint8_t> face;     // (8, nocts)
  std::vector<int32_t> onbr;     // (27, nocts) 1-based
  std::vector<int32_t> cutidx;   // (8, nocts) 1-based, 0 none
  std::vector<uint32_t> special; // (8, nocts)
  std::vector<int32_t> cut_slot; // (ncut) 1-based slot id k + 8 (o - 1)
  std::vector<int32_t> cut_off;  // (ncut + 1) 1-based
  std::vector<uint8_t> cut_dir;  // (nlinks) 2..19 (reference numbering)
  std::vector<float> cut_q;
  std::vector<int32_t> cut_tri;  // 1-based original triangle, 0 none
  std::vector<uint8_t> cut_partner;
  int32_t ntri = 0;
  int64_t counts[16] = {};
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
  const double dx = spec->dx;
  const double domain[3] = {spec->domain[0], spec->domain[1], spec->domain[2]};
  const bool no_geometry = ntri_in == 0;
  M->dx = dx;
  M->ntri = ntri_in;
  for (int a = 0; a < 3; ++a) M->periodic[a] = spec->periodic[a] != 0;
  for (int f = 0; f < 6; ++f) M->faces[f] = spec->faces[f];
  // root grid: even cell counts; periodic axes must divide exactly (generator.jl:168-178)
  for (int a = 0; a < 3; ++a) {
    const double c = domain[a] / dx;
    if (M->periodic[a]) {
      const long r = std::lround(c);
      if (std::fabs((double)r - c) > 1e-9 * std::max(1.0, std::fabs(c)) || (r & 1) || r < 2)
        return fail(OAL_E_INVALID_ARG, "periodic axis %d: the domain must be an even number of cells", a);
      M->n[a] = (int)r;
    } else {
      int v = (int)std::ceil(c - 1e-9);
      v += v % 2;
      if (v < 2) return fail(OAL_E_INVALID_ARG, "axis %d: domain smaller than two cells", a);
      M->n[a] = v;
    }
  }
  const int* n = M->n;
  // ---- the surface, replicated across periodic faces (generator.jl:116-140)
  std::vector<Tri> tri;
  std::vector<int32_t> tri_src;
  if (no_geometry) {
    const double far = 1e6 * (1 + std::max(domain[0], std::max(domain[1], domain[2])));
    tri.push_back({{{far, far, far}, {far + 1, far, far}, {far, far + 1, far}}});
    tri_src.push_back(-1);
  } else {
    for (int t = 0; t < ntri_in; ++t) {
      Tri T;
      for (int v = 0; v < 3; ++v) T.v[v] = {tri_in[9 * t + 3 * v], tri_in[9 * t + 3 * v + 1], tri_in[9 * t + 3 * v + 2]};
      tri.push_back(T);
      tri_src.push_back(t);
    }
    const double margin = spec->band_fine * dx + 4 * dx;
    for (int a = 0; a < 3; ++a) {
      if (!M->periodic[a]) continue;
      double blo = INFINITY, bhi = -INFINITY;
      for (const Tri& T : tri)
        for (int v = 0; v < 3; ++v) {
          blo = std::min(blo, T.v[v][a]);
          bhi = std::max(bhi, T.v[v][a]);
        }
      if (bhi - blo >= domain[a] - 1e-9) {
        std::vector<Tri> keep;
        std::vector<int32_t> ksrc;
        for (size_t t = 0; t < tri.size(); ++t) {
          const double mx = std::max(tri[t].v[0][a], std::max(tri[t].v[1][a], tri[t].v[2][a]));
          const double mn = std::min(tri[t].v[0][a], std::min(tri[t].v[1][a], tri[t].v[2][a]));
          if (mx > 0 && mn < domain[a]) {
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
        sh[a] = domain[a];
        if (lo < margin) {
          extra.push_back({{vadd(tri[t].v[0], sh), vadd(tri[t].v[1], sh), vadd(tri[t].v[2], sh)}});
          esrc.push_back(tri_src[t]);
        }
        if (hi > domain[a] - margin) {
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

  // ---- octs: real octs of the root grid, boundary octs beyond non-periodic faces (generator.jl:278-350)
  auto wrap = [&](int p[3]) {
    bool inside = true;
    for (int a = 0; a < 3; ++a) {
      if (p[a] < 0 || p[a] >= n[a]) {
        if (M->periodic[a]) p[a] = ((p[a] % n[a]) + n[a]) % n[a];
        else inside = false;
      }
    }
    return inside;
  };
  auto key_of = [&](int x, int y, int z) -> int64_t {
    // origins lie in [-2, n]: shift by one oct so the key is non-negative
    return (((int64_t)(x + 2) / 2) * ((n[1] + 4) / 2) + (y + 2) / 2) * ((n[2] + 4) / 2) + (z + 2) / 2;
  };
  std::vector<std::array<int, 3>> origins;
  for (int k = 0; k < n[2]; k += 2)
    for (int j = 0; j < n[1]; j += 2)
      for (int i = 0; i < n[0]; i += 2) origins.push_back({i, j, k});
  const size_t nreal = origins.size();
  {
    std::map<int64_t, std::array<int, 3>> bset;
    for (size_t r = 0; r < nreal; ++r)
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dxo = -1; dxo <= 1; ++dxo) {
            if (!dxo && !dy && !dz) continue;
            int p[3] = {origins[r][0] + 2 * dxo, origins[r][1] + 2 * dy, origins[r][2] + 2 * dz};
            if (!wrap(p)) bset[key_of(p[0], p[1], p[2])] = {p[0], p[1], p[2]};
          }
    for (auto& kv : bset) origins.push_back(kv.second);
  }
  const int64_t nocts = (int64_t)origins.size();
  if (nocts * 27 > INT32_MAX) return fail(OAL_E_TOO_LARGE, "too many octs");
  std::vector<std::pair<uint64_t, int32_t>> order(nocts);
  for (int64_t o = 0; o < nocts; ++o)
    order[o] = {morton((origins[o][0] >> 1) + 1, (origins[o][1] >> 1) + 1, (origins[o][2] >> 1) + 1), (int32_t)o};
  std::sort(order.begin(), order.end());
  M->nocts = (int32_t)nocts;
  M->origin.assign(3 * nocts, 0);
  M->real.assign(nocts, 0);
  M->kind.assign(8 * nocts, K_NONE);
  M->face.assign(8 * nocts, 0);
  M->onbr.assign(27 * nocts, 0);
  M->cutidx.assign(8 * nocts, 0);
  M->special.assign(8 * nocts, 0);
  std::map<int64_t, int32_t> octmap;
  for (int64_t o = 0; o < nocts; ++o) {
    const int src = order[o].second;
    for (int a = 0; a < 3; ++a) M->origin[3 * o + a] = origins[src][a];
    const bool real = (size_t)src < nreal;
    M->real[o] = real;
    octmap[key_of(origins[src][0], origins[src][1], origins[src][2])] = (int32_t)o + 1;
    for (int k = 0; k < 8; ++k) {
      int x, y, z;
      slot_offset(k, x, y, z);
      if (real) {
        M->kind[8 * o + k] = K_FLUID;
      } else {
        const int c[3] = {origins[src][0] + x, origins[src][1] + y, origins[src][2] + z};
        uint8_t m = 0;
        if (c[0] < 0) m |= 1;
        if (c[0] >= n[0]) m |= 2;
        if (c[1] < 0) m |= 4;
        if (c[1] >= n[1]) m |= 8;
        if (c[2] < 0) m |= 16;
        if (c[2] >= n[2]) m |= 32;
        M->kind[8 * o + k] = K_BOUNDARY;
        M->face[8 * o + k] = m;
      }
    }
  }
  for (int64_t o = 0; o < nocts; ++o)
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dxo = -1; dxo <= 1; ++dxo) {
          int p[3] = {M->origin[3 * o] + 2 * dxo, M->origin[3 * o + 1] + 2 * dy, M->origin[3 * o + 2] + 2 * dz};
          wrap(p);
          bool in_range = true;  // octs exist only at origins in [-2, n] (the padding layer)
          for (int a = 0; a < 3; ++a) in_range = in_range && p[a] >= -2 && p[a] <= n[a];
          auto it = in_range ? octmap.find(key_of(p[0], p[1], p[2])) : octmap.end();
          M->onbr[27 * o + nbr_index(dxo, dy, dz)] = it == octmap.end() ? 0 : it->second;
        }
  auto centre = [&](int64_t o, int k) {
    int x, y, z;
    slot_offset(k, x, y, z);
    return V3{(M->origin[3 * o] + x + 0.5) * dx, (M->origin[3 * o + 1] + y + 0.5) * dx, (M->origin[3 * o + 2] + z + 0.5) * dx};
  };
  auto neighbour = [&](int64_t o, int k, int ex, int ey, int ez, int& no, int& nk) {
    int x, y, z;
    slot_offset(k, x, y, z);
    const int nx = x + ex, ny = y + ey, nz = z + ez;
    const int ox = clamp1(nx), oy = clamp1(ny), oz = clamp1(nz);
    no = M->onbr[27 * o + nbr_index(ox, oy, oz)] - 1;
    nk = slot_index(nx - 2 * ox, ny - 2 * oy, nz - 2 * oz);
  };

  // ---- near slots: within 2 cell diagonals of the surface (generator.jl:851-870)
  std::vector<uint8_t> near(8 * nocts, 0);
  const double bound = 2.0 * std::sqrt(3.0) * dx;
  parallel_for(nocts, [&](int, int64_t b, int64_t e) {
    std::vector<int32_t> st(stack_size);
    for (int64_t o = b; o < e; ++o) {
      const V3 oc{(M->origin[3 * o] + 1.0) * dx, (M->origin[3 * o + 1] + 1.0) * dx, (M->origin[3 * o + 2] + 1.0) * dx};
      const double d = bvh.nearest(oc, bound + std::sqrt(3.0) * dx, st);
      if (d >= bound + std::sqrt(3.0) * dx) continue;
      for (int k = 0; k < 8; ++k) {
        if (M->kind[8 * o + k] == K_BOUNDARY) continue;
        near[8 * o + k] = bvh.nearest(centre(o, k), bound, st) < bound;
      }
    }
  });
  // ---- crossings of every link of the near slots (generator.jl:352-378)
  std::vector<int32_t> nearrow(8 * nocts, 0);
  std::vector<int64_t> slots;
  for (int64_t s = 0; s < 8 * nocts; ++s)
    if (near[s] && M->kind[s] != K_BOUNDARY && M->kind[s] != K_COVERED) {
      slots.push_back(s);
      nearrow[s] = (int32_t)slots.size();
    }
  std::vector<float> cq(18 * slots.size(), 1.0f);
  std::vector<int32_t> ct(18 * slots.size(), -1);
  parallel_for((int64_t)slots.size(), [&](int, int64_t b, int64_t e) {
    std::vector<int32_t> st(stack_size);
    for (int64_t r = b; r < e; ++r) {
      const int64_t o = slots[r] / 8;
      const int k = (int)(slots[r] % 8);
      const V3 pc = centre(o, k);
      for (int i = 1; i < 19; ++i) {
        const V3 target{pc.x + CX[i] * dx, pc.y + CY[i] * dx, pc.z + CZ[i] * dx};
        int ti;
        const double q = bvh.first_crossing(pc, target, st, &ti);
        cq[18 * r + i - 1] = (float)q;
        ct[18 * r + i - 1] = ti;
      }
    }
  });
  auto crossq = [&](int64_t s, int i) -> float {  // q of link i of slot s (1 when not near)
    const int32_t row = nearrow[s];
    return row ? cq[18 * (int64_t)(row - 1) + i - 1] : 1.0f;
  };
  // ---- flood fill from the -x face over uncut face links (generator.jl:410-470)
  std::vector<uint8_t> reached(8 * nocts, 0);
  std::vector<int64_t> queue;
  {
    std::vector<int32_t> st(stack_size);
    for (int64_t o = 0; o < nocts; ++o) {
      if (!M->real[o] || M->origin[3 * o] != 0) continue;
      for (int k = 0; k < 8; ++k) {
        if ((k & 1) || M->kind[8 * o + k] != K_FLUID) continue;
        if (!no_geometry && bvh.is_inside(centre(o, k), st)) continue;
        if (!reached[8 * o + k]) {
          reached[8 * o + k] = 1;
          queue.push_back(8 * o + k);
        }
      }
    }
  }
  if (queue.empty()) return fail(OAL_E_INVALID_ARG, "no fluid cell on the inlet face: the geometry covers the -x face");
  const int face_dirs[6] = {1, 2, 3, 4, 5, 6};
  while (!queue.empty()) {
    const int64_t s = queue.back();
    queue.pop_back();
    const int64_t o = s / 8;
    const int k = (int)(s % 8);
    for (int i : face_dirs) {
      int no, nk;
      neighbour(o, k, CX[i], CY[i], CZ[i], no, nk);
      if (no < 0) continue;
      const int64_t ns = 8 * (int64_t)no + nk;
      if (crossq(s, i) < 1.0f || crossq(ns, opp(i)) < 1.0f) continue;
      if (M->kind[ns] == K_FLUID && !reached[ns]) {
        reached[ns] = 1;
        queue.push_back(ns);
      }
    }
  }
  int64_t nsolid = 0;
  for (int64_t s = 0; s < 8 * nocts; ++s)
    if (M->kind[s] == K_FLUID && !reached[s]) {
      M->kind[s] = K_SOLID;
      ++nsolid;
    }
  // leak check: fluid near slots inside by parity
  int64_t leaks = 0;
  if (!no_geometry) {
    std::vector<int32_t> st(stack_size);
    for (int64_t s = 0; s < 8 * nocts; ++s)
      if (M->kind[s] == K_FLUID && near[s] && bvh.is_inside(centre(s / 8, (int)(s % 8)), st)) ++leaks;
  }
  // ---- cut links (generator.jl:543-600)
  struct Link {
    int64_t slot;
    uint8_t dir;
    float q;
    int32_t tri;
    uint8_t ok;
  };
  std::vector<Link> links;
  for (int64_t s = 0; s < 8 * nocts; ++s) {
    if (M->kind[s] != K_FLUID || !near[s]) continue;
    const int64_t o = s / 8;
    const int k = (int)(s % 8);
    const int32_t row = nearrow[s];
    for (int i = 1; i < 19; ++i) {
      int no, nk;
      neighbour(o, k, CX[i], CY[i], CZ[i], no, nk);
      double q = cq[18 * (int64_t)(row - 1) + i - 1];
      int ti = ct[18 * (int64_t)(row - 1) + i - 1];
      bool cut = q < 1.0;
      if (!cut && no >= 0) {
        if (M->kind[8 * (int64_t)no + nk] == K_SOLID) {
          cut = true;
          q = 0.5;
          ti = -1;
        }
      } else if (!cut && no < 0) {
        cut = true;
        q = 0.5;
        ti = -1;
      }
      if (!cut) continue;
      int po, pk;
      neighbour(o, k, -CX[i], -CY[i], -CZ[i], po, pk);
      bool ok = false;
      if (po >= 0) {
        const uint8_t pkind = M->kind[8 * (int64_t)po + pk];
        if (pkind == K_FLUID || pkind == K_GHOST) ok = cq[18 * (int64_t)(row - 1) + opp(i) - 1] >= 1.0f;
      }
      links.push_back({s, (uint8_t)(i + 1), (float)std::max(q, 1e-6), ti >= 0 ? tri_src[ti] + 1 : 0, (uint8_t)ok});
    }
  }
  // (already in (slot, dir) order)
  int64_t missing_partner = 0;
  std::vector<uint8_t> tri_hit(std::max(ntri_in, 1), 0);
  for (size_t li = 0; li < links.size(); ++li) {
    const Link& x = links[li];
    if (li == 0 || x.slot != links[li - 1].slot) {
      M->cut_slot.push_back((int32_t)((x.slot % 8) + 1 + 8 * (x.slot / 8)));
      M->cut_off.push_back((int32_t)li + 1);
      M->cutidx[x.slot] = (int32_t)M->cut_slot.size();
    }
    M->cut_dir.push_back(x.dir);
    M->cut_q.push_back(x.q);
    M->cut_tri.push_back(x.tri);
    M->cut_partner.push_back(x.ok);
    if (x.tri > 0) tri_hit[x.tri - 1] = 1;
    if (!x.ok) ++missing_partner;
  }
  M->cut_off.push_back((int32_t)links.size() + 1);
  // ---- special-direction masks (generator.jl:794-816)
  for (int64_t o = 0; o < nocts; ++o) {
    if (!M->real[o]) continue;
    for (int k = 0; k < 8; ++k) {
      const int64_t s = 8 * o + k;
      if (M->kind[s] != K_FLUID) continue;
      uint32_t m = 0;
      int x, y, z;
      slot_offset(k, x, y, z);
      for (int j = 1; j < 19; ++j) {
        const int px = x - CX[j], py = y - CY[j], pz = z - CZ[j];
        const int ox = clamp1(px), oy = clamp1(py), oz = clamp1(pz);
        const int so = M->onbr[27 * o + nbr_index(ox, oy, oz)] - 1;
        const int child = slot_index(px - 2 * ox, py - 2 * oy, pz - 2 * oz);
        if (so < 0 || M->kind[8 * (int64_t)so + child] == K_BOUNDARY) m |= 1u << j;
      }
      const int ci = M->cutidx[s];
      if (ci)
        for (int li = M->cut_off[ci - 1] - 1; li < M->cut_off[ci] - 1; ++li) m |= 1u << opp(M->cut_dir[li] - 1);
      M->special[s] = m;
    }
  }
  // ---- counts
  int64_t fluid = 0, boundary = 0, special_slots = 0;
  for (int64_t s = 0; s < 8 * nocts; ++s) {
    fluid += M->kind[s] == K_FLUID;
    boundary += M->kind[s] == K_BOUNDARY;
    special_slots += M->special[s] != 0;
  }
  int64_t unreached = 0;
  for (int t = 0; t < ntri_in; ++t) unreached += !tri_hit[t];
  int64_t* c = M->counts;
  c[0] = nocts;
  c[1] = n[0];
  c[2] = n[1];
  c[3] = n[2];
  c[4] = fluid;
  c[5] = nsolid;
  c[6] = boundary;
  c[7] = (int64_t)M->cut_slot.size();
  c[8] = (int64_t)links.size();
  c[9] = leaks;
  c[10] = missing_partner;
  c[11] = unreached;
  c[12] = special_slots;
  c[13] = (int64_t)nreal;
  c[14] = (int64_t)tri.size();
  return OAL_OK;
}

}  // namespace

extern "C" {

oal_status oal_q19_default_mesh_spec(oal_q19_mesh_spec* s) {
  if (!s) return fail(OAL_E_INVALID_ARG, "null argument");
  std::memset(s, 0, sizeof *s);
  s->dx = 1.0;
  s->band_fine = 8;
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

oal_status oal_q19_mesh_counts(const oal_q19_mesh* m, int64_t* out) {
  if (!m || !out) return fail(OAL_E_INVALID_ARG, "null argument");
  std::memcpy(out, m->counts, sizeof m->counts);
  return OAL_OK;
}

oal_status oal_q19_mesh_level_desc(const oal_q19_mesh* m, oal_q19_level_desc* d) {
  if (!m || !d) return fail(OAL_E_INVALID_ARG, "null argument");
  std::memset(d, 0, sizeof *d);
  d->nocts = m->nocts;
  d->origin = m->origin.data();
  d->real = m->real.data();
  d->onbr = m->onbr.data();
  d->kind = m->kind.data();
  d->face = m->face.data();
  d->special = m->special.data();
  d->cutidx = m->cutidx.data();
  d->ncut = (int32_t)m->cut_slot.size();
  d->cut_slot = m->cut_slot.data();
  d->cut_off = m->cut_off.data();
  d->nlinks = (int32_t)m->cut_dir.size();
  d->cut_dir = m->cut_dir.data();
  d->cut_q = m->cut_q.data();
  d->cut_tri = m->cut_tri.data();
  d->cut_partner = m->cut_partner.data();
  d->ntri = m->ntri;
  for (int f = 0; f < 6; ++f) d->faces[f] = m->faces[f];
  return OAL_OK;
}

}  // extern "C"
