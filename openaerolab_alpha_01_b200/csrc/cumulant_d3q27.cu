// cumulant_d3q27.cu — fused pull-stream + D3Q27 cumulant collision for 8^3-cell blocks on sm_100a.
//
// Behaviour follows the reference's `stream_collide_cumulant!` (src/collision/kernel_cumulant.jl:
// 29-912) for a level without a parent: pull of 27 populations through the 27-entry neighbour
// table (:190-400), full-way bounce-back inside obstacle cells (:402-417), macros, sponge and
// wall model (:420-491), WALE eddy viscosity from the previous step's velocity (:496-595),
// cumulant relaxation (:597-844), positivity limiter (:849-884) and Guo forcing (:889-908). The
// half-way link rule with momentum exchange is the octree solver's
// (src/octree_q19/src/stream.jl:229-256) on the 27 links.
//
// The kernels share the collision code (cumulant_math.cuh):
//   k_fill_ghosts   writes, into ghost blocks around the level, the value every domain-face pull
//                   receives (inlet equilibrium, outlet copy, mirrors, walls, lattice weight), so
//                   the main kernel needs no face logic;
//   k_cumulant_pairs the uniform step of blocks without solids, sponge or wall model (FP32 and
//                   16-bit storage): two x-adjacent cells per thread in packed f32x2 arithmetic,
//                   one warp per z plane of a block;
//   k_cumulant_fast the same step one cell per thread (FP64 storage: a CTA of 128 threads covers
//                   a quarter block);
//   k_cumulant_gen  everything else, one cell per thread: per-cell solid masks (full-way or
//                   half-way walls with FP64 momentum exchange), sponge, wall model, Guo forcing,
//                   and the face conditions when the level has no ghost blocks (caller-owned
//                   arrays).
#include <algorithm>
#include <utility>
#include <vector>
#include <type_traits>

#include "common.cuh"
#include "vmath.cuh"
#include "cumulant_math.cuh"
#include "pairs_math.cuh"

// Tuning knobs of the uniform kernel (compile time): resident CTAs per SM the register budget
// is sized for, and cells per thread (2 = packed f32x2 pairs, 1 = scalar float).
#ifndef OAL_FAST_MIN_CTAS
#define OAL_FAST_MIN_CTAS 4
#endif
#ifndef OAL_FAST_CELLS
#define OAL_FAST_CELLS 2
#endif
// refined levels' ghost fill: resident CTAs per SM its registers are sized for, and whether the
// interpolation at a precomputed position is inlined
#ifndef OAL_PAR_FILL_MIN_CTAS
#define OAL_PAR_FILL_MIN_CTAS 4
#endif
#ifndef OAL_POS_NOINLINE
#define OAL_POS_NOINLINE 0
#endif
#if OAL_POS_NOINLINE
#define OAL_POS_LINKAGE __noinline__
#else
#define OAL_POS_LINKAGE
#endif
// threads per CTA of the x-pair kernel, one warp per z plane of a block: 32, 64, 128 or 256
// (measured on the config-2 channel: 64 best, 128 1 % slower, 32 2 %, 256 12 %)
#ifndef OAL_PAIRS_THREADS
#define OAL_PAIRS_THREADS 64
#endif
// resident warps per SM the x-pair kernel's registers are sized for, 16-bit storage (20: 96
// registers; 16 was 11 % slower on the FP16 config-2 channel, 24 spilled and was 2 % slower) and
// FP32 storage and the general-rate or positivity-limiter instances (whose wider state needs the
// 128 registers of 16 warps)
#ifndef OAL_PAIRS_WARPS
#define OAL_PAIRS_WARPS 20
#endif
#ifndef OAL_PAIRS_WARPS_WIDE
#define OAL_PAIRS_WARPS_WIDE 16
#endif

namespace oal {

// physics_utils.jl:5-17
__device__ __forceinline__ float gradient_noise(int32_t gx, int32_t gy, int32_t gz, int32_t seed) {
  uint32_t h = (uint32_t)gx * 374761393u + (uint32_t)gy * 668265263u + (uint32_t)gz * 1274126177u + (uint32_t)seed;
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  h = h ^ (h >> 16);
  return ((float)(h & 0xFFFFu) / 32768.0f) - 1.0f;
}

template <class S, class R>
__device__ __forceinline__ R dec_k(const S* __restrict__ f, int64_t i, int k) {
  return Codec<S>::dec(f[i], R(q27_w(k)), R(1.0 / q27_w(k)));
}

// ------------------------------------------------------------------------------------------------
// block AMR: parent interpolation of a refined level's pulls (physics_interpolation.jl:705-1198 at
// the reference's default flags: cubic Lagrange macros over the 64 parent nodes when all exist,
// else the trilinear / extrapolated macros of sample_parent_macro_for_fine_cell; cubic f_neq over
// the time-blended parent nodes; f_neq scaled by (tau_f - 1/2)/(tau_c - 1/2) and the
// post-collision factor (1 - omega_f)/(1 - omega_c))
// ------------------------------------------------------------------------------------------------
template <class R>
struct PNode {
  R f, rho, ux, uy, uz, fneq;
  bool ok;
};

// parent cell (1-based global index) -> element of the cell (block * 512 + cell), -1 when absent
__device__ __forceinline__ int64_t parent_cell(const ParentView& P, int pgx, int pgy, int pgz) {
  if (pgx < 1 || pgy < 1 || pgz < 1) return -1;
  const int pbx = (pgx - 1) / kBS + 1, pby = (pgy - 1) / kBS + 1, pbz = (pgz - 1) / kBS + 1;
  if (pbx > P.dim_x || pby > P.dim_y || pbz > P.dim_z) return -1;
  const int32_t pb = P.ptr[(pbx - 1) + (int64_t)P.dim_x * ((pby - 1) + (int64_t)P.dim_y * (pbz - 1))];
  if (pb <= 0) return -1;
  return (int64_t)(pb - 1) * kCells + (((pgx - 1) % kBS) | (((pgy - 1) % kBS) << 3) | (((pgz - 1) % kBS) << 6));
}

template <class R>
__device__ __forceinline__ void parent_bracket(R p_cont, int n, int& i0, int& i1, R& w) {
  if (n <= 1) { i0 = 1; i1 = 1; w = R(0); return; }
  const R pc = fmin(fmax(p_cont, R(1)), R(n));
  i0 = min(max((int)floor(pc), 1), n - 1);
  i1 = i0 + 1;
  w = fmin(fmax(pc - R(i0), R(0)), R(1));
}

// time-blended parent node c (a valid parent cell) in direction k: f, macros and f_neq
template <class S, class R>
__device__ PNode<R> parent_blended_at(const ParentView& P, int64_t c, int k, R wk, R cx, R cy, R cz, bool comp) {
  const int64_t n = (int64_t)P.nb * kCells;
  const int64_t fi = (c >> 9) * (27 * kCells) + k * kCells + (c & 511);
  const S* fn = static_cast<const S*>(P.f_new);
  const R* rn = static_cast<const R*>(P.rho_new);
  const R* vn = static_cast<const R*>(P.vel_new);
  R f = Codec<S>::dec(fn[fi], R(q27_w(k)), R(1.0 / q27_w(k)));
  R rho = rn[c], ux = vn[c], uy = vn[c + n], uz = vn[c + 2 * n];
  if (P.use_temporal == 1 && R(P.tw) < R(0.99) && P.f_old) {
    const R tw = R(P.tw);
    const S* fo = static_cast<const S*>(P.f_old);
    const R* ro = static_cast<const R*>(P.rho_old);
    const R* vo = static_cast<const R*>(P.vel_old);
    f = Codec<S>::dec(fo[fi], R(q27_w(k)), R(1.0 / q27_w(k))) * (R(1) - tw) + f * tw;
    rho = ro[c] * (R(1) - tw) + rho * tw;
    ux = vo[c] * (R(1) - tw) + ux * tw;
    uy = vo[c + n] * (R(1) - tw) + uy * tw;
    uz = vo[c + 2 * n] * (R(1) - tw) + uz * tw;
  }
  const R feqc = feq_c<R>(rho, ux, uy, uz, wk, cx, cy, cz, comp);
  return PNode<R>{f, rho, ux, uy, uz, f - feqc, true};
}

template <class R>
__device__ PNode<R> parent_macro_at(const ParentView& P, int64_t c) {
  const int64_t n = (int64_t)P.nb * kCells;
  const R* rn = static_cast<const R*>(P.rho_new);
  const R* vn = static_cast<const R*>(P.vel_new);
  R rho = rn[c], ux = vn[c], uy = vn[c + n], uz = vn[c + 2 * n];
  if (P.use_temporal == 1 && R(P.tw) < R(0.99) && P.rho_old) {
    const R tw = R(P.tw);
    const R* ro = static_cast<const R*>(P.rho_old);
    const R* vo = static_cast<const R*>(P.vel_old);
    rho = ro[c] * (R(1) - tw) + rho * tw;
    ux = vo[c] * (R(1) - tw) + ux * tw;
    uy = vo[c + n] * (R(1) - tw) + uy * tw;
    uz = vo[c + 2 * n] * (R(1) - tw) + uz * tw;
  }
  return PNode<R>{R(0), rho, ux, uy, uz, R(0), true};
}

// parent node lookups: the per-substep records when the level has them, else on the fly
template <class S, class R>
__device__ __forceinline__ PNode<R> parent_blended(const ParentView& P, int pgx, int pgy, int pgz, int k, R wk, R cx,
                                                   R cy, R cz, bool comp) {
  const int64_t c = parent_cell(P, pgx, pgy, pgz);
  if (c < 0) return PNode<R>{wk, R(1), R(0), R(0), R(0), R(0), false};
  if (P.node_map) {
    const int32_t i = P.node_map[c];
    if (i >= 0) {
      const R* v = static_cast<const R*>(P.node_vals) + (int64_t)i * 32;
      return PNode<R>{R(0), v[0], v[1], v[2], v[3], v[4 + k], true};
    }
  }
  return parent_blended_at<S, R>(P, c, k, wk, cx, cy, cz, comp);
}

template <class R>
__device__ __forceinline__ PNode<R> parent_macro(const ParentView& P, int pgx, int pgy, int pgz) {
  const int64_t c = parent_cell(P, pgx, pgy, pgz);
  if (c < 0) return PNode<R>{R(0), R(1), R(0), R(0), R(0), R(0), false};
  if (P.node_map) {
    const int32_t i = P.node_map[c];
    if (i >= 0) {
      const R* v = static_cast<const R*>(P.node_vals) + (int64_t)i * 32;
      return PNode<R>{R(0), v[0], v[1], v[2], v[3], R(0), true};
    }
  }
  return parent_macro_at<R>(P, c);
}

// One thread per needed parent node: its time-blended macros and the f_neq of the 27 directions,
// the same expressions the interpolation evaluates per stencil node
template <class S, class R>
__global__ void __launch_bounds__(256) k_parent_nodes(const ParentView P, const int32_t* __restrict__ nodes, int32_t n,
                                                      R* __restrict__ vals, int32_t comp) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = nodes[i];
  R* v = vals + (int64_t)i * 32;
  const PNode<R> m = parent_macro_at<R>(P, c);
  v[0] = m.rho; v[1] = m.ux; v[2] = m.uy; v[3] = m.uz;
#pragma unroll
  for (int k = 0; k < kQ27; ++k)
    v[4 + k] = parent_blended_at<S, R>(P, c, k, R(q27_w(k)), R(q27_cx(k)), R(q27_cy(k)), R(q27_cz(k)), comp != 0).fneq;
  v[31] = R(0);
}

template <class S, class R>
cudaError_t launch_parent_nodes(const ParentView& P, const int32_t* nodes, int32_t n, void* vals, int32_t comp,
                                cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_parent_nodes<S, R><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, nodes, n, static_cast<R*>(vals), comp);
  return cudaGetLastError();
}

template <class R>
__device__ __forceinline__ R lagrange3(int i, R w) {
  return i == -1 ? (-w * (w - R(1)) * (w - R(2)) / R(6))
       : i == 0  ? ((w + R(1)) * (w - R(1)) * (w - R(2)) / R(2))
       : i == 1  ? (-w * (w + R(1)) * (w - R(2)) / R(2))
                 : (w * (w + R(1)) * (w - R(1)) / R(6));
}
// the four cubic weights of one axis, lagrange3(-1 .. 2, w): evaluated once per stencil, so that a
// node's weight is two products ((lx ly) lz, the order of the direct product of three calls)
template <class R>
struct Lagrange4 {
  R v[4];
  __device__ __forceinline__ explicit Lagrange4(R w) {
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = lagrange3<R>(i - 1, w);
  }
};

// sample_parent_macro_for_fine_cell (physics_interpolation.jl:188-346)
template <class R>
__device__ bool parent_sample_macro(const ParentView& P, int fgx, int fgy, int fgz, R& r_out, R& x_out, R& y_out,
                                    R& z_out) {
  int px0, px1, py0, py1, pz0, pz1;
  R wx, wy, wz;
  parent_bracket<R>(R(fgx) * R(0.5) + R(0.25), P.dim_x * kBS, px0, px1, wx);
  parent_bracket<R>(R(fgy) * R(0.5) + R(0.25), P.dim_y * kBS, py0, py1, wy);
  parent_bracket<R>(R(fgz) * R(0.5) + R(0.25), P.dim_z * kBS, pz0, pz1, wz);
  PNode<R> d[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) d[c] = parent_macro<R>(P, (c & 1) ? px1 : px0, (c & 2) ? py1 : py0, (c & 4) ? pz1 : pz0);
  const R w[8] = {(R(1) - wx) * (R(1) - wy) * (R(1) - wz), wx * (R(1) - wy) * (R(1) - wz),
                  (R(1) - wx) * wy * (R(1) - wz),         wx * wy * (R(1) - wz),
                  (R(1) - wx) * (R(1) - wy) * wz,         wx * (R(1) - wy) * wz,
                  (R(1) - wx) * wy * wz,                  wx * wy * wz};
  bool all = true, any = false;
#pragma unroll
  for (int c = 0; c < 8; ++c) { all = all && d[c].ok; any = any || d[c].ok; }
  if (!all) {
    if (!any) { r_out = R(1); x_out = y_out = z_out = R(0); return false; }
    const int pxm = px0 - 1, pxp = px1 + 1, pym = py0 - 1, pyp = py1 + 1, pzm = pz0 - 1, pzp = pz1 + 1;
    // edges in the reference's order: along x, then y, then z; (a, b, far of a, far of b)
    const int ea[12] = {0, 2, 4, 6, 0, 1, 4, 5, 0, 1, 2, 3};
    const int eb[12] = {1, 3, 5, 7, 2, 3, 6, 7, 4, 5, 6, 7};
#pragma unroll 1
    for (int e = 0; e < 12; ++e) {
      const int a = ea[e], b = eb[e];
      if (d[a].ok == d[b].ok) continue;
      const int src = d[a].ok ? a : b, dst = d[a].ok ? b : a;
      // the far node continues the edge beyond the valid node
      int gx = (src & 1) ? px1 : px0, gy = (src & 2) ? py1 : py0, gz = (src & 4) ? pz1 : pz0;
      if (e < 4) gx = d[a].ok ? pxm : pxp;
      else if (e < 8) gy = d[a].ok ? pym : pyp;
      else gz = d[a].ok ? pzm : pzp;
      const PNode<R> fd = parent_macro<R>(P, gx, gy, gz);
      const PNode<R> s0 = d[src];
      d[dst].rho = fd.ok ? R(2) * s0.rho - fd.rho : s0.rho;
      d[dst].ux = fd.ok ? R(2) * s0.ux - fd.ux : s0.ux;
      d[dst].uy = fd.ok ? R(2) * s0.uy - fd.uy : s0.uy;
      d[dst].uz = fd.ok ? R(2) * s0.uz - fd.uz : s0.uz;
      d[dst].ok = true;
    }
  }
  R r = w[0] * d[0].rho, ux = w[0] * d[0].ux, uy = w[0] * d[0].uy, uz = w[0] * d[0].uz;
#pragma unroll
  for (int c = 1; c < 8; ++c) {
    r = r + w[c] * d[c].rho; ux = ux + w[c] * d[c].ux; uy = uy + w[c] * d[c].uy; uz = uz + w[c] * d[c].uz;
  }
  r_out = r; x_out = ux; y_out = uy; z_out = uz;
  return true;
}

// ---- interpolation at a precomputed position: the same arithmetic as parent_population below,
// with the stencil's node records listed per position and its macros evaluated once per substep
template <class R>
__device__ __forceinline__ void pos_record(const ParentView& P, const int32_t* nodes, int a, int b, int c,
                                           bool& ok, const R*& v) {
  const int32_t i = nodes[16 * (a + 1) + 4 * (b + 1) + (c + 1)];
  ok = i >= 0;
  v = static_cast<const R*>(P.node_vals) + (int64_t)(ok ? i : 0) * 32;
}

// interpolated macros of a position (the macro half of interpolate_with_rescaling, :924-1129)
template <class R>
__device__ void pos_macros(const ParentView& P, int32_t pos, int fgx, int fgy, int fgz, R* out) {
  const int32_t* nodes = P.pos_nodes + (int64_t)pos * 64;
  const int pnx = P.dim_x * kBS, pny = P.dim_y * kBS, pnz = P.dim_z * kBS;
  int px0, px1, py0, py1, pz0, pz1;
  R wx, wy, wz;
  parent_bracket<R>(R(fgx) * R(0.5) + R(0.25), pnx, px0, px1, wx);
  parent_bracket<R>(R(fgy) * R(0.5) + R(0.25), pny, py0, py1, wy);
  parent_bracket<R>(R(fgz) * R(0.5) + R(0.25), pnz, pz0, pz1, wz);
  const bool use_cubic = px0 - 2 >= 1 && px0 + 2 <= pnx && py0 - 2 >= 1 && py0 + 2 <= pny && pz0 - 2 >= 1 &&
                         pz0 + 2 <= pnz;
  bool all_valid = use_cubic;
  if (use_cubic)
    for (int i = 0; i < 64 && all_valid; ++i) all_valid = nodes[i] >= 0;
  R rho_i, ux_i, uy_i, uz_i;
  if (all_valid) {
    rho_i = ux_i = uy_i = uz_i = R(0);
    const Lagrange4<R> lx(wx), ly(wy), lz(wz);
#pragma unroll 4
    for (int i = 0; i < 64; ++i) {
      const int a = i >> 4, bb = (i >> 2) & 3, c = i & 3;
      const R* v = static_cast<const R*>(P.node_vals) + (int64_t)nodes[i] * 32;
      const R w3 = lx.v[a] * ly.v[bb] * lz.v[c];
      rho_i += w3 * v[0];
      ux_i += w3 * v[1];
      uy_i += w3 * v[2];
      uz_i += w3 * v[3];
    }
  } else {
    // sample_parent_macro_for_fine_cell on the stencil's corner records (far nodes a, b, c = -1 or 2)
    PNode<R> d[8];
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) {
      bool ok;
      const R* v;
      pos_record<R>(P, nodes, cc & 1, (cc >> 1) & 1, (cc >> 2) & 1, ok, v);
      d[cc] = ok ? PNode<R>{R(0), v[0], v[1], v[2], v[3], R(0), true} : PNode<R>{R(0), R(1), R(0), R(0), R(0), R(0), false};
    }
    const R w[8] = {(R(1) - wx) * (R(1) - wy) * (R(1) - wz), wx * (R(1) - wy) * (R(1) - wz),
                    (R(1) - wx) * wy * (R(1) - wz),         wx * wy * (R(1) - wz),
                    (R(1) - wx) * (R(1) - wy) * wz,         wx * (R(1) - wy) * wz,
                    (R(1) - wx) * wy * wz,                  wx * wy * wz};
    bool all = true, any = false;
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) { all = all && d[cc].ok; any = any || d[cc].ok; }
    bool sampled = true;
    if (!all) {
      if (!any) {
        sampled = false;
      } else {
        const int ea[12] = {0, 2, 4, 6, 0, 1, 4, 5, 0, 1, 2, 3};
        const int eb[12] = {1, 3, 5, 7, 2, 3, 6, 7, 4, 5, 6, 7};
#pragma unroll 1
        for (int e = 0; e < 12; ++e) {
          const int a = ea[e], b = eb[e];
          if (d[a].ok == d[b].ok) continue;
          const int src = d[a].ok ? a : b, dst = d[a].ok ? b : a;
          int ia = src & 1, ib = (src >> 1) & 1, ic = (src >> 2) & 1;
          if (e < 4) ia = d[a].ok ? -1 : 2;
          else if (e < 8) ib = d[a].ok ? -1 : 2;
          else ic = d[a].ok ? -1 : 2;
          bool fok;
          const R* fv;
          pos_record<R>(P, nodes, ia, ib, ic, fok, fv);
          const PNode<R> s0 = d[src];
          d[dst].rho = fok ? R(2) * s0.rho - fv[0] : s0.rho;
          d[dst].ux = fok ? R(2) * s0.ux - fv[1] : s0.ux;
          d[dst].uy = fok ? R(2) * s0.uy - fv[2] : s0.uy;
          d[dst].uz = fok ? R(2) * s0.uz - fv[3] : s0.uz;
          d[dst].ok = true;
        }
      }
    }
    if (sampled) {
      rho_i = w[0] * d[0].rho; ux_i = w[0] * d[0].ux; uy_i = w[0] * d[0].uy; uz_i = w[0] * d[0].uz;
#pragma unroll
      for (int cc = 1; cc < 8; ++cc) {
        rho_i = rho_i + w[cc] * d[cc].rho; ux_i = ux_i + w[cc] * d[cc].ux;
        uy_i = uy_i + w[cc] * d[cc].uy; uz_i = uz_i + w[cc] * d[cc].uz;
      }
    } else {
      // no corner exists: the trilinear blend of corners that all carry the absent node's
      // rho = 1, u = 0
      auto tri = [&](R a) {
        const R c00 = a * (R(1) - wx) + a * wx, c0 = c00 * (R(1) - wy) + c00 * wy;
        return c0 * (R(1) - wz) + c0 * wz;
      };
      rho_i = tri(R(1)); ux_i = uy_i = uz_i = tri(R(0));
    }
  }
  out[0] = rho_i; out[1] = ux_i; out[2] = uy_i; out[3] = uz_i;
}

// One thread per interpolation position of the level: its interpolated macros for this substep
template <class R>
__global__ void __launch_bounds__(256) k_parent_positions(const ParentView P, const int4* __restrict__ pos_xyz,
                                                          int32_t n, R* __restrict__ macro) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 q = pos_xyz[i];
  pos_macros<R>(P, i, q.x, q.y, q.z, macro + (int64_t)i * 4);
}

template <class R>
cudaError_t launch_parent_positions(const ParentView& P, const int4* pos_xyz, int32_t n, void* macro, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_parent_positions<R><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, pos_xyz, n, static_cast<R*>(macro));
  return cudaGetLastError();
}

// the direction-dependent half at a position: f_neq over the stencil's records, then
// feq(interpolated macros) + f_neq * scale (:1131-1198)
template <class R>
__device__ OAL_POS_LINKAGE R pos_population(const ParentView& P, int32_t pos, int fgx, int fgy, int fgz, int k, R cx, R cy, R cz,
                            bool comp) {
  const int32_t* nodes = P.pos_nodes + (int64_t)pos * 64;
  const R* mac = static_cast<const R*>(P.pos_macro) + (int64_t)pos * 4;
  const R wk = R(q27_w(k));
  const int pnx = P.dim_x * kBS, pny = P.dim_y * kBS, pnz = P.dim_z * kBS;
  int px0, px1, py0, py1, pz0, pz1;
  R wx, wy, wz;
  parent_bracket<R>(R(fgx) * R(0.5) + R(0.25), pnx, px0, px1, wx);
  parent_bracket<R>(R(fgy) * R(0.5) + R(0.25), pny, py0, py1, wy);
  parent_bracket<R>(R(fgz) * R(0.5) + R(0.25), pnz, pz0, pz1, wz);
  const bool use_cubic = px0 - 2 >= 1 && px0 + 2 <= pnx && py0 - 2 >= 1 && py0 + 2 <= pny && pz0 - 2 >= 1 &&
                         pz0 + 2 <= pnz;
  // corner records and the anchor (first existing corner in 000, 100, 010, 110, 001, ... order)
  int32_t corner[8];
#pragma unroll
  for (int cc = 0; cc < 8; ++cc) corner[cc] = nodes[16 * ((cc & 1) + 1) + 4 * (((cc >> 1) & 1) + 1) + ((cc >> 2) & 1) + 1];
  int anchor = 7;
#pragma unroll
  for (int cc = 6; cc >= 0; --cc)
    if (corner[cc] >= 0) anchor = cc;
  const R* vals = static_cast<const R*>(P.node_vals);
  // absent corner of a present anchor: the anchor's f_neq; no corner present: 0 (parent_blended's
  // absent node)
  const R anchor_neq = corner[anchor] >= 0 ? vals[(int64_t)corner[anchor] * 32 + 4 + k] : R(0);
  R f_neq = R(0);
  if (use_cubic) {
    const Lagrange4<R> lx(wx), ly(wy), lz(wz);
#pragma unroll 4
    for (int i = 0; i < 64; ++i) {
      const int a = i >> 4, bb = (i >> 2) & 3, c = i & 3;
      const int32_t ni = nodes[i];
      const R nv = ni >= 0 ? vals[(int64_t)ni * 32 + 4 + k] : anchor_neq;
      f_neq += lx.v[a] * ly.v[bb] * lz.v[c] * nv;
    }
  } else {
    R v[8];
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) v[cc] = corner[cc] >= 0 ? vals[(int64_t)corner[cc] * 32 + 4 + k] : anchor_neq;
    const R c00 = v[0] * (R(1) - wx) + v[1] * wx;
    const R c01 = v[4] * (R(1) - wx) + v[5] * wx;
    const R c10 = v[2] * (R(1) - wx) + v[3] * wx;
    const R c11 = v[6] * (R(1) - wx) + v[7] * wx;
    const R c0 = c00 * (R(1) - wy) + c10 * wy;
    const R c1 = c01 * (R(1) - wy) + c11 * wy;
    f_neq = c0 * (R(1) - wz) + c1 * wz;
  }
  const R feq_i = feq_c<R>(mac[0], mac[1], mac[2], mac[3], wk, cx, cy, cz, comp);
  const R tau_p = R(P.tau_parent), tau_f = R(P.tau_fine);
  const R tau_c = tau_p - R(0.5), tau_fm = tau_f - R(0.5);
  R scale = tau_c > R(1e-6) ? fmin(fmax(tau_fm / tau_c, R(0.01)), R(100)) : R(1);
  if (P.level_visc_physical == 1) scale = fmin(fmax(tau_f / (R(2) * fmax(tau_p, R(0.500001))), R(0.01)), R(100));
  const R omega_c = R(1) / fmax(tau_p, R(0.500001)), omega_f = R(1) / fmax(tau_f, R(0.500001));
  const R one_m_wc = R(1) - omega_c, one_m_wf = R(1) - omega_f;
  if (fabs(one_m_wc) > R(1e-6)) scale = fmin(fmax(scale * (one_m_wf / one_m_wc), R(0.01)), R(100));
  return feq_i + f_neq * scale;
}

// interpolate_with_rescaling at the fine cell (fgx, fgy, fgz) of the refined level, direction k
template <class S, class R>
__device__ __noinline__ R parent_population(const ParentView& P, int fgx, int fgy, int fgz, int k, R cx, R cy, R cz,
                                            bool comp) {
  const R wk = R(q27_w(k));
  const int pnx = P.dim_x * kBS, pny = P.dim_y * kBS, pnz = P.dim_z * kBS;
  int px0, px1, py0, py1, pz0, pz1;
  R wx, wy, wz;
  parent_bracket<R>(R(fgx) * R(0.5) + R(0.25), pnx, px0, px1, wx);
  parent_bracket<R>(R(fgy) * R(0.5) + R(0.25), pny, py0, py1, wy);
  parent_bracket<R>(R(fgz) * R(0.5) + R(0.25), pnz, pz0, pz1, wz);
  const bool use_cubic = px0 - 2 >= 1 && px0 + 2 <= pnx && py0 - 2 >= 1 && py0 + 2 <= pny && pz0 - 2 >= 1 &&
                         pz0 + 2 <= pnz;
  PNode<R> d[8];
#pragma unroll
  for (int c = 0; c < 8; ++c)
    d[c] = parent_blended<S, R>(P, (c & 1) ? px1 : px0, (c & 2) ? py1 : py0, (c & 4) ? pz1 : pz0, k, wk, cx, cy, cz,
                                comp);
  int anchor = 7;
#pragma unroll
  for (int c = 6; c >= 0; --c)
    if (d[c].ok) anchor = c;
  PNode<R> v[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) v[c] = d[c].ok ? d[c] : d[anchor];
  auto trilin = [&](R PNode<R>::*m) {
    const R c00 = (v[0].*m) * (R(1) - wx) + (v[1].*m) * wx;
    const R c01 = (v[4].*m) * (R(1) - wx) + (v[5].*m) * wx;
    const R c10 = (v[2].*m) * (R(1) - wx) + (v[3].*m) * wx;
    const R c11 = (v[6].*m) * (R(1) - wx) + (v[7].*m) * wx;
    const R c0 = c00 * (R(1) - wy) + c10 * wy;
    const R c1 = c01 * (R(1) - wy) + c11 * wy;
    return c0 * (R(1) - wz) + c1 * wz;
  };
  bool cubic_all_valid = use_cubic;
  if (use_cubic) {
#pragma unroll 1
    for (int i = 0; i < 64 && cubic_all_valid; ++i)
      if (parent_cell(P, px0 + (i >> 4) - 1, py0 + ((i >> 2) & 3) - 1, pz0 + (i & 3) - 1) < 0) cubic_all_valid = false;
  }
  R rho_i, ux_i, uy_i, uz_i;
  if (cubic_all_valid) {
    rho_i = ux_i = uy_i = uz_i = R(0);
    const Lagrange4<R> lx(wx), ly(wy), lz(wz);
#pragma unroll 1
    for (int i = 0; i < 64; ++i) {
      const int a = (i >> 4) - 1, bb = ((i >> 2) & 3) - 1, c = (i & 3) - 1;
      const PNode<R> m = parent_macro<R>(P, px0 + a, py0 + bb, pz0 + c);
      const R w3 = lx.v[a + 1] * ly.v[bb + 1] * lz.v[c + 1];
      rho_i += w3 * m.rho;
      ux_i += w3 * m.ux;
      uy_i += w3 * m.uy;
      uz_i += w3 * m.uz;
    }
  } else if (!parent_sample_macro<R>(P, fgx, fgy, fgz, rho_i, ux_i, uy_i, uz_i)) {
    rho_i = trilin(&PNode<R>::rho); ux_i = trilin(&PNode<R>::ux);
    uy_i = trilin(&PNode<R>::uy); uz_i = trilin(&PNode<R>::uz);
  }
  const R feq_i = feq_c<R>(rho_i, ux_i, uy_i, uz_i, wk, cx, cy, cz, comp);
  R f_neq = R(0);
  if (use_cubic) {
    const R anchor_neq = d[anchor].fneq;
    const Lagrange4<R> lx(wx), ly(wy), lz(wz);
#pragma unroll 1
    for (int i = 0; i < 64; ++i) {
      const int a = (i >> 4) - 1, bb = ((i >> 2) & 3) - 1, c = (i & 3) - 1;
      const PNode<R> nd = parent_blended<S, R>(P, px0 + a, py0 + bb, pz0 + c, k, wk, cx, cy, cz, comp);
      f_neq += lx.v[a + 1] * ly.v[bb + 1] * lz.v[c + 1] * (nd.ok ? nd.fneq : anchor_neq);
    }
  } else {
    f_neq = trilin(&PNode<R>::fneq);
  }
  const R tau_p = R(P.tau_parent), tau_f = R(P.tau_fine);
  const R tau_c = tau_p - R(0.5), tau_fm = tau_f - R(0.5);
  R scale = tau_c > R(1e-6) ? fmin(fmax(tau_fm / tau_c, R(0.01)), R(100)) : R(1);
  if (P.level_visc_physical == 1) scale = fmin(fmax(tau_f / (R(2) * fmax(tau_p, R(0.500001))), R(0.01)), R(100));
  const R omega_c = R(1) / fmax(tau_p, R(0.500001)), omega_f = R(1) / fmax(tau_f, R(0.500001));
  const R one_m_wc = R(1) - omega_c, one_m_wf = R(1) - omega_f;
  if (fabs(one_m_wc) > R(1e-6)) scale = fmin(fmax(scale * (one_m_wf / one_m_wc), R(0.01)), R(100));
  return feq_i + f_neq * scale;
}

// Population arriving at cell (x,y,z) of block b in direction k from outside every block
// (kernel_cumulant.jl:221-391), level without parent. `nbr` is the block's 27-entry row; entries
// >= n_real are ghost blocks, which count as missing here. k may be a run-time value.
template <class S, class R, bool DENSE = false, bool PAR = false>
__device__ __forceinline__ R face_population_impl(const S* __restrict__ fin, int64_t bbase, int cell, int64_t kst,
                                                  const int32_t* nbr, int n_real, int64_t bst, int k, int x, int y,
                                                  int z, int gx, int gy, int gz, const CaseParams& cp,
                                                  const StepArgs* da = nullptr) {
  // block layouts: own = bbase + cell; dense layout: bbase is the cell's own element, cell = 0
  const int64_t own = bbase + cell;
  const int cx = q27_cx(k), cy = q27_cy(k), cz = q27_cz(k);
  const int src_gx = gx - cx, src_gy = gy - cy, src_gz = gz - cz;
  const bool is_inlet = src_gx < 1, is_outlet = src_gx > cp.nx;
  const bool is_y_min = src_gy < 1, is_y_max = src_gy > cp.ny;
  const bool is_z_min = src_gz < 1, is_z_max = src_gz > cp.nz;
  const bool comp = (cp.flags & CF_COMPRESSIBLE) != 0;
  if (is_inlet) {
    const float noise = (cp.flags & CF_INLET_NOISE)
                            ? gradient_noise(gy, gz, cp.time_step_seed, 1234) * cp.inlet_turbulence * cp.u_inlet
                            : 0.0f;
    const R u_inst = R(cp.u_inlet) + R(noise);
    return feq_k<R>(k, R(1), u_inst, R(0), R(0), comp);
  }
  int j = k;             // own-cell direction that supplies the value, or
  int64_t src = -1;      // another cell's element (z-wall slip image)
  bool blend = false;    // transverse freestream
  if (is_outlet) {
    j = k;
  } else if ((cp.flags & (CF_ZWALL_SLIP | CF_ZWALL_NOSLIP)) && (is_z_min || is_z_max)) {
    if (cp.flags & CF_ZWALL_NOSLIP) {
      j = q27_opp(k);
    } else {
      j = q27_mir_z(k);
      if constexpr (DENSE) {
        // the image cell (x - cx, y - cy, z) of the box, wrapped on periodic axes
        int ix = gx - cx, iy = gy - cy;
        if (cp.flags & CF_PERIODIC_X) ix = ix < 1 ? ix + cp.nx : (ix > cp.nx ? ix - cp.nx : ix);
        if (cp.flags & CF_PERIODIC_Y) iy = iy < 1 ? iy + cp.ny : (iy > cp.ny ? iy - cp.ny : iy);
        if (ix >= 1 && ix <= cp.nx && iy >= 1 && iy <= cp.ny) src = dense_idx(*da, ix + 7, iy, gz) + j * kst;
      } else {
        const int zw_ix = x - cx, zw_iy = y - cy;
        if (zw_ix >= 0 && zw_ix < kBS && zw_iy >= 0 && zw_iy < kBS) {
          src = bbase + (zw_ix + 8 * zw_iy + 64 * z) + j * kst;
        } else {
          const int zw_nb = nbr[nbr_dir(zw_ix >> 3, zw_iy >> 3, 0)];
          if (zw_nb >= 0 && zw_nb < n_real) {
            src = (int64_t)zw_nb * bst + j * kst + ((zw_ix & 7) + 8 * (zw_iy & 7) + 64 * z);
          } else if (PAR && da && da->par.ptr && src_gy >= 1 && src_gy <= cp.ny) {
            // refined level: the image cell comes from the parent (kernel_cumulant.jl:286-312)
            return parent_population<S, R>(da->par, src_gx, src_gy, gz, j, R(cx), R(cy), R(-cz), comp);
          }
        }
      }
    }
  } else if ((cp.flags & CF_TRANSVERSE_FS) && (is_y_min || is_y_max || is_z_min || is_z_max)) {
    j = k;
    blend = true;
  } else if (is_y_min && (cp.flags & CF_YMIN_WALL)) {
    j = q27_opp(k);
  } else if (is_y_min || is_y_max) {
    j = q27_mir_y(k);
  } else if (is_z_min || is_z_max) {
    j = q27_mir_z(k);
  } else if (PAR && da && da->par.ptr) {
    // refined level: interpolated from the parent (kernel_cumulant.jl:346-388); the source is a
    // ghost cell whose interpolation position may be precomputed
    if (da->par.slot_pos && !DENSE) {
      const int sx = x - cx, sy = y - cy, sz = z - cz;
      const int g = nbr[nbr_dir(sx >> 3, sy >> 3, sz >> 3)];
      if (g >= n_real) {
        const int32_t pos = da->par.slot_pos[(int64_t)(g - n_real) * kCells + ((sx & 7) | ((sy & 7) << 3) | ((sz & 7) << 6))];
        if (pos >= 0) return pos_population<R>(da->par, pos, src_gx, src_gy, src_gz, k, R(cx), R(cy), R(cz), comp);
      }
    }
    return parent_population<S, R>(da->par, src_gx, src_gy, src_gz, k, R(cx), R(cy), R(cz), comp);
  } else {
    return R(q27_w(k));  // kernel_cumulant.jl:389-391
  }
  const R v = dec_k<S, R>(fin, src >= 0 ? src : own + j * kst, j);
  if (!blend) return v;
  const R beta = R(cp.transverse_blend);
  const R fe = feq_k<R>(k, R(1), R(cp.u_inlet), R(0), R(0), comp);
  return vfma(R(1) - beta, v, beta * fe);
}

// The general kernel calls the face logic from 27 unrolled sites; one out-of-line copy keeps
// its code small.
template <class S, class R>
__device__ __noinline__ R face_population(const S* __restrict__ fin, int64_t bbase, int cell, int64_t kst,
                                           const int32_t* nbr, int n_real, int64_t bst, int k, int x, int y, int z,
                                           int gx, int gy, int gz, const CaseParams& cp) {
  return face_population_impl<S, R>(fin, bbase, cell, kst, nbr, n_real, bst, k, x, y, z, gx, gy, gz, cp);
}

__device__ __forceinline__ const CaseParams& case_of(const StepArgs& a, int case_id) {
  return a.cases ? a.cases[case_id] : a.p0;
}

// ------------------------------------------------------------------------------------------------
// ghost fill: one thread per (destination cell, direction) whose pull source is a ghost cell
// ------------------------------------------------------------------------------------------------
// PAR: the level has a parent (its ghost pulls from inside the domain interpolate from it); the
// plain instance carries none of that code and stays small
template <class S, class R, bool DENSE, bool PAR>
__global__ void __launch_bounds__(256, PAR ? OAL_PAR_FILL_MIN_CTAS : 1) k_fill_ghosts(const StepArgs a, const uint2* __restrict__ entries, int64_t n) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  const uint2 en = entries[e];
  const int b = (int)en.x;
  const int cell = (int)(en.y & 511u), k = (int)((en.y >> 9) & 31u);
  const bool wrap = (en.y >> 31) != 0;  // dense periodic crossing: a copy of the wrapped interior cell
  const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
  const int4 bi = a.binfo[b];
  const CaseParams& cp = case_of(a, a.cases ? bi.w : 0);
  S* __restrict__ f = const_cast<S*>(static_cast<const S*>(a.f_in));
  const int32_t* nbr = a.nbr + (int64_t)b * 27;
  const int64_t bst = a.f_bstride, kst = a.f_kstride;
  const int gx = (bi.x - 1) * kBS + x + 1, gy = (bi.y - 1) * kBS + y + 1, gz = (bi.z - 1) * kBS + z + 1;
  const int cx = q27_cx(k), cy = q27_cy(k), cz = q27_cz(k);
  if constexpr (DENSE) {
    // ghost slot: the padded position of the source cell (1-based global g - c_k)
    const int64_t slot = dense_idx(a, gx - cx + 7, gy - cy, gz - cz) + k * kst;
    if (wrap) {
      int sx = gx - cx, sy = gy - cy, sz = gz - cz;
      sx = sx < 1 ? sx + cp.nx : (sx > cp.nx ? sx - cp.nx : sx);
      sy = sy < 1 ? sy + cp.ny : (sy > cp.ny ? sy - cp.ny : sy);
      sz = sz < 1 ? sz + cp.nz : (sz > cp.nz ? sz - cp.nz : sz);
      f[slot] = f[dense_idx(a, sx + 7, sy, sz) + k * kst];
      return;
    }
    const int64_t own = dense_idx(a, gx + 7, gy, gz);
    const R val = face_population_impl<S, R, true, PAR>(f, own, 0, kst, nbr, a.n_blocks, bst, k, x, y, z, gx, gy, gz, cp, &a);
    f[slot] = Codec<S>::enc(val, R(q27_w(k)), R(1.0 / q27_w(k)));
  } else {
    const R val = face_population_impl<S, R, false, PAR>(f, (int64_t)b * bst, cell, kst, nbr, a.n_blocks, bst, k, x, y, z, gx, gy,
                                             gz, cp, &a);
    const int sx = x - cx, sy = y - cy, sz = z - cz;
    const int g = nbr[nbr_dir(sx >> 3, sy >> 3, sz >> 3)];
    f[(int64_t)g * bst + k * kst + ((sx & 7) | ((sy & 7) << 3) | ((sz & 7) << 6))] =
        Codec<S>::enc(val, R(q27_w(k)), R(1.0 / q27_w(k)));
  }
}

// ------------------------------------------------------------------------------------------------
// fast kernel
// ------------------------------------------------------------------------------------------------
// two stored values of direction k -> one F2 (decoded), and back
template <class S>
__device__ __forceinline__ F2 load2(const S* __restrict__ f, int64_t i0, int64_t i1, int k) {
  if constexpr (std::is_same<S, float>::value) {
    return f2(f[i0], f[i1]);
  } else {
    float a, b;
    if constexpr (std::is_same<S, __half>::value) { a = __half2float(f[i0]); b = __half2float(f[i1]); }
    else { a = __bfloat162float(f[i0]); b = __bfloat162float(f[i1]); }
    const F2 w = splat<F2>(float(q27_w(k)));
    return vfma(f2(a, b), w, w);
  }
}
template <class S>
__device__ __forceinline__ void store2(S* __restrict__ f, int64_t i0, int64_t i1, F2 v, int k) {
  if constexpr (std::is_same<S, float>::value) {
    float a, b;
    f2split(v, a, b);
    f[i0] = a; f[i1] = b;
  } else {
    const F2 d = vfma(v, splat<F2>(float(1.0 / q27_w(k))), splat<F2>(-1.0f));
    float a, b;
    f2split(d, a, b);
    if constexpr (std::is_same<S, __half>::value) { f[i0] = __float2half_rn(a); f[i1] = __float2half_rn(b); }
    else { f[i0] = __float2bfloat16_rn(a); f[i1] = __float2bfloat16_rn(b); }
  }
}

// Library-owned block-major layout: block stride 27*512, direction stride 512 (compile time).
// IDX = uint32_t when the buffer (real + ghost blocks) has fewer than 2^32 elements.
template <class S, class V, class IDX>
__global__ void __launch_bounds__(128, OAL_FAST_MIN_CTAS) k_cumulant_fast(const StepArgs a, const int32_t* __restrict__ work) {
  constexpr int NL = Lane<V>::N;  // cells per thread
  constexpr int CPB = 4 / NL;     // CTAs per block
  using T = SC<V>;
  __shared__ int32_t s_nbr[28];
  __shared__ CaseParams s_cp;
  const int tid = threadIdx.x;
  const int b = work[blockIdx.x / CPB];
  const int part = blockIdx.x % CPB;
  if (tid < 27) s_nbr[tid] = a.nbr[(int64_t)b * 27 + tid];
  if (tid >= 32 && tid < 32 + (int)(sizeof(CaseParams) / 4)) {
    const int case_id = a.cases ? a.binfo[b].w : 0;
    reinterpret_cast<uint32_t*>(&s_cp)[tid - 32] = reinterpret_cast<const uint32_t*>(&case_of(a, case_id))[tid - 32];
  }
  __syncthreads();
  const CaseParams& cp = s_cp;

  const S* __restrict__ fin = static_cast<const S*>(a.f_in);
  S* __restrict__ fout = static_cast<S*>(a.f_out);
  T* __restrict__ rho_out = static_cast<T*>(a.rho_out);
  T* __restrict__ vel_out = static_cast<T*>(a.vel_out);
  const T* __restrict__ vel_in = static_cast<const T*>(a.vel_in);
  constexpr IDX bst = 27 * kCells, kst = kCells;
  const IDX vcs = (IDX)a.v_cstride;
  const int n_real = a.n_blocks;

  const int x = tid & 7, y = (tid >> 3) & 7;
  int z[NL];
  z[0] = 2 * part + (tid >> 6);
  if constexpr (NL == 2) z[1] = z[0] + 4;

  // ---- pull (kernel_cumulant.jl:190-220): every source lies in a real or ghost block ----
  V A[kQ27];
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const int sx = x - q27_cx(k), sy = y - q27_cy(k);
    IDX idx[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const int sz = z[l] - q27_cz(k);
      const int nb = s_nbr[nbr_dir(sx >> 3, sy >> 3, sz >> 3)];
      idx[l] = (IDX)nb * bst + (IDX)(k * kst) + (IDX)((sx & 7) | ((sy & 7) << 3) | ((sz & 7) << 6));
    }
    if constexpr (NL == 2) A[k] = load2<S>(fin, idx[0], idx[1], k);
    else A[k] = dec_k<S, T>(fin, idx[0], k);
  }
  // density in k order; the momentum sums skip the zero terms (adding +0 leaves a sum unchanged)
  V rho = A[0], jx = splat<V>(T(0)), jy = splat<V>(T(0)), jz = splat<V>(T(0));
#pragma unroll
  for (int k = 1; k < kQ27; ++k) rho = rho + A[k];
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    if (q27_cx(k)) jx = q27_cx(k) > 0 ? jx + A[k] : jx - A[k];
    if (q27_cy(k)) jy = q27_cy(k) > 0 ? jy + A[k] : jy - A[k];
    if (q27_cz(k)) jz = q27_cz(k) > 0 ? jz + A[k] : jz - A[k];
  }

  // ---- macros (kernel_cumulant.jl:424-431) ----
  rho = vmaxc(rho, T(0.01));
  const V inv_rho = vrcp(rho);
  const V ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  IDX vown[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) vown[l] = (IDX)b * kCells + (IDX)(x | (y << 3) | (z[l] << 6));
  if constexpr (NL == 2) {
    float r0, r1, a0, a1;
    f2split(rho, r0, r1); rho_out[vown[0]] = r0; rho_out[vown[1]] = r1;
    f2split(ux, a0, a1); vel_out[vown[0]] = a0; vel_out[vown[1]] = a1;
    f2split(uy, a0, a1); vel_out[vown[0] + vcs] = a0; vel_out[vown[1] + vcs] = a1;
    f2split(uz, a0, a1); vel_out[vown[0] + 2 * vcs] = a0; vel_out[vown[1] + 2 * vcs] = a1;
  } else {
    rho_out[vown[0]] = rho;
    vel_out[vown[0]] = ux; vel_out[vown[0] + vcs] = uy; vel_out[vown[0] + 2 * vcs] = uz;
  }

  // ---- WALE from the previous step's velocity (kernel_cumulant.jl:496-549) ----
  V nu_eddy = splat<V>(T(0));
  if (cp.flags & CF_GRADIENTS) {
    // neighbour velocity; the own value when the neighbour block is a ghost (physics_utils.jl:2031-2034)
    auto nbv = [&](int dx, int dy, int dz, int c) -> V {
      T v[NL];
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        const int nx = x + dx, ny = y + dy, nz = z[l] + dz;
        const int nb = s_nbr[nbr_dir(nx >> 3, ny >> 3, nz >> 3)];
        const IDX i = nb < n_real ? (IDX)nb * kCells + (IDX)((nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6)) : vown[l];
        v[l] = vel_in[i + (IDX)c * vcs];
      }
      if constexpr (NL == 2) return f2(v[0], v[1]);
      else return v[0];
    };
    const V h = splat<V>(T(0.5));
    const V g11 = h * (nbv(1, 0, 0, 0) - nbv(-1, 0, 0, 0));
    const V g12 = h * (nbv(0, 1, 0, 0) - nbv(0, -1, 0, 0));
    const V g13 = h * (nbv(0, 0, 1, 0) - nbv(0, 0, -1, 0));
    const V g21 = h * (nbv(1, 0, 0, 1) - nbv(-1, 0, 0, 1));
    const V g22 = h * (nbv(0, 1, 0, 1) - nbv(0, -1, 0, 1));
    const V g23 = h * (nbv(0, 0, 1, 1) - nbv(0, 0, -1, 1));
    const V g31 = h * (nbv(1, 0, 0, 2) - nbv(-1, 0, 0, 2));
    const V g32 = h * (nbv(0, 1, 0, 2) - nbv(0, -1, 0, 2));
    const V g33 = h * (nbv(0, 0, 1, 2) - nbv(0, 0, -1, 2));
    nu_eddy = wale_nu<V>(g11, g12, g13, g21, g22, g23, g31, g32, g33, cp.c_wale);
  }
  const V omega1 = omega1_from<V>(nu_eddy, cp);

  cumulant_collide<V>(A, rho, ux, uy, uz, omega1, cp);

  // ---- store (kernel_cumulant.jl:889-908 with zero force) ----
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    IDX o[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) o[l] = (IDX)b * bst + (IDX)(k * kst) + (IDX)(x | (y << 3) | (z[l] << 6));
    if constexpr (NL == 2) store2<S>(fout, o[0], o[1], A[k], k);
    else fout[o[0]] = Codec<S>::enc(A[k], T(q27_w(k)), T(1.0 / q27_w(k)));
  }
}

// ------------------------------------------------------------------------------------------------
// x-pair kernel: the uniform step with two x-adjacent cells (2i, 2i+1) per thread in packed f32x2
// ------------------------------------------------------------------------------------------------
// A direction's two stored values of a pair are one aligned word (2 x 16 bit or 2 x 32 bit), so
// the pull reads one word where the source pair is aligned (c_x = 0) and two words plus a lane
// shuffle within the register where it is not (c_x = +-1); the store writes one word. The WALE
// stencil reads pairs of the previous velocity. Same collision and the same per-cell results as
// the one-cell-per-lane kernels up to the rounding of the density and momentum sums, which are
// taken from the velocity-free x sums of the chimera transform.
template <class S> struct PairWord { using W = uint32_t; };
template <> struct PairWord<float> { using W = uint2; };

// (high element of q, low element of p): the pair straddling two aligned pairs
__device__ __forceinline__ uint32_t pair_mid(uint32_t q, uint32_t p) { return __byte_perm(q, p, 0x5432); }
__device__ __forceinline__ uint2 pair_mid(uint2 q, uint2 p) { return make_uint2(q.y, p.x); }

// the stored word of a direction -> the two values as stored (deviations d for 16-bit codecs)
template <class S> __device__ __forceinline__ F2 pair_raw(uint32_t w);
template <> __device__ __forceinline__ F2 pair_raw<__half>(uint32_t w) {
  const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w));
  return f2(f.x, f.y);
}
template <> __device__ __forceinline__ F2 pair_raw<__nv_bfloat16>(uint32_t w) {
  const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
  return f2(f.x, f.y);
}
__device__ __forceinline__ F2 pair_raw_f32(uint2 w) { return f2(__uint_as_float(w.x), __uint_as_float(w.y)); }

// populations of direction k -> the stored word (encode d = f / w - 1 for 16-bit codecs)
template <class S> __device__ __forceinline__ typename PairWord<S>::W pair_word(F2 v, int k);
template <> __device__ __forceinline__ uint32_t pair_word<__half>(F2 v, int k) {
  float a, b;
  f2split(vfma(v, splat<F2>(float(1.0 / q27_w(k))), splat<F2>(-1.0f)), a, b);
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
template <> __device__ __forceinline__ uint32_t pair_word<__nv_bfloat16>(F2 v, int k) {
  float a, b;
  f2split(vfma(v, splat<F2>(float(1.0 / q27_w(k))), splat<F2>(-1.0f)), a, b);
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
template <> __device__ __forceinline__ uint2 pair_word<float>(F2 v, int) {
  float a, b;
  f2split(v, a, b);
  return make_uint2(__float_as_uint(a), __float_as_uint(b));
}

// Stochastic rounding of the 16-bit deviations (the default writer of FP16/BF16 levels): the
// hardware conversion cvt.rs adds the random bits below the format's last place and truncates,
// so a stored value is unbiased in expectation; rounding to nearest rounds a slowly varying state
// the same way step after step, a bias that shows in integrated quantities (the sphere drag of
// the 256 x 128 x 128 channel drifts 3-5 % from FP64 in FP16 and up to 25 % in BF16 within 10,000
// steps with nearest rounding, 0.1-0.3 % and ~1 % with stochastic rounding). The random bits
// are a hash of the cell's position in its case and the low bits of the cell's new density and
// velocity, which change whenever the state does: a deterministic function of the case's own
// state, so single steps, captured graphs and batched members store identical values (no step
// counter to keep in step). The random operand's low 16 bits feed the lower half of the pair and
// its high 16 bits the upper half.
__device__ __forceinline__ uint32_t sr_hash(int gx, int gy, int gz, uint32_t state) {
  uint32_t h = (uint32_t)gx * 0x9E3779B1u ^ (uint32_t)gy * 0x85EBCA77u ^ (uint32_t)gz * 0xC2B2AE3Du ^ state;
  h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
  return h;
}
// odd multipliers: independent random words per direction from one hash
__host__ __device__ constexpr uint32_t sr_mult(int k) { return (2u * (uint32_t)k + 1u) * 0x9E3779B1u; }
template <class S> __device__ __forceinline__ uint32_t pack_dev_rs(F2 d, uint32_t r);
template <> __device__ __forceinline__ uint32_t pack_dev_rs<__half>(F2 d, uint32_t r) {
  float a, b;
  f2split(d, a, b);
  uint32_t out;
  asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(out) : "f"(b), "f"(a), "r"(r));
  return out;
}
template <> __device__ __forceinline__ uint32_t pack_dev_rs<__nv_bfloat16>(F2 d, uint32_t r) {
  float a, b;
  f2split(d, a, b);
  uint32_t out;
  asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(out) : "f"(b), "f"(a), "r"(r));
  return out;
}
template <> __device__ __forceinline__ uint32_t pack_dev_rs<float>(F2, uint32_t) { return 0u; }
// one deviation (lower half of the conversion, low 16 random bits)
template <class S> __device__ __forceinline__ S enc_rs(float d, uint32_t r) {
  uint32_t out;
  if constexpr (std::is_same<S, __half>::value)
    asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(out) : "f"(0.0f), "f"(d), "r"(r));
  else
    asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(out) : "f"(0.0f), "f"(d), "r"(r));
  const unsigned short lo = (unsigned short)(out & 0xFFFFu);
  return *reinterpret_cast<const S*>(&lo);
}

// two deviations -> the stored 16-bit pair, rounded to nearest
template <class S> __device__ __forceinline__ uint32_t pack_dev(F2 d);
template <> __device__ __forceinline__ uint32_t pack_dev<__half>(F2 d) {
  float a, b;
  f2split(d, a, b);
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
template <> __device__ __forceinline__ uint32_t pack_dev<__nv_bfloat16>(F2 d) {
  float a, b;
  f2split(d, a, b);
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
template <> __device__ __forceinline__ uint32_t pack_dev<float>(F2) { return 0u; }

// Library-owned block-major layout; IDX indexes words (pairs): block stride 27*256, direction
// stride 256, row (y, z) stride 4 and 32.
// One unit (a block's OAL_PAIRS_THREADS / 32 z planes) of the x-pair step; `unit` and `n_units`
// index the launch's units (the CTA's own in the plain form, a walked sequence in the persistent one).
template <class S, class IDX, bool POS, bool GEN>
__device__ __forceinline__ void pairs_unit(const StepArgs& a, unsigned unit, unsigned n_units, IDX* s_wbase,
                                           int32_t* s_nbr, int32_t* s_tail, CaseParams& s_cp, int32_t& s_pf) {
  constexpr bool DEV = !std::is_same<S, float>::value;  // 16-bit deviation codec
  constexpr float E = PairScale<DEV>::E;
  using W = typename PairWord<S>::W;
  using V = F2;
  using T = float;
  constexpr IDX wbst = 27 * kCells / 2, wkst = kCells / 2;
  const int tid = threadIdx.x;
  // a CTA covers OAL_PAIRS_THREADS / 32 z planes of a block (one warp per plane); the block's
  // neighbour row, coordinates and index come in one coalesced 128-byte record
  constexpr int CPB = 256 / OAL_PAIRS_THREADS;
  const int32_t* __restrict__ rec = a.fast_rec + (int64_t)(unit / CPB) * 32;
  const int part = unit % CPB;
  if (tid < 32) {
    const int32_t v = rec[tid];
    if (tid < 27) {
      s_nbr[tid] = v;
      s_wbase[tid] = (IDX)v * wbst;
    } else {
      s_tail[tid - 27] = v;
    }
  }
  // L2 prefetch of a later CTA's data (the CTA prefetch_ctas ahead in this launch): its block
  // index now, the bulk prefetches once this CTA's own loads are in flight
  if (tid == 32 % OAL_PAIRS_THREADS) {
    const unsigned pf_cta = unit + (unsigned)a.prefetch_ctas;
    s_pf = (a.prefetch_ctas > 0 && pf_cta < n_units) ? a.fast_rec[(int64_t)(pf_cta / CPB) * 32 + 31] : -1;
  }
  // the case parameters: copied by the second warp, or by the first one in one-warp CTAs
  const int cw = OAL_PAIRS_THREADS >= 64 ? tid - 32 : tid;
  if (cw >= 0 && cw < (int)(sizeof(CaseParams) / 4)) {
    const int case_id = a.cases ? rec[30] : 0;
    reinterpret_cast<uint32_t*>(&s_cp)[cw] = reinterpret_cast<const uint32_t*>(&case_of(a, case_id))[cw];
  }
  __syncthreads();
  const CaseParams& cp = s_cp;
  const int b = s_tail[4];

  const W* __restrict__ fin = static_cast<const W*>(a.f_in);
  W* __restrict__ fout = static_cast<W*>(a.f_out);
  float2* __restrict__ rho_out = static_cast<float2*>(a.rho_out);
  float* __restrict__ vel_out = static_cast<float*>(a.vel_out);
  const float* __restrict__ vel_in = static_cast<const float*>(a.vel_in);
  const IDX vcs = (IDX)a.v_cstride;
  const int n_real = a.n_blocks;

  const int i = tid & 3, y = (tid >> 2) & 7, z = (OAL_PAIRS_THREADS / 32) * part + (tid >> 5);
  if (tid < 30 && s_pf >= 0) {
    // one lane per direction: the later CTA's z planes of that direction are contiguous
    // (OAL_PAIRS_THREADS words); three lanes for its velocity components
    const IDX pz = (IDX)((OAL_PAIRS_THREADS / 32) * ((unit + (unsigned)a.prefetch_ctas) % CPB));
    if (tid < 27) {
      prefetch_l2(fin + (IDX)s_pf * wbst + (IDX)tid * wkst + 32 * pz, OAL_PAIRS_THREADS * (uint32_t)sizeof(W));
    } else if (cp.flags & CF_GRADIENTS) {
      prefetch_l2(vel_in + (IDX)(tid - 27) * vcs + (IDX)s_pf * kCells + 64 * pz, (OAL_PAIRS_THREADS / 32) * 64 * 4u);
    }
  }

  // ---- WALE stencil of the previous step's velocity (kernel_cumulant.jl:496-549): its loads
  // are issued before the pull so that both round trips to memory overlap ----
  const bool grad = (cp.flags & CF_GRADIENTS) != 0;
  const IDX cown = (IDX)b * kCells + (IDX)(2 * i + 8 * y + 64 * z);  // cell id of the pair's first cell
  float2 vo[3], vym[3], vyp[3], vzm[3], vzp[3];
  float vxm[3], vxp[3];
  if (grad) {
    // a neighbour in a ghost block contributes the own cell's value (physics_utils.jl:2031-2034)
    const int nb_xm = s_nbr[nbr_dir(-1, 0, 0)], nb_xp = s_nbr[nbr_dir(1, 0, 0)];
    const int nb_y = s_nbr[nbr_dir(0, y == 0 ? -1 : 0, 0)], nb_Y = s_nbr[nbr_dir(0, y == 7 ? 1 : 0, 0)];
    const int nb_z = s_nbr[nbr_dir(0, 0, z == 0 ? -1 : 0)], nb_Z = s_nbr[nbr_dir(0, 0, z == 7 ? 1 : 0)];
    const bool ok_xm = i > 0 || (unsigned)nb_xm < (unsigned)n_real;
    const bool ok_xp = i < 3 || (unsigned)nb_xp < (unsigned)n_real;
    const bool ok_ym = (unsigned)nb_y < (unsigned)n_real, ok_yp = (unsigned)nb_Y < (unsigned)n_real;
    const bool ok_zm = (unsigned)nb_z < (unsigned)n_real, ok_zp = (unsigned)nb_Z < (unsigned)n_real;
    const IDX c_xm = i > 0 ? cown - 1 : (IDX)nb_xm * kCells + (IDX)(7 + 8 * y + 64 * z);
    const IDX c_xp = i < 3 ? cown + 2 : (IDX)nb_xp * kCells + (IDX)(8 * y + 64 * z);
    const IDX c_ym = (IDX)nb_y * kCells + (IDX)(2 * i + 8 * ((y + 7) & 7) + 64 * z);
    const IDX c_yp = (IDX)nb_Y * kCells + (IDX)(2 * i + 8 * ((y + 1) & 7) + 64 * z);
    const IDX c_zm = (IDX)nb_z * kCells + (IDX)(2 * i + 8 * y + 64 * ((z + 7) & 7));
    const IDX c_zp = (IDX)nb_Z * kCells + (IDX)(2 * i + 8 * y + 64 * ((z + 1) & 7));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float* vc = vel_in + (IDX)c * vcs;
      vo[c] = reinterpret_cast<const float2*>(vc + cown)[0];
      vxm[c] = ok_xm ? vc[c_xm] : vo[c].x;
      vxp[c] = ok_xp ? vc[c_xp] : vo[c].y;
      vym[c] = ok_ym ? reinterpret_cast<const float2*>(vc + c_ym)[0] : vo[c];
      vyp[c] = ok_yp ? reinterpret_cast<const float2*>(vc + c_yp)[0] : vo[c];
      vzm[c] = ok_zm ? reinterpret_cast<const float2*>(vc + c_zm)[0] : vo[c];
      vzp[c] = ok_zp ? reinterpret_cast<const float2*>(vc + c_zp)[0] : vo[c];
    }
  }

  // ---- pull (kernel_cumulant.jl:190-220): every source lies in a real or ghost block ----
  V A[kQ27];
#pragma unroll
  for (int n = 0; n < 9; ++n) {
    // the three directions of one (c_y, c_z): their source rows share the neighbour block
    const int cy = n % 3 - 1, cz = n / 3 - 1;
    const int sy = y - cy, sz = z - cz;
    const int dyz = 3 * ((sy >> 3) + 1) + 9 * ((sz >> 3) + 1);
    const IDX row = (IDX)(((sy & 7) << 2) | ((sz & 7) << 5));
    const IDX own = s_wbase[1 + dyz] + row + (IDX)i;
    // the outer word of the row for the edge pairs: -x block's last pair (i = 0), +x block's first (i = 3)
    const IDX outer = i == 0 ? s_wbase[dyz] + row + 3 : s_wbase[2 + dyz] + row;
    const IDX left = i == 0 ? outer : own - 1, right = i == 3 ? outer : own + 1;
    const int k_m = 3 * n, k_0 = 3 * n + 1, k_p = 3 * n + 2;  // c_x = -1, 0, +1
    // c_x = -1: source x + 1 = (hi of own pair, lo of the right pair)
    const W pm = fin[own + (IDX)(k_m * wkst)], rm = fin[right + (IDX)(k_m * wkst)];
    const W p0 = fin[own + (IDX)(k_0 * wkst)];
    // c_x = +1: source x - 1 = (hi of the left pair, lo of own pair)
    const W pp = fin[own + (IDX)(k_p * wkst)], lp = fin[left + (IDX)(k_p * wkst)];
    if constexpr (std::is_same<S, float>::value) {
      A[k_m] = pair_raw_f32(pair_mid(pm, rm));
      A[k_0] = pair_raw_f32(p0);
      A[k_p] = pair_raw_f32(pair_mid(lp, pp));
    } else {
      // deviations; the decode f = w (1 + d) is folded into the x sums below
      A[k_m] = pair_raw<S>(pair_mid(pm, rm));
      A[k_0] = pair_raw<S>(p0);
      A[k_p] = pair_raw<S>(pair_mid(lp, pp));
    }
  }
  // WALE eddy viscosity from the stencil
  V nu_eddy = splat<V>(T(0));
  if (grad) {
    // twice the central differences (wale_nu_2g absorbs the factor)
    V g[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      g[c][0] = f2(vo[c].y, vxp[c]) - f2(vxm[c], vo[c].x);
      g[c][1] = f2(vyp[c].x, vyp[c].y) - f2(vym[c].x, vym[c].y);
      g[c][2] = f2(vzp[c].x, vzp[c].y) - f2(vzm[c].x, vzm[c].y);
    }
    nu_eddy = wale_nu_2g(g[0][0], g[0][1], g[0][2], g[1][0], g[1][1], g[1][2], g[2][0], g[2][1], g[2][2], cp.c_wale);
  }

  // raw moments (density and momentum among them), then the macros (kernel_cumulant.jl:424-431)
  raw_moments<DEV, GEN>(A);
  const V m000 = A[0];  // E x the unclamped density
  const V rc = pmaxc(m000, 0.01f * E);
  const V inv = vrcp(rc);
  const V i4 = DEV ? inv * splat<V>(0.25f) : inv;
  const V ux = i4 * A[1], uy = i4 * A[3], uz = i4 * A[9];
  const V rho = DEV ? rc * splat<V>(1.0f / E) : rc;
  {
    float r_0, r_1, a0, a1;
    f2split(rho, r_0, r_1);
    rho_out[cown >> 1] = make_float2(r_0, r_1);
    f2split(ux, a0, a1); reinterpret_cast<float2*>(vel_out + cown)[0] = make_float2(a0, a1);
    f2split(uy, a0, a1); reinterpret_cast<float2*>(vel_out + cown + vcs)[0] = make_float2(a0, a1);
    f2split(uz, a0, a1); reinterpret_cast<float2*>(vel_out + cown + 2 * vcs)[0] = make_float2(a0, a1);
  }

  const V omega1 = omega1_pairs(nu_eddy, cp);
  collide_scaled<DEV, GEN>(A, inv, ux, uy, uz, omega1, cp);

  // ---- store (kernel_cumulant.jl:889-908 with zero force): A[k] = f_k 2^n / rho_raw ----
  W* __restrict__ o = fout + (IDX)b * wbst + (IDX)(i + 4 * y + 32 * z);
  if (POS && (cp.flags & CF_LIMITER_POSITIVITY)) {
    // positivity limiter (kernel_cumulant.jl:849-884) on the populations themselves
    const V rr = DEV ? m000 * splat<V>(1.0f / E) : m000;
    const V sc[4] = {rr, rr * splat<V>(0.5f), rr * splat<V>(0.25f), rr * splat<V>(0.125f)};
#pragma unroll
    for (int k = 0; k < kQ27; ++k) A[k] = A[k] * sc[q27_d2(k)];
    V fmin = A[0];
#pragma unroll
    for (int k = 1; k < kQ27; ++k) fmin = vmin(fmin, A[k]);
    if (vany_gt(splat<V>(0.0f), fmin)) positivity_blend<V>(A, fmin, rho, ux, uy, uz, (cp.flags & CF_COMPRESSIBLE) != 0);
#pragma unroll
    for (int k = 0; k < kQ27; ++k) o[k * wkst] = pair_word<S>(A[k], k);
    return;
  }
  if constexpr (DEV) {
    // d_k = f_k / w_k - 1 = A[k] (27/8 rho_raw) 2^n - 1
    const V c0 = m000, c1 = c0 + c0, c2 = c1 + c1, c3 = c2 + c2;
    const V sc[4] = {c0, c1, c2, c3};
    if (a.round_nearest) {
#pragma unroll
      for (int k = 0; k < kQ27; ++k) o[k * wkst] = pack_dev<S>(vfma(A[k], sc[q27_d2(k)], splat<V>(-1.0f)));
    } else {
      const uint32_t st = __float_as_uint(f2lo(ux)) * 0x2545F491u + __float_as_uint(f2hi(uy)) + __float_as_uint(f2lo(uz));
      const uint32_t h = sr_hash((s_tail[0] - 1) * kBS + 2 * i, (s_tail[1] - 1) * kBS + y, (s_tail[2] - 1) * kBS + z, st);
#pragma unroll
      for (int k = 0; k < kQ27; ++k) o[k * wkst] = pack_dev_rs<S>(vfma(A[k], sc[q27_d2(k)], splat<V>(-1.0f)), h * sr_mult(k));
    }
  } else {
    const V c0 = m000, c1 = c0 * splat<V>(0.5f), c2 = c0 * splat<V>(0.25f), c3 = c0 * splat<V>(0.125f);
    const V sc[4] = {c0, c1, c2, c3};
#pragma unroll
    for (int k = 0; k < kQ27; ++k) o[k * wkst] = pair_word<S>(A[k] * sc[q27_d2(k)], k);
  }

}

// POS: some case of the launch uses the positivity limiter (its code is left out otherwise).
// GEN: some case of the launch relaxes with omega_bulk, omega3 or omega4 other than 1.
// PERS: the persistent form, resident CTAs walking the launch's units (launch tuning).
template <class S, class IDX, bool POS, bool GEN, bool PERS>
__global__ void __launch_bounds__(OAL_PAIRS_THREADS, ((sizeof(S) == 4 || GEN || POS) ? OAL_PAIRS_WARPS_WIDE : OAL_PAIRS_WARPS) * 32 / OAL_PAIRS_THREADS) k_cumulant_pairs(const StepArgs a, const int32_t* __restrict__ work) {
  (void)work;
  __shared__ IDX s_wbase[28];  // first word of each neighbour block
  __shared__ int32_t s_nbr[28];
  __shared__ int32_t s_tail[5];  // the block's coordinates and case (stochastic rounding), its index
  __shared__ CaseParams s_cp;
  __shared__ int32_t s_pf;
  if constexpr (PERS) {
    const unsigned n_units = (unsigned)a.pairs_units;
    for (unsigned unit = blockIdx.x; unit < n_units; unit += gridDim.x) {
      if (unit != blockIdx.x) __syncthreads();  // the previous unit no longer reads shared memory
      pairs_unit<S, IDX, POS, GEN>(a, unit, n_units, s_wbase, s_nbr, s_tail, s_cp, s_pf);
    }
  } else {
    pairs_unit<S, IDX, POS, GEN>(a, blockIdx.x, gridDim.x, s_wbase, s_nbr, s_tail, s_cp, s_pf);
  }
}

// ------------------------------------------------------------------------------------------------
// general kernel: one cell per thread, every option
// ------------------------------------------------------------------------------------------------
template <class S, class R, bool DENSE>
__global__ void __launch_bounds__(128) k_cumulant_gen(const StepArgs a, const int32_t* __restrict__ work) {
  __shared__ int32_t s_nbr[28];
  __shared__ CaseParams s_cp;
  __shared__ double s_mom[4][3];
  const int tid = threadIdx.x;
  const int b = work ? work[blockIdx.x >> 2] : a.block_base + (int)(blockIdx.x >> 2);
  const int part = blockIdx.x & 3;
  if (tid < 27) s_nbr[tid] = a.nbr[(int64_t)b * 27 + tid];
  const int4 bi = a.binfo[b];
  if (tid >= 32 && tid < 32 + (int)(sizeof(CaseParams) / 4))
    reinterpret_cast<uint32_t*>(&s_cp)[tid - 32] =
        reinterpret_cast<const uint32_t*>(&case_of(a, a.cases ? bi.w : 0))[tid - 32];
  __syncthreads();
  const CaseParams& cp = s_cp;
  const uint32_t flags = cp.flags;
  const uint32_t bflags = a.bflags[b];

  const S* __restrict__ fin = static_cast<const S*>(a.f_in);
  S* __restrict__ fout = static_cast<S*>(a.f_out);
  S* __restrict__ fpost = static_cast<S*>(a.f_post);
  R* __restrict__ rho_out = static_cast<R*>(a.rho_out);
  R* __restrict__ vel_out = static_cast<R*>(a.vel_out);
  const R* __restrict__ vel_in = static_cast<const R*>(a.vel_in);
  R* __restrict__ pi_neq = static_cast<R*>(a.pi_neq);
  const int64_t bst = a.f_bstride, kst = a.f_kstride, vcs = a.v_cstride;
  const int n_real = a.n_blocks;

  const int x = tid & 7, y = (tid >> 3) & 7, z = 2 * part + (tid >> 6);
  const int cell = x | (y << 3) | (z << 6);
  const int gx = (bi.x - 1) * kBS + x + 1, gy = (bi.y - 1) * kBS + y + 1, gz = (bi.z - 1) * kBS + z + 1;
  // own element of direction 0: block layouts b*bst + cell; dense layout the padded grid position
  const int64_t own = DENSE ? dense_idx(a, gx + 7, gy, gz) : (int64_t)b * bst + cell;
  const int64_t vown = (int64_t)b * kCells + cell;
  const bool store_post = (flags & CF_STORE_POST) && fpost;

  uint32_t mask = 0;
  if (bflags & BF_NEAR_SOLID) mask = a.cmask[(int64_t)a.mslot[b] * kCells + cell];
  const bool is_obs = (mask >> 13) & 1u;
  const bool halfway = (flags & CF_HALFWAY) != 0;
  double mx = 0.0, my = 0.0, mz = 0.0;

  if (is_obs && halfway) {
    // half-way mode: a solid cell holds the rest equilibrium; no fluid cell reads it
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      const S v = Codec<S>::enc(R(q27_w(k)), R(q27_w(k)), R(1.0 / q27_w(k)));
      fout[own + k * kst] = v;
      if (store_post) fpost[own + k * kst] = v;
    }
    rho_out[vown] = R(1);
    vel_out[vown] = R(0); vel_out[vown + vcs] = R(0); vel_out[vown + 2 * vcs] = R(0);
    if (flags & CF_SGS_PI) {
#pragma unroll
      for (int m = 0; m < 6; ++m) pi_neq[vown + m * vcs] = R(0);
    }
  } else {
    // ---- pull (kernel_cumulant.jl:190-400): where every source lies in a block (ghost blocks
    // included), the stored word of the neighbour and, for half-way links, the own cell's
    // opposite word are both read without a branch, so that all loads are in flight together ----
    R A[kQ27];
    S raw[kQ27], rawo[kQ27];
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      const int cx = q27_cx(k), cy = q27_cy(k), cz = q27_cz(k);
      const int sx = x - cx, sy = y - cy, sz = z - cz;
      const int nb = DENSE ? 0 : s_nbr[nbr_dir(sx >> 3, sy >> 3, sz >> 3)];
      if (DENSE) {
        // the padded grid holds every source, ghost frame included
        raw[k] = fin[own - cx - (int64_t)cy * a.PX - (int64_t)cz * a.PX * a.PY + k * kst];
      } else {
        raw[k] = fin[(int64_t)(nb >= 0 ? nb : b) * bst + k * kst + ((sx & 7) | ((sy & 7) << 3) | ((sz & 7) << 6))];
      }
      rawo[k] = halfway ? fin[own + q27_opp(k) * kst] : raw[k];
    }
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      const int cx = q27_cx(k), cy = q27_cy(k), cz = q27_cz(k);
      const int sx = x - cx, sy = y - cy, sz = z - cz;
      const int nb = DENSE ? 0 : s_nbr[nbr_dir(sx >> 3, sy >> 3, sz >> 3)];
      R val;
      if (DENSE || nb >= 0) {
        if (halfway && ((mask >> k) & 1u)) {
          // the link opp(k) of this cell is cut: its own post-collision population returns
          const int i = q27_opp(k);
          const R fi = Codec<S>::dec(rawo[k], R(q27_w(i)), R(1.0 / q27_w(i)));
          val = fi;
          if (flags & CF_COLLECT) {
            const double mom = 2.0 * (double)fi;  // (f_i* + f_k(t+1)) c_i with c_i = -c_k
            mx -= mom * cx; my -= mom * cy; mz -= mom * cz;
          }
        } else {
          val = Codec<S>::dec(raw[k], R(q27_w(k)), R(1.0 / q27_w(k)));
        }
      } else {
        val = face_population<S, R>(fin, (int64_t)b * bst, cell, kst, s_nbr, n_real, bst, k, x, y, z, gx, gy, gz, cp);
      }
      A[k] = val;
    }
    R rho = A[0], jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
    for (int k = 1; k < kQ27; ++k) rho = rho + A[k];
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      if (q27_cx(k)) jx = q27_cx(k) > 0 ? jx + A[k] : jx - A[k];
      if (q27_cy(k)) jy = q27_cy(k) > 0 ? jy + A[k] : jy - A[k];
      if (q27_cz(k)) jz = q27_cz(k) > 0 ? jz + A[k] : jz - A[k];
    }

    if (is_obs) {
      // simple bounce-back inside the obstacle (kernel_cumulant.jl:402-417)
      rho_out[vown] = R(1);
      vel_out[vown] = R(0); vel_out[vown + vcs] = R(0); vel_out[vown + 2 * vcs] = R(0);
#pragma unroll
      for (int k = 0; k < kQ27; ++k) {
        const S v = Codec<S>::enc(A[q27_opp(k)], R(q27_w(k)), R(1.0 / q27_w(k)));
        fout[own + k * kst] = v;
        if (store_post) fpost[own + k * kst] = v;
      }
      if (flags & CF_SGS_PI) {
#pragma unroll
        for (int m = 0; m < 6; ++m) pi_neq[vown + m * vcs] = R(0);
      }
    } else {
      // ---- macros, sponge, wall model (kernel_cumulant.jl:420-491) ----
      rho = vmaxc(rho, R(0.01));
      const R inv_rho = vrcp(rho);
      R ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
      const bool comp = (flags & CF_COMPRESSIBLE) != 0;
      if (a.sponge) {
        const R sp = R(a.sponge[vown]);
        if (sp > R(0)) {
          const R ut = R(cp.u_inlet), ms = R(1) - sp;
          rho = vfma(rho, ms, sp);
          ux = vfma(ux, ms, ut * sp);
          uy = uy * ms;
          uz = uz * ms;
          if (flags & CF_SPONGE_BLEND) {
#pragma unroll
            for (int k = 0; k < kQ27; ++k) A[k] = vfma(A[k], ms, feq_k<R>(k, R(1), ut, R(0), R(0), comp) * sp);
          }
        }
      }
      R Fx = R(0), Fy = R(0), Fz = R(0);
      if ((flags & CF_WALL_MODEL) && a.wall_dist) {
        const R dw = R(a.wall_dist[vown]);
        if (dw > R(0) && dw < R(cp.wall_model_max_distance)) {
          const R u_mag = sqrt(ux * ux + uy * uy + uz * uz);
          const R nu_visc = (R(cp.tau) - R(0.5)) * R(1.0 / 3.0);
          if (u_mag > R(1e-6) && nu_visc > R(1e-10)) {
            R u_tau = u_mag * pow(nu_visc / (dw * u_mag + R(1e-10)), R(1) / R(7)) * pow(R(2) * R(8.3), -R(1) / R(7));
            u_tau = u_tau > R(1e-6) ? u_tau : R(1e-6);
            const R y_p = u_tau * dw / nu_visc;
            if (y_p > R(11.81)) {
              const R u_plus = (R(1) / R(0.41)) * log(y_p) + R(5.2);
              if (u_plus > R(0.1)) {
                u_tau = u_tau * ((u_mag / u_tau) / u_plus);
                u_tau = u_tau > R(1e-6) ? u_tau : R(1e-6);
              }
            }
            const R tau_wall = rho * u_tau * u_tau;
            const R tau_res = rho * nu_visc * (u_mag / dw);
            if (tau_wall > tau_res) {
              const R fm = (tau_wall - tau_res) / dw;
              Fx = -fm * ux / u_mag; Fy = -fm * uy / u_mag; Fz = -fm * uz / u_mag;
            }
          }
        }
      }
      const R uxe = vfma(R(0.5) * Fx, inv_rho, ux);
      const R uye = vfma(R(0.5) * Fy, inv_rho, uy);
      const R uze = vfma(R(0.5) * Fz, inv_rho, uz);
      rho_out[vown] = rho;
      vel_out[vown] = ux; vel_out[vown + vcs] = uy; vel_out[vown + 2 * vcs] = uz;

      // ---- WALE (kernel_cumulant.jl:496-549): own value for missing, ghost or solid neighbours ----
      R nu_eddy = R(0), nu_dyn = R(0);
      if (flags & CF_GRADIENTS) {
        auto nbv = [&](int dx, int dy, int dz, int c, uint32_t solid) -> R {
          const int nx = x + dx, ny = y + dy, nz = z + dz;
          const int nb = s_nbr[nbr_dir(nx >> 3, ny >> 3, nz >> 3)];
          const bool own_v = nb < 0 || nb >= n_real || solid;
          return vel_in[(own_v ? vown : (int64_t)nb * kCells + ((nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6))) + c * vcs];
        };
        const uint32_t sE = (mask >> 12) & 1u, sW = (mask >> 14) & 1u, sN = (mask >> 10) & 1u;
        const uint32_t sS = (mask >> 16) & 1u, sT = (mask >> 4) & 1u, sB = (mask >> 22) & 1u;
        const R h = R(0.5);
        const R g11 = h * (nbv(1, 0, 0, 0, sE) - nbv(-1, 0, 0, 0, sW));
        const R g12 = h * (nbv(0, 1, 0, 0, sN) - nbv(0, -1, 0, 0, sS));
        const R g13 = h * (nbv(0, 0, 1, 0, sT) - nbv(0, 0, -1, 0, sB));
        const R g21 = h * (nbv(1, 0, 0, 1, sE) - nbv(-1, 0, 0, 1, sW));
        const R g22 = h * (nbv(0, 1, 0, 1, sN) - nbv(0, -1, 0, 1, sS));
        const R g23 = h * (nbv(0, 0, 1, 1, sT) - nbv(0, 0, -1, 1, sB));
        const R g31 = h * (nbv(1, 0, 0, 2, sE) - nbv(-1, 0, 0, 2, sW));
        const R g32 = h * (nbv(0, 1, 0, 2, sN) - nbv(0, -1, 0, 2, sS));
        const R g33 = h * (nbv(0, 0, 1, 2, sT) - nbv(0, 0, -1, 2, sB));
        nu_eddy = wale_nu<R>(g11, g12, g13, g21, g22, g23, g31, g32, g33, cp.c_wale);
        if (flags & CF_SGS_DYNAMIC) {
          // Germano-Lilly (kernel_cumulant.jl:553-565): the face neighbours' previous-step
          // velocities, this cell's current one for missing, ghost or solid neighbours
          // (kernel_dynamic_sgs.jl:57-103)
          R c[3] = {ux, uy, uz}, n[6][3];
          auto nbd = [&](int dx, int dy, int dz, uint32_t solid, R (&o)[3]) {
            const int nx = x + dx, ny = y + dy, nz = z + dz;
            const int nb = s_nbr[nbr_dir(nx >> 3, ny >> 3, nz >> 3)];
            if (nb < 0 || nb >= n_real || solid) { o[0] = ux; o[1] = uy; o[2] = uz; return; }
            const int64_t v = (int64_t)nb * kCells + ((nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6));
            o[0] = vel_in[v]; o[1] = vel_in[v + vcs]; o[2] = vel_in[v + 2 * vcs];
          };
          nbd(1, 0, 0, sE, n[0]); nbd(-1, 0, 0, sW, n[1]); nbd(0, 1, 0, sN, n[2]);
          nbd(0, -1, 0, sS, n[3]); nbd(0, 0, 1, sT, n[4]); nbd(0, 0, -1, sB, n[5]);
          const R S12 = h * (g12 + g21), S13 = h * (g13 + g31), S23 = h * (g23 + g32);
          const R cd = dynamic_cs2<R>(c, n, g11, g22, g33, S12, S13, S23);
          const R s_sq = R(2) * (g11 * g11 + g22 * g22 + g33 * g33) + R(4) * (S12 * S12 + S13 * S13 + S23 * S23);
          const R s_mag = sqrt(s_sq > R(1e-30) ? s_sq : R(1e-30));
          const R nd = cd * s_mag * R(cp.amr_sgs_scale);
          nu_dyn = nd < R(0.1) ? nd : R(0.1);
        }
      }
      R omega1;
      if (flags & (CF_SGS_PI | CF_SGS_DYNAMIC)) {
        // variable nu_sgs (kernel_cumulant.jl:551-586): max(WALE, model stress, floor)
        R stress = nu_dyn;
        if (flags & CF_SGS_PI) {
          R pv[6];
#pragma unroll
          for (int m = 0; m < 6; ++m) pv[m] = pi_neq[vown + m * vcs];
          stress = pi_stress_nu<R>(pv, rho, cp);
        }
        R nu = nu_eddy * R(cp.amr_sgs_scale);
        nu = fmax(fmax(nu, stress), R(cp.nu_sgs_floor) * R(cp.amr_sgs_scale));
        omega1 = omega1_of_nu<R>(nu, cp);
      } else {
        omega1 = omega1_from<R>(nu_eddy, cp);
      }
      cumulant_collide<R>(A, rho, uxe, uye, uze, omega1, cp);

      // ---- Guo forcing + store (kernel_cumulant.jl:889-908) ----
      const bool forced = Fx != R(0) || Fy != R(0) || Fz != R(0);
      const R gpre = R(1) - R(0.5) * omega1;
      if (forced) {
#pragma unroll
        for (int k = 0; k < kQ27; ++k) {
          const R cxf = R(q27_cx(k)), cyf = R(q27_cy(k)), czf = R(q27_cz(k));
          const R cu = cxf * uxe + cyf * uye + czf * uze;
          const R ft = R(q27_w(k)) * R(3) *
                       ((cxf - ux + R(3) * cu * cxf) * Fx + (cyf - uy + R(3) * cu * cyf) * Fy + (czf - uz + R(3) * cu * czf) * Fz);
          A[k] = vfma(gpre, ft, A[k]);
        }
      }
      if ((flags & CF_GRAD_WALL) && (mask & ~(1u << 13)) != 0u) {
        // a fluid cell with a link into a solid: the Grad-reconstruction wall overwrites its
        // post-collision populations and velocity (grad_wall_kernel.jl:42-144, timestep.jl:1738)
        grad_wall<R>(A, rho, R(1) / R(cp.tau), R(cp.grad_pineq_scale));
        vel_out[vown] = R(0); vel_out[vown + vcs] = R(0); vel_out[vown + 2 * vcs] = R(0);
        ux = R(0); uy = R(0); uz = R(0);
      }
      if (flags & CF_SGS_PI) {
        // Pi_neq refresh of the post-collision populations against the stored macros
        // (refresh_pi_neq!, kernel_pi_neq.jl:39-180, fused into the store)
        const bool skip = !isfinite(rho) || rho < R(0.01) || rho > R(10) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz);
        R pv[6];
        pi_neq_of<R>(A, rho, ux, uy, uz, comp, skip, pv);
#pragma unroll
        for (int m = 0; m < 6; ++m) pi_neq[vown + m * vcs] = pv[m];
      }
      uint32_t hsr = 0u;
      if constexpr (sizeof(S) == 2) {
        if (!a.round_nearest) {
          const uint32_t st = __float_as_uint(float(uxe)) * 0x2545F491u + __float_as_uint(float(uye)) +
                              __float_as_uint(float(uze) + float(rho));
          hsr = sr_hash(gx - 1, gy - 1, gz - 1, st);
        }
      }
#pragma unroll
      for (int k = 0; k < kQ27; ++k) {
        S v;
        if constexpr (sizeof(S) == 2) {
          if (a.round_nearest) v = Codec<S>::enc(A[k], R(q27_w(k)), R(1.0 / q27_w(k)));
          else v = enc_rs<S>(fmaf(float(A[k]), float(1.0 / q27_w(k)), -1.0f), hsr * sr_mult(k));
        } else {
          v = Codec<S>::enc(A[k], R(q27_w(k)), R(1.0 / q27_w(k)));
        }
        if (store_post) fpost[own + k * kst] = v;
        fout[own + k * kst] = v;
      }
    }
  }

  if ((flags & CF_COLLECT) && a.force_part) {
    // deterministic FP64 reduction: warp tree, then the four warps in order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mx += __shfl_down_sync(0xffffffffu, mx, o);
      my += __shfl_down_sync(0xffffffffu, my, o);
      mz += __shfl_down_sync(0xffffffffu, mz, o);
    }
    if ((tid & 31) == 0) { s_mom[tid >> 5][0] = mx; s_mom[tid >> 5][1] = my; s_mom[tid >> 5][2] = mz; }
    __syncthreads();
    if (tid < 3) a.force_part[(int64_t)blockIdx.x * 3 + tid] = ((s_mom[0][tid] + s_mom[1][tid]) + s_mom[2][tid]) + s_mom[3][tid];
    if (a.force_out) {
      // the CTA that finishes last sums every CTA's partial in a fixed order, so the total does
      // not depend on which CTA that is: the order of the 256-lane strided sum and tree of the
      // pool's per-member reduction (k_reduce3_segments), each thread carrying lanes t and
      // t + 128, so that a case gets the same bits alone and in a pool
      __shared__ uint32_t s_last;
      __shared__ double s_red[3][128];
      __threadfence();
      __syncthreads();
      if (tid == 0) s_last = atomicAdd(a.force_ticket, 1u) == gridDim.x - 1 ? 1u : 0u;
      __syncthreads();
      if (s_last) {
        double r0 = 0.0, r1 = 0.0, r2 = 0.0, q0 = 0.0, q1 = 0.0, q2 = 0.0;
        for (int64_t i = tid; i < (int64_t)gridDim.x; i += 256) {
          r0 += __ldcg(a.force_part + 3 * i); r1 += __ldcg(a.force_part + 3 * i + 1); r2 += __ldcg(a.force_part + 3 * i + 2);
        }
        for (int64_t i = tid + 128; i < (int64_t)gridDim.x; i += 256) {
          q0 += __ldcg(a.force_part + 3 * i); q1 += __ldcg(a.force_part + 3 * i + 1); q2 += __ldcg(a.force_part + 3 * i + 2);
        }
        s_red[0][tid] = r0 + q0; s_red[1][tid] = r1 + q1; s_red[2][tid] = r2 + q2;
        __syncthreads();
        for (int w = 64; w > 0; w >>= 1) {
          if (tid < w) { s_red[0][tid] += s_red[0][tid + w]; s_red[1][tid] += s_red[1][tid + w]; s_red[2][tid] += s_red[2][tid + w]; }
          __syncthreads();
        }
        if (tid < 3) a.force_out[tid] = s_red[tid][0];
        if (tid == 0) *a.force_ticket = 0u;
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------
// ghost fill by copy list: for the default face conditions every ghost value is either a stored
// word of a real cell (zero-gradient outlet: the cell's own direction k; mirrors and walls: the
// mirrored or opposite direction, which has the same lattice weight, so the stored word itself),
// the inlet equilibrium (kernel_cumulant.jl:235-239 without noise) or the lattice weight. Entry
// (dst, code): code < 2^31 is the source element; 0x80000000 | k the inlet value of direction k;
// 0xC0000000 | k the weight of direction k.
// ------------------------------------------------------------------------------------------------
// Four entries per thread (a stride of the grid apart, so that a warp's accesses stay
// contiguous), their loads issued before any store. RAW: every code is a source element (the
// copies of a block pool, whose element indices use all 32 bits).
template <class S, class R, bool RAW>
__global__ void __launch_bounds__(256) k_fill_copy(const StepArgs a, const uint2* __restrict__ entries, int64_t n) {
  constexpr int E = 4;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t e0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  S* __restrict__ f = const_cast<S*>(static_cast<const S*>(a.f_in));
  uint2 en[E];
  S v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int64_t e = e0 + j * stride;
    en[j] = e < n ? entries[e] : make_uint2(0xFFFFFFFFu, 0x80000000u);
  }
#pragma unroll
  for (int j = 0; j < E; ++j)
    if (en[j].x != 0xFFFFFFFFu && (RAW || !(en[j].y & 0x80000000u))) v[j] = f[en[j].y];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    if (en[j].x == 0xFFFFFFFFu) continue;
    if (!RAW && (en[j].y & 0x80000000u)) {
      const int k = (int)(en[j].y & 31u);
      const R w = R(q27_w(k));
      R val = w;
      if (!(en[j].y & 0x40000000u)) {
        const CaseParams& cp = a.p0;
        val = feq_k<R>(k, R(1), R(cp.u_inlet), R(0), R(0), (cp.flags & CF_COMPRESSIBLE) != 0);
      }
      v[j] = Codec<S>::enc(val, w, R(1) / w);
    }
    f[en[j].x] = v[j];
  }
}

// per work entry of the x-pair kernel: its block's neighbour row, coordinates + case, index
__global__ void k_fast_records(const int32_t* __restrict__ work, int n, const int32_t* __restrict__ nbr,
                               const int4* __restrict__ binfo, int32_t* __restrict__ rec) {
  const int f = blockIdx.x, l = threadIdx.x;
  if (f >= n || l >= 32) return;
  const int32_t b = work[f];
  int32_t v = b;
  if (l < 27) v = nbr[(int64_t)b * 27 + l];
  else if (l < 31) { const int4 bi = binfo[b]; v = l == 27 ? bi.x : l == 28 ? bi.y : l == 29 ? bi.z : bi.w; }
  rec[(int64_t)f * 32 + l] = v;
}

cudaError_t build_fast_records(const int32_t* work, int n, const int32_t* nbr, const int4* binfo, int32_t* rec,
                               cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_fast_records<<<(unsigned)n, 32, 0, st>>>(work, n, nbr, binfo, rec);
  return cudaGetLastError();
}

template <class S, class R>
cudaError_t launch_fill_copy(const StepArgs& a, const uint2* entries, int64_t n, cudaStream_t st, bool raw) {
  if (n <= 0) return cudaSuccess;
  if (raw) k_fill_copy<S, R, true><<<(unsigned)((n + 1023) / 1024), 256, 0, st>>>(a, entries, n);
  else k_fill_copy<S, R, false><<<(unsigned)((n + 1023) / 1024), 256, 0, st>>>(a, entries, n);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------------
// ------------------------------------------------------------------------------------------------
// block AMR: restriction of a child level onto its parent (restrict_child_state_to_parent_kernel!,
// amr_coupling.jl:1900-3242, default flags): every parent cell whose 8 children exist takes the
// average of its fluid children, f = feq + ratio (avg - feq), two moment-correction passes
// (solve_shell_moment4, :130-176) and the shell macros. One thread per parent cell of a block
// that has children; the parent's populations stay in registers (the reference keeps Float32).
// ------------------------------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ bool shell_solve4(R m00, R m01, R m02, R m03, R m11, R m12, R m13, R m22, R m23, R m33,
                                             R r0, R r1, R r2, R r3, R& x0, R& x1, R& x2, R& x3) {
  const R eps = R(1e-12);
  R a00 = m00 + eps, a01 = m01, a02 = m02, a03 = m03, b0 = r0;
  R a10 = m01, a11 = m11 + eps, a12 = m12, a13 = m13, b1 = r1;
  R a20 = m02, a21 = m12, a22 = m22 + eps, a23 = m23, b2 = r2;
  R a30 = m03, a31 = m13, a32 = m23, a33 = m33 + eps, b3 = r3;
  const bool ok0 = fabs(a00) > eps;
  const R inv0 = ok0 ? R(1) / a00 : R(0);
  const R f10 = a10 * inv0, f20 = a20 * inv0, f30 = a30 * inv0;
  a11 -= f10 * a01; a12 -= f10 * a02; a13 -= f10 * a03; b1 -= f10 * b0;
  a21 -= f20 * a01; a22 -= f20 * a02; a23 -= f20 * a03; b2 -= f20 * b0;
  a31 -= f30 * a01; a32 -= f30 * a02; a33 -= f30 * a03; b3 -= f30 * b0;
  const bool ok1 = fabs(a11) > eps;
  const R inv1 = ok1 ? R(1) / a11 : R(0);
  const R f21 = a21 * inv1, f31 = a31 * inv1;
  a22 -= f21 * a12; a23 -= f21 * a13; b2 -= f21 * b1;
  a32 -= f31 * a12; a33 -= f31 * a13; b3 -= f31 * b1;
  const bool ok2 = fabs(a22) > eps;
  const R inv2 = ok2 ? R(1) / a22 : R(0);
  const R f32 = a32 * inv2;
  a33 -= f32 * a23; b3 -= f32 * b2;
  const bool ok3 = fabs(a33) > eps;
  const R inv3 = ok3 ? R(1) / a33 : R(0);
  x3 = b3 * inv3;
  x2 = (b2 - a23 * x3) * inv2;
  x1 = (b1 - a12 * x2 - a13 * x3) * inv1;
  x0 = (b0 - a01 * x1 - a02 * x2 - a03 * x3) * inv0;
  return ok0 && ok1 && ok2 && ok3;
}

template <class S, class R>
__global__ void __launch_bounds__(128) k_restrict(const RestrictArgs r) {
  const int pb = r.covered[blockIdx.x >> 2];
  const int cell = ((blockIdx.x & 3) << 7) | threadIdx.x;
  const int lx = (cell & 7) + 1, ly = ((cell >> 3) & 7) + 1, lz = (cell >> 6) + 1;
  const int4 bi = r.pbinfo[pb];
  const int cbx0 = 2 * bi.x - 1, cby0 = 2 * bi.y - 1, cbz0 = 2 * bi.z - 1;
  int32_t cblk[8], ccell[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int sx = i >> 2, sy = (i >> 1) & 1, sz = i & 1;  // sx outer, sz inner (the reference's order)
    const int fx = 2 * (lx - 1) + 1 + sx, fy = 2 * (ly - 1) + 1 + sy, fz = 2 * (lz - 1) + 1 + sz;
    const int cbx = cbx0 + (fx - 1) / kBS, cby = cby0 + (fy - 1) / kBS, cbz = cbz0 + (fz - 1) / kBS;
    if (cbx < 1 || cby < 1 || cbz < 1 || cbx > r.cdx || cby > r.cdy || cbz > r.cdz) return;
    const int32_t cb = r.cptr[(cbx - 1) + (int64_t)r.cdx * ((cby - 1) + (int64_t)r.cdy * (cbz - 1))];
    if (cb == 0) return;
    cblk[i] = cb - 1;
    ccell[i] = ((fx - 1) % kBS) | (((fy - 1) % kBS) << 3) | (((fz - 1) % kBS) << 6);
  }
  const S* cf = static_cast<const S*>(r.cf);
  R avg[kQ27];
#pragma unroll
  for (int k = 0; k < kQ27; ++k) avg[k] = R(0);
  int fluid = 0;
#pragma unroll 1
  for (int i = 0; i < 8; ++i) {
    const int cb = cblk[i];
    if ((r.cbflags[cb] & BF_NEAR_SOLID) && ((r.ccmask[(int64_t)r.cmslot[cb] * kCells + ccell[i]] >> 13) & 1u)) continue;
    ++fluid;
    const int64_t base = (int64_t)cb * (27 * kCells) + ccell[i];
#pragma unroll
    for (int k = 0; k < kQ27; ++k) avg[k] += Codec<S>::dec(cf[base + k * kCells], R(q27_w(k)), R(1.0 / q27_w(k)));
  }
  if (fluid == 0) return;
  const R inv_children = R(1) / R(fluid);
  R rho_raw = R(0), jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R favg = avg[k] * inv_children;
    avg[k] = favg;
    rho_raw += favg;
    jx += favg * R(q27_cx(k));
    jy += favg * R(q27_cy(k));
    jz += favg * R(q27_cz(k));
  }
  const R rho_p = fmax(rho_raw, R(0.01));
  const R inv_rho = R(1) / rho_p;
  const R ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  const bool comp = r.comp != 0;
  const R ratio = R(r.ratio);
  S* pf = static_cast<S*>(r.pf);
  const int64_t pbase = (int64_t)pb * (27 * kCells) + cell;
  R fp[kQ27];
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R feq = feq_c<R>(rho_p, ux, uy, uz, R(q27_w(k)), R(q27_cx(k)), R(q27_cy(k)), R(q27_cz(k)), comp);
    const R prior = Codec<S>::dec(pf[pbase + k * kCells], R(q27_w(k)), R(1.0 / q27_w(k)));
    const R fr = feq + ratio * (avg[k] - feq);
    fp[k] = fmax(R(1) * fr + R(0) * prior, R(1e-10));
  }
  R m00 = 0, m01 = 0, m02 = 0, m03 = 0, m11 = 0, m12 = 0, m13 = 0, m22 = 0, m23 = 0, m33 = 0;
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R cx = R(q27_cx(k)), cy = R(q27_cy(k)), cz = R(q27_cz(k)), w = R(q27_w(k));
    m00 += w; m01 += w * cx; m02 += w * cy; m03 += w * cz;
    m11 += w * cx * cx; m12 += w * cx * cy; m13 += w * cx * cz;
    m22 += w * cy * cy; m23 += w * cy * cz; m33 += w * cz * cz;
  }
  const R inv_cs2 = R(1) / fmax(R(1.0 / 3.0), R(1e-6));
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    R rr = R(0), rx = R(0), ry = R(0), rz = R(0);
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      rr += fp[k]; rx += fp[k] * R(q27_cx(k)); ry += fp[k] * R(q27_cy(k)); rz += fp[k] * R(q27_cz(k));
    }
    const R dr = rho_p - rr, dx = jx - rx, dy = jy - ry, dz = jz - rz;
    if (fabs(dr) > R(1e-12) || fabs(dx) > R(1e-12) || fabs(dy) > R(1e-12) || fabs(dz) > R(1e-12)) {
      R c0, c1, c2, c3;
      const bool ok = shell_solve4<R>(m00, m01, m02, m03, m11, m12, m13, m22, m23, m33, dr, dx, dy, dz, c0, c1, c2, c3);
#pragma unroll
      for (int k = 0; k < kQ27; ++k) {
        const R cx = R(q27_cx(k)), cy = R(q27_cy(k)), cz = R(q27_cz(k)), w = R(q27_w(k));
        const R delta = ok ? w * (c0 + c1 * cx + c2 * cy + c3 * cz) : w * (dr + inv_cs2 * (cx * dx + cy * dy + cz * dz));
        fp[k] = fmax(fp[k] + delta, R(1e-10));
      }
    }
  }
  R rs = R(0), sx = R(0), sy = R(0), sz = R(0);
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    rs += fp[k]; sx += fp[k] * R(q27_cx(k)); sy += fp[k] * R(q27_cy(k)); sz += fp[k] * R(q27_cz(k));
    pf[pbase + k * kCells] = Codec<S>::enc(fp[k], R(q27_w(k)), R(1.0 / q27_w(k)));
  }
  const R rho_s = fmax(rs, R(0.01));
  const R inv_s = R(1) / rho_s;
  R* prho = static_cast<R*>(r.prho);
  R* pvel = static_cast<R*>(r.pvel);
  const int64_t pc = (int64_t)pb * kCells + cell, pn = (int64_t)r.pnb * kCells;
  prho[pc] = rho_s;
  pvel[pc] = sx * inv_s;
  pvel[pc + pn] = sy * inv_s;
  pvel[pc + 2 * pn] = sz * inv_s;
}

template <class S, class R>
cudaError_t launch_restrict(const RestrictArgs& r, cudaStream_t st) {
  if (r.n_covered <= 0) return cudaSuccess;
  k_restrict<S, R><<<(unsigned)r.n_covered * 4, 128, 0, st>>>(r);
  return cudaGetLastError();
}

template <class S, class R>
cudaError_t launch_fill_ghosts(const StepArgs& a, const uint2* entries, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (a.par.ptr) {
    if (a.dense) k_fill_ghosts<S, R, true, true><<<grid, 256, 0, st>>>(a, entries, n);
    else k_fill_ghosts<S, R, false, true><<<grid, 256, 0, st>>>(a, entries, n);
  } else {
    if (a.dense) k_fill_ghosts<S, R, true, false><<<grid, 256, 0, st>>>(a, entries, n);
    else k_fill_ghosts<S, R, false, false><<<grid, 256, 0, st>>>(a, entries, n);
  }
  return cudaGetLastError();
}

template <class S, class R>
cudaError_t launch_fast(const StepArgs& a, const int32_t* work, int n_work, cudaStream_t st) {
  if (n_work <= 0) return cudaSuccess;
  // element count of the buffer (real + ghost blocks) decides the index width
  const bool idx32 = (uint64_t)a.n_total_blocks * 27u * kCells < (1ull << 32);
  if constexpr (sizeof(R) == 8) {
    if (idx32) k_cumulant_fast<S, double, uint32_t><<<(unsigned)n_work * 4u, 128, 0, st>>>(a, work);
    else k_cumulant_fast<S, double, int64_t><<<(unsigned)n_work * 4u, 128, 0, st>>>(a, work);
  } else if constexpr (OAL_FAST_CELLS == 1) {
    if (idx32) k_cumulant_fast<S, float, uint32_t><<<(unsigned)n_work * 4u, 128, 0, st>>>(a, work);
    else k_cumulant_fast<S, float, int64_t><<<(unsigned)n_work * 4u, 128, 0, st>>>(a, work);
  } else if constexpr (OAL_FAST_CELLS == 3) {
    if (idx32) k_cumulant_fast<S, F2, uint32_t><<<(unsigned)n_work * 2u, 128, 0, st>>>(a, work);
    else k_cumulant_fast<S, F2, int64_t><<<(unsigned)n_work * 2u, 128, 0, st>>>(a, work);
  } else {
    // x pairs; word indices (half the element count) decide the index width
    const unsigned units = (unsigned)n_work * (256u / OAL_PAIRS_THREADS);
    const bool pos = (a.flags_any & CF_LIMITER_POSITIVITY) != 0, gen = (a.flags_any & CF_GENERAL_RATES) != 0;
    auto go = [&](auto plain, auto pers) -> cudaError_t {
      if (!a.persistent) {
        plain<<<units, OAL_PAIRS_THREADS, 0, st>>>(a, work);
        return cudaGetLastError();
      }
      // persistent: as many CTAs as stay resident on the device at once, each walking the units
      static thread_local std::vector<std::pair<const void*, int>> resident;
      int n = 0;
      for (const auto& r : resident)
        if (r.first == reinterpret_cast<const void*>(pers)) n = r.second;
      if (n == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pers, OAL_PAIRS_THREADS, 0);
        if (e != cudaSuccess) return e;
        n = std::max(1, sms * per_sm);
        resident.emplace_back(reinterpret_cast<const void*>(pers), n);
      }
      StepArgs b = a;
      b.pairs_units = (int32_t)units;
      pers<<<std::min(units, (unsigned)n), OAL_PAIRS_THREADS, 0, st>>>(b, work);
      return cudaGetLastError();
    };
    if (pos || gen) {
      if (idx32) return go(k_cumulant_pairs<S, uint32_t, true, true, false>, k_cumulant_pairs<S, uint32_t, true, true, true>);
      return go(k_cumulant_pairs<S, int64_t, true, true, false>, k_cumulant_pairs<S, int64_t, true, true, true>);
    }
    if (idx32) return go(k_cumulant_pairs<S, uint32_t, false, false, false>, k_cumulant_pairs<S, uint32_t, false, false, true>);
    return go(k_cumulant_pairs<S, int64_t, false, false, false>, k_cumulant_pairs<S, int64_t, false, false, true>);
  }
  return cudaGetLastError();
}

template <class S, class R>
cudaError_t launch_general(const StepArgs& a, const int32_t* work, int n_work, cudaStream_t st) {
  if (n_work <= 0) return cudaSuccess;
  if (a.dense) k_cumulant_gen<S, R, true><<<(unsigned)n_work * 4u, 128, 0, st>>>(a, work);
  else k_cumulant_gen<S, R, false><<<(unsigned)n_work * 4u, 128, 0, st>>>(a, work);
  return cudaGetLastError();
}

#define OAL_INST(S, R)                                                                               \
  template cudaError_t launch_fill_ghosts<S, R>(const StepArgs&, const uint2*, int64_t, cudaStream_t); \
  template cudaError_t launch_fill_copy<S, R>(const StepArgs&, const uint2*, int64_t, cudaStream_t, bool); \
  template cudaError_t launch_restrict<S, R>(const RestrictArgs&, cudaStream_t);                       \
  template cudaError_t launch_parent_nodes<S, R>(const ParentView&, const int32_t*, int32_t, void*, int32_t,  \
                                                 cudaStream_t);                                            \
  template cudaError_t launch_fast<S, R>(const StepArgs&, const int32_t*, int, cudaStream_t);         \
  template cudaError_t launch_general<S, R>(const StepArgs&, const int32_t*, int, cudaStream_t);
OAL_INST(float, float)
OAL_INST(__half, float)
OAL_INST(__nv_bfloat16, float)
OAL_INST(double, double)
#undef OAL_INST
template cudaError_t launch_parent_positions<float>(const ParentView&, const int4*, int32_t, void*, cudaStream_t);
template cudaError_t launch_parent_positions<double>(const ParentView&, const int4*, int32_t, void*, cudaStream_t);

}  // namespace oal
