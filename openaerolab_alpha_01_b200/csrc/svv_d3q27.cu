// svv_d3q27.cu — spectral vanishing viscosity of the reference's D3Q27 levels
// (apply_svv_d3q19_postcollision!, src/collision/kernel_svv_yz_d3q39.jl:426-458, with
// apply_svv_d3q19_inline!, :301-375, and the tap helpers get_pop_neighbor_x / _yz, :225-250 and
// :78-116), launched after the step kernels (timestep.jl:1576-1611).
//
// For every fluid cell and direction k, the post-collision population f_k is filtered by the
// 5-point bi-Laplacian of the step's input populations along x (eps_x) and along y and z
// (eps_yz), the centre tap being f_k itself:
//   f_k' = f_k - eps_x (t-2 - 4 t-1 + 6 f_k - 4 t+1 + t+2)_x - eps_yz (...)_y - eps_yz (...)_z
// A tap in a solid cell or past a missing neighbour block reads the cell's own input population
// (a zero-flux wall for the operator). The 4-moment correction f_k' -= w_k (drho + c_k.dj / cs2)
// then restores the cell's mass and momentum, and every population is floored at 1e-12.
//
// One thread per cell, 256 per CTA (half a block; 128 in FP64). A population's address is linear in its
// direction in both layouts (block-major: b 27*512 + k 512 + cell; dense: cell + k PX PY PZ), so a
// thread resolves its twelve taps once — the neighbour block, the solid masks and the fall-back
// to its own slot — into twelve direction-0 offsets, and each direction then costs one load per
// tap (the block's rows, mostly L1 hits) and the arithmetic. The filtered populations wait in
// shared memory (the thread's own column) for the correction. HBM traffic per fluid cell: the
// 27 input populations once, the 27 output populations read and written.
#include "svv_d3q27.h"

namespace oal {

namespace {

// one thread per cell: 256 per CTA (two per block), 128 for FP64 (the filtered populations of a
// CTA in shared memory stay within the 48 KB of static shared memory)
template <class R> constexpr int svv_threads() { return sizeof(R) == 8 ? 128 : 256; }

struct SvvArgs {
  PopIndex pi;
  const int32_t* __restrict__ nbr;    // [nb*27] 0-based, -1 = no neighbour
  int32_t n_real;
  const int32_t* __restrict__ mslot;  // per-block mask slot or -1
  const uint32_t* __restrict__ cmask; // bit 13: the cell itself is solid
  float eps_x, eps_yz;
};

__device__ __forceinline__ bool svv_solid(const SvvArgs& a, int64_t b, int cell) {
  if (!a.mslot) return false;
  const int32_t s = a.mslot[b];
  return s >= 0 && ((a.cmask[(int64_t)s * kCells + cell] >> 13) & 1u);
}

// the direction-0 offset of the input population at (x, y, z) + d along one axis, or `own`
template <class IDX>
__device__ __forceinline__ IDX svv_tap_offset(const SvvArgs& a, int b, int x, int y, int z, int dx, int dy, int dz,
                                              IDX own) {
  const int nx = x + dx, ny = y + dy, nz = z + dz;
  const int ox = nx < 0 ? -1 : (nx >= kBS ? 1 : 0), oy = ny < 0 ? -1 : (ny >= kBS ? 1 : 0),
            oz = nz < 0 ? -1 : (nz >= kBS ? 1 : 0);
  int32_t bb = b;
  if (ox | oy | oz) {
    bb = a.nbr[(int64_t)b * kQ27 + nbr_dir(ox, oy, oz)];
    if (bb < 0 || bb >= a.n_real) return own;
  }
  const int c = (nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6);
  if (svv_solid(a, bb, c)) return own;
  return (IDX)a.pi(bb, c, 0);
}

template <class S, class R, class IDX>
__global__ void __launch_bounds__(svv_threads<R>(), 3) k_svv(const SvvArgs a, const S* __restrict__ fin, S* __restrict__ fout,
                                                             S* __restrict__ fpost2) {
  constexpr int kT = svv_threads<R>(), kPer = kCells / kT;
  const int b = blockIdx.x / kPer;
  const int cell = (blockIdx.x % kPer) * kT + threadIdx.x;
  if (svv_solid(a, b, cell)) return;
  const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
  const IDX own = (IDX)a.pi(b, cell, 0);
  const IDX kst = (IDX)a.pi.kst;
  const bool fx = a.eps_x > 0.0f, fyz = a.eps_yz > 0.0f;
  // taps: x-2, x-1, x+1, x+2, then y, then z
  IDX t[12];
#pragma unroll
  for (int j = 0; j < 12; ++j) {
    const int axis = j >> 2, s = (j & 3) < 2 ? (j & 3) - 2 : (j & 3) - 1;
    const bool used = axis == 0 ? fx : fyz;
    t[j] = used ? svv_tap_offset<IDX>(a, b, x, y, z, axis == 0 ? s : 0, axis == 1 ? s : 0, axis == 2 ? s : 0, own)
                : own;
  }
  const R ex = R(a.eps_x), eyz = R(a.eps_yz);
  __shared__ R s_fl[kQ27][kT];  // the filtered populations until the correction
  R d_rho = R(0), d_jx = R(0), d_jy = R(0), d_jz = R(0);
#pragma unroll 3
  for (int k = 0; k < kQ27; ++k) {
    const R w = R(q27_w(k)), inv_w = R(1.0 / q27_w(k));
    const S* fk = fin + (IDX)k * kst;
    auto tap = [&](int j) { return Codec<S>::dec(fk[t[j]], w, inv_w); };
    const R fc = Codec<S>::dec(fout[own + (IDX)k * kst], w, inv_w);
    R bilap = R(0);
    if (fx) bilap += ex * ((((tap(0) - R(4) * tap(1)) + R(6) * fc) - R(4) * tap(2)) + tap(3));
    if (fyz) {
      bilap += eyz * ((((tap(4) - R(4) * tap(5)) + R(6) * fc) - R(4) * tap(6)) + tap(7));
      bilap += eyz * ((((tap(8) - R(4) * tap(9)) + R(6) * fc) - R(4) * tap(10)) + tap(11));
    }
    const R ff = fc - bilap;
    const R diff = ff - fc;
    d_rho += diff;
    d_jx += diff * R(q27_cx(k));
    d_jy += diff * R(q27_cy(k));
    d_jz += diff * R(q27_cz(k));
    s_fl[k][threadIdx.x] = ff;
  }
  const R inv_cs2 = R(1) / R(1.0 / 3.0);  // CS2_LATTICE
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R w = R(q27_w(k)), inv_w = R(1.0 / q27_w(k));
    const R cu = R(q27_cx(k)) * d_jx + R(q27_cy(k)) * d_jy + R(q27_cz(k)) * d_jz;
    R v = s_fl[k][threadIdx.x] - w * (d_rho + inv_cs2 * cu);
    v = v < R(1e-12f) ? R(1e-12f) : v;  // NaN passes
    const S word = Codec<S>::enc(v, w, inv_w);
    fout[own + (IDX)k * kst] = word;
    if (fpost2) fpost2[own + (IDX)k * kst] = word;
  }
}

// ---- two x-adjacent cells per thread (block layout, FP32/FP16/BF16 storage) -------------------
// The same filter with one 32- or 64-bit load per tap pair: the y and z taps of cells (x, x+1)
// are adjacent words, and the x taps of the pair come from the pairs (x-2, x-1), (x, x+1) and
// (x+2, x+3). Each lane keeps its own fall-back flags (a solid target or a missing block selects
// the lane's own input population), so every lane computes exactly what the one-cell kernel does.
template <class S> struct PairIO;
template <> struct PairIO<float> {
  static __device__ __forceinline__ float2 load(const float* p, float, float) { return *reinterpret_cast<const float2*>(p); }
  static __device__ __forceinline__ void store(float* p, float a, float b, float, float) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
  }
};
template <> struct PairIO<__half> {
  static __device__ __forceinline__ float2 load(const __half* p, float w, float) {
    const float2 h = __half22float2(*reinterpret_cast<const __half2*>(p));
    return make_float2(fmaf(w, h.x, w), fmaf(w, h.y, w));
  }
  static __device__ __forceinline__ void store(__half* p, float a, float b, float, float inv_w) {
    *reinterpret_cast<__half2*>(p) = __floats2half2_rn(fmaf(a, inv_w, -1.0f), fmaf(b, inv_w, -1.0f));
  }
};
template <> struct PairIO<__nv_bfloat16> {
  static __device__ __forceinline__ float2 load(const __nv_bfloat16* p, float w, float) {
    const float2 h = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
    return make_float2(fmaf(w, h.x, w), fmaf(w, h.y, w));
  }
  static __device__ __forceinline__ void store(__nv_bfloat16* p, float a, float b, float, float inv_w) {
    *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(fmaf(a, inv_w, -1.0f), fmaf(b, inv_w, -1.0f));
  }
};

// the direction-0 offset of the pair starting at (x, y, z) + d (x + dx even), whether its block
// exists, and per lane whether the target cell is solid
template <class IDX>
__device__ __forceinline__ IDX svv_pair_offset(const SvvArgs& a, int b, int x, int y, int z, int dx, int dy, int dz,
                                               IDX own, bool& s0, bool& s1) {
  const int nx = x + dx, ny = y + dy, nz = z + dz;
  const int ox = nx < 0 ? -1 : (nx >= kBS ? 1 : 0), oy = ny < 0 ? -1 : (ny >= kBS ? 1 : 0),
            oz = nz < 0 ? -1 : (nz >= kBS ? 1 : 0);
  int32_t bb = b;
  if (ox | oy | oz) {
    bb = a.nbr[(int64_t)b * kQ27 + nbr_dir(ox, oy, oz)];
    if (bb < 0 || bb >= a.n_real) { s0 = s1 = true; return own; }
  }
  const int c = (nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6);
  s0 = svv_solid(a, bb, c);
  s1 = svv_solid(a, bb, c + 1);
  return (IDX)a.pi(bb, c, 0);
}

// the filter of the 27 directions of a pair of cells: the filtered values into s_fl, the changes
// of mass and momentum of each lane into acc; PICK: some tap of the pair falls back
template <class S, class IDX, bool PICK>
__device__ __forceinline__ void svv_pairs_filter(const SvvArgs& a, const S* __restrict__ fin, const S* __restrict__ fout,
                                                 IDX own, IDX kst, const IDX (&t)[10], uint32_t fb, bool fx, bool fyz,
                                                 float (*s_fl)[256], int l0, float (&acc)[8]) {
  const float ex = a.eps_x, eyz = a.eps_yz;
  float r0 = 0.0f, x0 = 0.0f, y0 = 0.0f, z0 = 0.0f, r1 = 0.0f, x1 = 0.0f, y1 = 0.0f, z1 = 0.0f;
#pragma unroll 3
  for (int k = 0; k < kQ27; ++k) {
    const float w = float(q27_w(k)), inv_w = float(1.0 / q27_w(k));
    const S* fk = fin + (IDX)k * kst;
    const float2 o = PairIO<S>::load(fk + own, w, inv_w);  // the pair's own input populations
    const float2 fc = PairIO<S>::load(fout + own + (IDX)k * kst, w, inv_w);
    auto pick = [&](int bit, float v, float mine) {
      if constexpr (PICK) return ((fb >> bit) & 1u) ? mine : v;
      else return v;
    };
    float bl0 = 0.0f, bl1 = 0.0f;
    if (fx) {
      const float2 m = PairIO<S>::load(fk + t[0], w, inv_w), p = PairIO<S>::load(fk + t[1], w, inv_w);
      bl0 += ex * ((((pick(0, m.x, o.x) - 4.0f * pick(2, m.y, o.x)) + 6.0f * fc.x) - 4.0f * pick(4, o.y, o.x)) +
                   pick(6, p.x, o.x));
      bl1 += ex * ((((pick(1, m.y, o.y) - 4.0f * pick(3, o.x, o.y)) + 6.0f * fc.y) - 4.0f * pick(5, p.x, o.y)) +
                   pick(7, p.y, o.y));
    }
    if (fyz) {
#pragma unroll
      for (int a2 = 0; a2 < 2; ++a2) {
        const int j0 = 2 + 4 * a2, bit = 8 + 8 * a2;
        const float2 v0 = PairIO<S>::load(fk + t[j0], w, inv_w), v1 = PairIO<S>::load(fk + t[j0 + 1], w, inv_w);
        const float2 v2 = PairIO<S>::load(fk + t[j0 + 2], w, inv_w), v3 = PairIO<S>::load(fk + t[j0 + 3], w, inv_w);
        bl0 += eyz * ((((pick(bit, v0.x, o.x) - 4.0f * pick(bit + 2, v1.x, o.x)) + 6.0f * fc.x) -
                       4.0f * pick(bit + 4, v2.x, o.x)) + pick(bit + 6, v3.x, o.x));
        bl1 += eyz * ((((pick(bit + 1, v0.y, o.y) - 4.0f * pick(bit + 3, v1.y, o.y)) + 6.0f * fc.y) -
                       4.0f * pick(bit + 5, v2.y, o.y)) + pick(bit + 7, v3.y, o.y));
      }
    }
    const float f0 = fc.x - bl0, f1 = fc.y - bl1;
    const float e0 = f0 - fc.x, e1 = f1 - fc.y;
    r0 += e0; x0 += e0 * float(q27_cx(k)); y0 += e0 * float(q27_cy(k)); z0 += e0 * float(q27_cz(k));
    r1 += e1; x1 += e1 * float(q27_cx(k)); y1 += e1 * float(q27_cy(k)); z1 += e1 * float(q27_cz(k));
    s_fl[k][l0] = f0;
    s_fl[k][l0 + 1] = f1;
  }
  acc[0] = r0; acc[1] = x0; acc[2] = y0; acc[3] = z0; acc[4] = r1; acc[5] = x1; acc[6] = y1; acc[7] = z1;
}

template <class S, class IDX>
__global__ void __launch_bounds__(128, 6) k_svv_pairs(const SvvArgs a, const S* __restrict__ fin, S* __restrict__ fout,
                                                      S* __restrict__ fpost2) {
  const int b = blockIdx.x >> 1;
  const int base = (blockIdx.x & 1) << 8;
  const int l0 = threadIdx.x << 1;  // the pair's first cell within the CTA's half block
  const int c0 = base + l0;
  const int x = c0 & 7, y = (c0 >> 3) & 7, z = c0 >> 6;
  const bool d0 = svv_solid(a, b, c0), d1 = svv_solid(a, b, c0 + 1);
  if (d0 && d1) return;
  const IDX own = (IDX)a.pi(b, c0, 0);
  const IDX kst = (IDX)a.pi.kst;
  const bool fx = a.eps_x > 0.0f, fyz = a.eps_yz > 0.0f;
  // pair taps: 0 (x-2, x-1), 1 (x+2, x+3), 2-5 y-2, y-1, y+1, y+2, 6-9 z-2 .. z+2; fb bit 2j + lane:
  // the lane takes its own input population for tap j (x taps: j 0-3 of the lane's x-2 .. x+2)
  IDX t[10];
  uint32_t fb = 0;
  bool m0, m1, p0, p1;
  t[0] = fx ? svv_pair_offset<IDX>(a, b, x, y, z, -2, 0, 0, own, m0, m1) : own;
  t[1] = fx ? svv_pair_offset<IDX>(a, b, x, y, z, 2, 0, 0, own, p0, p1) : own;
  if (fx) {
    // lane 0 (x): x-2, x-1, x+1 (the pair's second cell), x+2; lane 1 (x+1): x-1, x, x+2, x+3
    fb |= (uint32_t)m0 << 0 | (uint32_t)m1 << 2 | (uint32_t)d1 << 4 | (uint32_t)p0 << 6;
    fb |= (uint32_t)m1 << 1 | (uint32_t)d0 << 3 | (uint32_t)p0 << 5 | (uint32_t)p1 << 7;
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int s = (j & 3) < 2 ? (j & 3) - 2 : (j & 3) - 1;
    bool q0 = true, q1 = true;
    t[2 + j] = fyz ? svv_pair_offset<IDX>(a, b, x, y, z, 0, j < 4 ? s : 0, j < 4 ? 0 : s, own, q0, q1) : own;
    fb |= (uint32_t)q0 << (8 + 2 * j) | (uint32_t)q1 << (9 + 2 * j);
  }
  __shared__ float s_fl[kQ27][256];
  float acc[8];
  // the fall-back selects only where a tap of the pair falls back (cells next to a solid or a
  // missing block); elsewhere the loads are used as they are
  if (fb == 0) svv_pairs_filter<S, IDX, false>(a, fin, fout, own, kst, t, fb, fx, fyz, s_fl, l0, acc);
  else svv_pairs_filter<S, IDX, true>(a, fin, fout, own, kst, t, fb, fx, fyz, s_fl, l0, acc);
  const float r0 = acc[0], x0 = acc[1], y0 = acc[2], z0 = acc[3], r1 = acc[4], x1 = acc[5], y1 = acc[6], z1 = acc[7];
  const float inv_cs2 = 1.0f / float(1.0 / 3.0);  // CS2_LATTICE
#pragma unroll 3
  for (int k = 0; k < kQ27; ++k) {
    const float w = float(q27_w(k)), inv_w = float(1.0 / q27_w(k));
    const float cx = float(q27_cx(k)), cy = float(q27_cy(k)), cz = float(q27_cz(k));
    float v0 = s_fl[k][l0] - w * (r0 + inv_cs2 * ((cx * x0 + cy * y0) + cz * z0));
    float v1 = s_fl[k][l0 + 1] - w * (r1 + inv_cs2 * ((cx * x1 + cy * y1) + cz * z1));
    v0 = v0 < 1e-12f ? 1e-12f : v0;  // NaN passes
    v1 = v1 < 1e-12f ? 1e-12f : v1;
    // a solid cell of the pair keeps its stored word
    if (d0 || d1) {
      S* q = fout + own + (IDX)k * kst;
      S* q2 = fpost2 ? fpost2 + own + (IDX)k * kst : nullptr;
      if (!d0) { q[0] = Codec<S>::enc(v0, w, inv_w); if (q2) q2[0] = q[0]; }
      if (!d1) { q[1] = Codec<S>::enc(v1, w, inv_w); if (q2) q2[1] = q[1]; }
    } else {
      PairIO<S>::store(fout + own + (IDX)k * kst, v0, v1, w, inv_w);
      if (fpost2) PairIO<S>::store(fpost2 + own + (IDX)k * kst, v0, v1, w, inv_w);
    }
  }
}

template <class S, class R>
cudaError_t enqueue_t(const SvvArgs& a, const void* fin, void* fout, void* fpost2, int32_t nb, int64_t n_elements,
                      cudaStream_t st) {
  constexpr int kT = svv_threads<R>();
  const unsigned grid = (unsigned)nb * (unsigned)(kCells / kT);
  const S* in = static_cast<const S*>(fin);
  S* out = static_cast<S*>(fout);
  S* post = static_cast<S*>(fpost2);
  if constexpr (sizeof(R) == 4) {
    // pairs of x-adjacent cells are aligned words where the strides are even and the arrays start
    // on a word (every block layout this library allocates; a caller's arrays are checked)
    auto aligned = [](const void* p) { return p == nullptr || ((uintptr_t)p % (2 * sizeof(S))) == 0; };
    if (!a.pi.dense && a.pi.bst % 2 == 0 && a.pi.kst % 2 == 0 && aligned(fin) && aligned(fout) && aligned(fpost2)) {
      if (n_elements < (int64_t(1) << 32))
        k_svv_pairs<S, uint32_t><<<(unsigned)nb * 2u, 128, 0, st>>>(a, in, out, post);
      else
        k_svv_pairs<S, int64_t><<<(unsigned)nb * 2u, 128, 0, st>>>(a, in, out, post);
      return cudaGetLastError();
    }
  }
  if (n_elements < (int64_t(1) << 32))
    k_svv<S, R, uint32_t><<<grid, kT, 0, st>>>(a, in, out, post);
  else
    k_svv<S, R, int64_t><<<grid, kT, 0, st>>>(a, in, out, post);
  return cudaGetLastError();
}

}  // namespace

cudaError_t svv_enqueue(int32_t storage, const void* f_in, void* f_out, const PopIndex& pi, int32_t nb,
                        int64_t n_elements, const int32_t* nbr, int32_t n_real, const int32_t* mslot,
                        const uint32_t* cmask, float eps_x, float eps_yz, cudaStream_t st, void* f_post2) {
  if ((eps_x == 0.0f && eps_yz == 0.0f) || nb <= 0) return cudaSuccess;
  SvvArgs a;
  a.pi = pi; a.nbr = nbr; a.n_real = n_real; a.mslot = cmask ? mslot : nullptr; a.cmask = cmask;
  a.eps_x = eps_x; a.eps_yz = eps_yz;
  switch (storage) {
    case 0: return enqueue_t<float, float>(a, f_in, f_out, f_post2, nb, n_elements, st);
    case 1: return enqueue_t<__half, float>(a, f_in, f_out, f_post2, nb, n_elements, st);
    case 2: return enqueue_t<__nv_bfloat16, float>(a, f_in, f_out, f_post2, nb, n_elements, st);
    case 3: return enqueue_t<double, double>(a, f_in, f_out, f_post2, nb, n_elements, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace oal
