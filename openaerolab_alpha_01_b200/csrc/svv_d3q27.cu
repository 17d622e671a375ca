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
__global__ void __launch_bounds__(svv_threads<R>(), 3) k_svv(const SvvArgs a, const S* __restrict__ fin, S* __restrict__ fout) {
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
    fout[own + (IDX)k * kst] = Codec<S>::enc(v, w, inv_w);
  }
}

template <class S, class R>
cudaError_t enqueue_t(const SvvArgs& a, const void* fin, void* fout, int32_t nb, int64_t n_elements, cudaStream_t st) {
  constexpr int kT = svv_threads<R>();
  const unsigned grid = (unsigned)nb * (unsigned)(kCells / kT);
  if (n_elements < (int64_t(1) << 32))
    k_svv<S, R, uint32_t><<<grid, kT, 0, st>>>(a, static_cast<const S*>(fin), static_cast<S*>(fout));
  else
    k_svv<S, R, int64_t><<<grid, kT, 0, st>>>(a, static_cast<const S*>(fin), static_cast<S*>(fout));
  return cudaGetLastError();
}

}  // namespace

cudaError_t svv_enqueue(int32_t storage, const void* f_in, void* f_out, const PopIndex& pi, int32_t nb,
                        int64_t n_elements, const int32_t* nbr, int32_t n_real, const int32_t* mslot,
                        const uint32_t* cmask, float eps_x, float eps_yz, cudaStream_t st) {
  if ((eps_x == 0.0f && eps_yz == 0.0f) || nb <= 0) return cudaSuccess;
  SvvArgs a;
  a.pi = pi; a.nbr = nbr; a.n_real = n_real; a.mslot = cmask ? mslot : nullptr; a.cmask = cmask;
  a.eps_x = eps_x; a.eps_yz = eps_yz;
  switch (storage) {
    case 0: return enqueue_t<float, float>(a, f_in, f_out, nb, n_elements, st);
    case 1: return enqueue_t<__half, float>(a, f_in, f_out, nb, n_elements, st);
    case 2: return enqueue_t<__nv_bfloat16, float>(a, f_in, f_out, nb, n_elements, st);
    case 3: return enqueue_t<double, double>(a, f_in, f_out, nb, n_elements, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace oal
