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
// One CTA per block, one thread per cell. The taps of a cell reach two cells past its block along
// each axis only, so the CTA stages, per direction, the block and its axial halo (a 12^3 tile of
// which the 8^3 core and six 2-cell slabs are read) in shared memory: the neighbour/solid logic runs
// once per tile cell rather than per (cell, direction, tap), and each input population is read
// from memory about 2.5 times (core + the halo slabs of the six neighbours) instead of 13 times.
// The filtered populations of the cell wait in shared memory for the correction. HBM traffic per
// fluid cell: 27 input populations (plus the halo re-reads, mostly L2 hits) and 27 output
// populations read and written.
#include "svv_d3q27.h"

namespace oal {

namespace {

constexpr int kT = 12;            // tile edge: the block and 2 cells on each side
constexpr int kT3 = kT * kT * kT;
constexpr int kSvvThreads = 512;  // one thread per cell
constexpr uint32_t kNoSrc = 0xffffffffu;

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

template <class S, class R>
__global__ void __launch_bounds__(kSvvThreads) k_svv(const SvvArgs a, const S* __restrict__ fin, S* __restrict__ fout) {
  extern __shared__ __align__(16) unsigned char svv_smem[];
  R* s_fl = reinterpret_cast<R*>(svv_smem);                   // [27][512] filtered populations
  R* s_tile = s_fl + kQ27 * kSvvThreads;                       // [12^3] input populations of one k
  uint32_t* s_src = reinterpret_cast<uint32_t*>(s_tile + kT3);  // [12^3] block << 9 | cell, or none
  const int b = blockIdx.x;
  const int tid = threadIdx.x;
  // the source of every tile cell: this block's core, the axial halo in the face neighbours (at
  // most one block away, 2 < 8); the edge and corner regions of the tile are never read
  for (int t = tid; t < kT3; t += kSvvThreads) {
    const int lx = t % kT - 2, ly = (t / kT) % kT - 2, lz = t / (kT * kT) - 2;
    const int ox = lx < 0 ? -1 : (lx >= kBS ? 1 : 0), oy = ly < 0 ? -1 : (ly >= kBS ? 1 : 0),
              oz = lz < 0 ? -1 : (lz >= kBS ? 1 : 0);
    uint32_t src = kNoSrc;
    if ((ox != 0) + (oy != 0) + (oz != 0) <= 1) {
      int32_t bb = b;
      if (ox | oy | oz) {
        bb = a.nbr[(int64_t)b * kQ27 + nbr_dir(ox, oy, oz)];
        if (bb >= a.n_real) bb = -1;
      }
      if (bb >= 0) {
        const int c = (lx & 7) | ((ly & 7) << 3) | ((lz & 7) << 6);
        if (!svv_solid(a, bb, c)) src = ((uint32_t)bb << 9) | (uint32_t)c;
      }
    }
    s_src[t] = src;
  }
  const int cell = tid;
  const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
  const bool active = !svv_solid(a, b, cell);
  const int tc = (x + 2) + kT * (y + 2) + kT * kT * (z + 2);
  const R ex = R(a.eps_x), eyz = R(a.eps_yz);
  R d_rho = R(0), d_jx = R(0), d_jy = R(0), d_jz = R(0);
  for (int k = 0; k < kQ27; ++k) {
    const R w = R(q27_w(k)), inv_w = R(1.0 / q27_w(k));
    __syncthreads();  // the sources are set; the previous direction's tile has been read
    for (int t = tid; t < kT3; t += kSvvThreads) {
      const uint32_t s = s_src[t];
      s_tile[t] = s != kNoSrc ? Codec<S>::dec(fin[a.pi((int64_t)(s >> 9), (int)(s & 511u), k)], w, inv_w) : R(0);
    }
    __syncthreads();
    if (!active) continue;
    const R own = s_tile[tc];
    auto tap = [&](int d) { return s_src[tc + d] != kNoSrc ? s_tile[tc + d] : own; };
    const R fc = Codec<S>::dec(fout[a.pi(b, cell, k)], w, inv_w);
    R bilap = R(0);
    if (a.eps_x > 0.0f) bilap += ex * ((((tap(-2) - R(4) * tap(-1)) + R(6) * fc) - R(4) * tap(1)) + tap(2));
    if (a.eps_yz > 0.0f) {
      bilap += eyz * ((((tap(-2 * kT) - R(4) * tap(-kT)) + R(6) * fc) - R(4) * tap(kT)) + tap(2 * kT));
      bilap += eyz * ((((tap(-2 * kT * kT) - R(4) * tap(-kT * kT)) + R(6) * fc) - R(4) * tap(kT * kT)) + tap(2 * kT * kT));
    }
    const R ff = fc - bilap;
    const R diff = ff - fc;
    d_rho += diff;
    d_jx += diff * R(q27_cx(k));
    d_jy += diff * R(q27_cy(k));
    d_jz += diff * R(q27_cz(k));
    s_fl[k * kSvvThreads + tid] = ff;
  }
  if (!active) return;
  const R inv_cs2 = R(1) / R(1.0 / 3.0);  // CS2_LATTICE
#pragma unroll 3
  for (int k = 0; k < kQ27; ++k) {
    const R w = R(q27_w(k)), inv_w = R(1.0 / q27_w(k));
    const R cu = R(q27_cx(k)) * d_jx + R(q27_cy(k)) * d_jy + R(q27_cz(k)) * d_jz;
    R v = s_fl[k * kSvvThreads + tid] - w * (d_rho + inv_cs2 * cu);
    v = v < R(1e-12f) ? R(1e-12f) : v;  // NaN passes
    fout[a.pi(b, cell, k)] = Codec<S>::enc(v, w, inv_w);
  }
}

template <class R>
constexpr size_t svv_smem_bytes() {
  return sizeof(R) * ((size_t)kQ27 * kSvvThreads + kT3) + sizeof(uint32_t) * kT3;
}

template <class S, class R>
cudaError_t prepare_t() {
  return cudaFuncSetAttribute(k_svv<S, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)svv_smem_bytes<R>());
}

template <class S, class R>
cudaError_t enqueue_t(const SvvArgs& a, const void* fin, void* fout, int32_t nb, cudaStream_t st) {
  k_svv<S, R><<<(unsigned)nb, kSvvThreads, svv_smem_bytes<R>(), st>>>(a, static_cast<const S*>(fin), static_cast<S*>(fout));
  return cudaGetLastError();
}

}  // namespace

cudaError_t svv_prepare(int32_t storage) {
  switch (storage) {
    case 0: return prepare_t<float, float>();
    case 1: return prepare_t<__half, float>();
    case 2: return prepare_t<__nv_bfloat16, float>();
    case 3: return prepare_t<double, double>();
  }
  return cudaErrorInvalidValue;
}

cudaError_t svv_enqueue(int32_t storage, const void* f_in, void* f_out, const PopIndex& pi, int32_t nb,
                        const int32_t* nbr, int32_t n_real, const int32_t* mslot, const uint32_t* cmask, float eps_x,
                        float eps_yz, cudaStream_t st) {
  if ((eps_x == 0.0f && eps_yz == 0.0f) || nb <= 0) return cudaSuccess;
  if (nb >= (1 << 23)) return cudaErrorInvalidValue;  // block << 9 | cell must fit 32 bits
  SvvArgs a;
  a.pi = pi; a.nbr = nbr; a.n_real = n_real; a.mslot = cmask ? mslot : nullptr; a.cmask = cmask;
  a.eps_x = eps_x; a.eps_yz = eps_yz;
  switch (storage) {
    case 0: return enqueue_t<float, float>(a, f_in, f_out, nb, st);
    case 1: return enqueue_t<__half, float>(a, f_in, f_out, nb, st);
    case 2: return enqueue_t<__nv_bfloat16, float>(a, f_in, f_out, nb, st);
    case 3: return enqueue_t<double, double>(a, f_in, f_out, nb, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace oal
