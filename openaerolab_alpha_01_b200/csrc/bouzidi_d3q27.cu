// bouzidi_d3q27.cu — the linear Bouzidi wall of the reference's default bc_scheme "bouzidi_linear"
// (src/geometry/bouzidi_kernel.jl:150-380, bouzidi_correction_kernel_fixed! on the unshifted D3Q27
// lattice: out_k = opp k, no shifted-wall correction), applied after the step kernels of a level.
//
// The correction reads post-collision populations of the boundary cell and of the cell behind it
// and overwrites f_out[x, opp k]. One boundary cell can be the "behind" cell of another, so the
// reads of every link must see the uncorrected values: the first kernel evaluates all links into
// a side buffer, the second writes them. One thread per (boundary cell, direction); the boundary
// set is a thin shell (a few percent of the cells), so both kernels are a small share of a step.
#include "bouzidi_d3q27.h"

namespace oal {

struct BouzidiArgs {
  const int2* __restrict__ cells;
  const float* __restrict__ q;
  int32_t n;
  float q_min, rel_cap, abs_cap;
  int32_t ff;
  const int32_t* __restrict__ nbr;    // [nb*27] 0-based, -1 = no neighbour (the real topology)
  int32_t n_real;                     // neighbour indices >= n_real (a pool's ghost blocks) count as none
  const int32_t* __restrict__ mslot;  // per-block mask slot or -1 (no solid cell in the block)
  const uint32_t* __restrict__ cmask; // bit 13: the cell itself is solid
  PopIndex pi;
};

__device__ __forceinline__ bool cell_solid(const BouzidiArgs& a, int64_t b, int cell) {
  const int32_t s = a.mslot[b];
  return s >= 0 && ((a.cmask[(int64_t)s * kCells + cell] >> 13) & 1u);
}

template <class S, class R>
__device__ __forceinline__ R load_pop(const S* f, const PopIndex& pi, int64_t b, int cell, int k) {
  return Codec<S>::dec(f[pi(b, cell, k)], R(q27_w(k)), R(1.0 / q27_w(k)));
}

// Density of the boundary cell from its post-collision populations, summed in direction order.
template <class S, class R>
__device__ R cell_rho(const S* f, const PopIndex& pi, int64_t b, int cell) {
  R s = R(0);
  for (int kk = 0; kk < kQ27; ++kk) s += load_pop<S, R>(f, pi, b, cell, kk);
  return s;
}

template <class S, class R>
__global__ void __launch_bounds__(256) k_bouzidi_eval(const BouzidiArgs a, const S* __restrict__ f, R* __restrict__ vals) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)a.n * kQ27) return;
  const float qf = a.q[t];
  if (!(qf > a.q_min && qf <= 1.0f)) return;
  const int k = (int)(t % kQ27);
  const int ok = q27_opp(k);
  const int2 c = a.cells[t / kQ27];
  const int64_t b = c.x;
  const int cell = c.y;
  const R q = R(qf);
  const R fk = load_pop<S, R>(f, a.pi, b, cell, k);
  R rho_f = R(0);
  bool rho_valid = false;
  R raw;
  if (q < R(0.5)) {
    // x_ff = x + c_{opp k}: the cell behind x on the link
    const int nx = (cell & 7) - q27_cx(k), ny = ((cell >> 3) & 7) - q27_cy(k), nz = (cell >> 6) - q27_cz(k);
    R fff = fk;
    bool have = false;
    if (nx >= 0 && nx < kBS && ny >= 0 && ny < kBS && nz >= 0 && nz < kBS) {
      const int nc = nx | (ny << 3) | (nz << 6);
      if (!cell_solid(a, b, nc)) { fff = load_pop<S, R>(f, a.pi, b, nc, k); have = true; }
    } else {
      const int ox = nx < 0 ? -1 : (nx >= kBS ? 1 : 0), oy = ny < 0 ? -1 : (ny >= kBS ? 1 : 0),
                oz = nz < 0 ? -1 : (nz >= kBS ? 1 : 0);
      const int32_t nb = a.nbr[b * kQ27 + nbr_dir(ox, oy, oz)];
      if (nb >= 0 && nb < a.n_real) {
        const int nc = (nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6);
        if (!cell_solid(a, nb, nc)) { fff = load_pop<S, R>(f, a.pi, nb, nc, k); have = true; }
      }
    }
    if (!have && a.ff == 1) {
      rho_f = cell_rho<S, R>(f, a.pi, b, cell);
      rho_valid = true;
      fff = rho_f * R(q27_w(k));  // the no-slip wall equilibrium w_k rho_f
    } else if (!have && a.ff == 2) {
      fff = load_pop<S, R>(f, a.pi, b, cell, ok);
    }
    const R c1 = R(2) * q;
    raw = c1 * fk + (R(1) - c1) * fff;
  } else {
    const R fo = load_pop<S, R>(f, a.pi, b, cell, ok);
    const R inv_2q = R(1) / (R(2) * q);
    const R c2 = (R(2) * q - R(1)) * inv_2q;
    raw = inv_2q * fk + c2 * fo;
  }
  if (a.rel_cap > 0.0f || a.abs_cap > 0.0f) {
    // wall-population limiter about the wall equilibrium of the output direction
    if (!rho_valid) rho_f = cell_rho<S, R>(f, a.pi, b, cell);
    const R target = rho_f * R(q27_w(ok));
    const R scale = fmax(fabs(target), R(1e-12f));
    const R cap = fmax(R(a.abs_cap), R(a.rel_cap) * scale);
    const R lo = target - cap, hi = target + cap;
    raw = raw > hi ? hi : (raw < lo ? lo : raw);  // NaN passes
    raw = raw < R(1e-12f) ? R(1e-12f) : raw;
  }
  vals[t] = raw;
}

template <class S, class R>
__global__ void __launch_bounds__(256) k_bouzidi_apply(const BouzidiArgs a, S* __restrict__ f, const R* __restrict__ vals) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)a.n * kQ27) return;
  const float qf = a.q[t];
  if (!(qf > a.q_min && qf <= 1.0f)) return;
  const int ok = q27_opp((int)(t % kQ27));
  const int2 c = a.cells[t / kQ27];
  f[a.pi(c.x, c.y, ok)] = Codec<S>::enc(vals[t], R(q27_w(ok)), R(1.0 / q27_w(ok)));
}

template <class S, class R>
static cudaError_t enqueue_t(const BouzidiArgs& a, void* f, void* vals, cudaStream_t st) {
  const int64_t n = (int64_t)a.n * kQ27;
  const unsigned grid = (unsigned)((n + 255) / 256);
  k_bouzidi_eval<S, R><<<grid, 256, 0, st>>>(a, static_cast<const S*>(f), static_cast<R*>(vals));
  k_bouzidi_apply<S, R><<<grid, 256, 0, st>>>(a, static_cast<S*>(f), static_cast<const R*>(vals));
  return cudaGetLastError();
}

cudaError_t bouzidi_enqueue(const BouzidiSet& B, int32_t storage, void* f, const PopIndex& pi, const int32_t* nbr,
                            const int32_t* mslot, const uint32_t* cmask, cudaStream_t st, int32_t n_real) {
  if (B.n <= 0) return cudaSuccess;
  BouzidiArgs a;
  a.cells = B.cells; a.q = B.q; a.n = B.n;
  a.q_min = B.q_min; a.rel_cap = B.rel_cap; a.abs_cap = B.abs_cap; a.ff = B.ff_fallback;
  a.nbr = nbr; a.n_real = n_real; a.mslot = mslot; a.cmask = cmask; a.pi = pi;
  switch (storage) {
    case 0: return enqueue_t<float, float>(a, f, B.vals, st);
    case 1: return enqueue_t<__half, float>(a, f, B.vals, st);
    case 2: return enqueue_t<__nv_bfloat16, float>(a, f, B.vals, st);
    case 3: return enqueue_t<double, double>(a, f, B.vals, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace oal
