// level.cu — host runtime of liboal: geometry upload, library-owned level state (ping-pong
// buffers, parity), FP64 reductions, state conversion, CUDA-graph capture of multi-step runs and
// the C-ABI entry points of include/oal.h.
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>

#include "common.cuh"
#include "cumulant_math.cuh"
#include "../../include/oal.h"
#include "bouzidi_d3q27.h"
#include "svv_d3q27.h"
#include "kbc_d3q39.h"
#include "surface_d3q27.h"

namespace oal {
template <class S, class R>
cudaError_t launch_fill_ghosts(const StepArgs& a, const uint2* entries, int64_t n, cudaStream_t st);
template <class S, class R>
cudaError_t launch_fill_copy(const StepArgs& a, const uint2* entries, int64_t n, cudaStream_t st, bool raw = false);
cudaError_t build_fast_records(const int32_t* work, int n, const int32_t* nbr, const int4* binfo, int32_t* rec,
                               cudaStream_t st);
template <class S, class R>
cudaError_t launch_fast(const StepArgs& a, const int32_t* work, int n_work, cudaStream_t st);
template <class S, class R>
cudaError_t launch_general(const StepArgs& a, const int32_t* work, int n_work, cudaStream_t st);
template <class S>
cudaError_t launch_dense_fast(const StepArgs& a, const int32_t* work, int n_work, int grid, cudaStream_t st);
template <class S>
int dense_ctas_per_sm();
template <class S, class R>
cudaError_t launch_restrict(const RestrictArgs& r, cudaStream_t st);
template <class S, class R>
cudaError_t launch_parent_nodes(const ParentView& P, const int32_t* nodes, int32_t n, void* vals, int32_t comp,
                                cudaStream_t st);
template <class R>
cudaError_t launch_parent_positions(const ParentView& P, const int4* pos_xyz, int32_t n, void* macro, cudaStream_t st);
}
using namespace oal;

// IEEE binary16 bits -> float (the reference stores q maps as Float16).
static float half_bits_to_float(uint16_t h) {
  const int e = (h >> 10) & 31, m = h & 1023;
  float v;
  if (e == 0) v = std::ldexp((float)m, -24);                      // zero and subnormals: m 2^-24
  else if (e == 31) v = m ? NAN : INFINITY;
  else v = std::ldexp((float)(m | 1024), e - 25);                 // (1 + m/1024) 2^(e-15)
  return (h & 0x8000) ? -v : v;
}

static void bouzidi_free(BouzidiSet* B) {
  cudaFree(B->cells); cudaFree(B->q); cudaFree(B->vals);
  B->cells = nullptr; B->q = nullptr; B->vals = nullptr; B->n = 0;
}

// ------------------------------------------------------------------------------------------------
// error reporting
// ------------------------------------------------------------------------------------------------
static thread_local std::string g_last_error;

static oal_status set_error(oal_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

// error hook for the other translation units of the library
oal_status oal_internal_set_error(oal_status s, const char* msg) { return set_error(s, "%s", msg); }

// On failure the runtime's (non-sticky) last error is consumed, so it is not reported again by a
// later call's launch check.
#define OAL_CUDA_TRY(expr)                                                                           \
  do {                                                                                               \
    cudaError_t _e = (expr);                                                                         \
    if (_e != cudaSuccess && (cudaGetLastError(), true))                                             \
      return set_error(_e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "%s: %s (%s:%d)", \
                       #expr, cudaGetErrorString(_e), __FILE__, __LINE__);                           \
  } while (0)

// Validates a boundary-cell list (1-based block of a geometry of nb blocks, 1-based x, y, z, binary16
// q per direction) and uploads it as a Bouzidi set whose blocks are offset by `base` (a pool's
// range); replaces the set's previous contents.
static oal_status bouzidi_upload(BouzidiSet* bz, int32_t storage, int64_t nb, int64_t base, int32_t n_cells,
                                 const int32_t* cell_block, const int32_t* cell_x, const int32_t* cell_y,
                                 const int32_t* cell_z, const uint16_t* q_half, float q_min_threshold,
                                 int32_t ff_fallback, float limiter_rel_cap, float limiter_abs_cap) {
  if (n_cells < 0) return set_error(OAL_E_INVALID_ARG, "n_cells %d", n_cells);
  if (ff_fallback < 0 || ff_fallback > 2) return set_error(OAL_E_INVALID_ARG, "ff_fallback %d (0, 1 or 2)", ff_fallback);
  if (!(limiter_rel_cap >= 0.0f) || !(limiter_abs_cap >= 0.0f) || !std::isfinite(q_min_threshold))
    return set_error(OAL_E_INVALID_ARG, "limiter caps must be >= 0 and q_min_threshold finite");
  std::vector<int2> cells((size_t)n_cells);
  std::vector<float> q((size_t)n_cells * 27);
  if (n_cells > 0) {
    if (!cell_block || !cell_x || !cell_y || !cell_z || !q_half) return set_error(OAL_E_INVALID_ARG, "null array");
    for (int32_t i = 0; i < n_cells; ++i) {
      const int32_t b = cell_block[i], x = cell_x[i], y = cell_y[i], z = cell_z[i];
      if (b < 1 || b > nb || x < 1 || x > 8 || y < 1 || y > 8 || z < 1 || z > 8)
        return set_error(OAL_E_INVALID_ARG, "boundary cell %d: block %d, cell (%d, %d, %d) outside the level", i, b, x, y, z);
      cells[(size_t)i] = make_int2((int)(base + b - 1), (x - 1) | ((y - 1) << 3) | ((z - 1) << 6));
    }
    for (size_t j = 0; j < q.size(); ++j) q[j] = half_bits_to_float(q_half[j]);
  }
  bouzidi_free(bz);
  bz->q_min = q_min_threshold;
  bz->ff_fallback = ff_fallback;
  bz->rel_cap = limiter_rel_cap;
  bz->abs_cap = limiter_abs_cap;
  if (n_cells == 0) return OAL_OK;
  const size_t rsz = storage == OAL_STORE_F64 ? sizeof(double) : sizeof(float);
  OAL_CUDA_TRY(cudaMalloc(&bz->cells, cells.size() * sizeof(int2)));
  OAL_CUDA_TRY(cudaMalloc(&bz->q, q.size() * sizeof(float)));
  OAL_CUDA_TRY(cudaMalloc(&bz->vals, q.size() * rsz));
  OAL_CUDA_TRY(cudaMemcpy(bz->cells, cells.data(), cells.size() * sizeof(int2), cudaMemcpyHostToDevice));
  OAL_CUDA_TRY(cudaMemcpy(bz->q, q.data(), q.size() * sizeof(float), cudaMemcpyHostToDevice));
  bz->n = n_cells;
  return OAL_OK;
}


// ------------------------------------------------------------------------------------------------
// device helper kernels
// ------------------------------------------------------------------------------------------------
namespace {

// Deterministic FP64 sum of n triples (fixed strided order per thread, fixed tree).
__global__ void k_reduce3(const double* __restrict__ part, int64_t n, double* __restrict__ out) {
  __shared__ double s[3][256];
  const int t = threadIdx.x;
  double a0 = 0, a1 = 0, a2 = 0;
  for (int64_t i = t; i < n; i += 256) {
    a0 += part[3 * i]; a1 += part[3 * i + 1]; a2 += part[3 * i + 2];
  }
  s[0][t] = a0; s[1][t] = a1; s[2][t] = a2;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w) { s[0][t] += s[0][t + w]; s[1][t] += s[1][t + w]; s[2][t] += s[2][t + w]; }
    __syncthreads();
  }
  if (t == 0) { out[0] = s[0][0]; out[1] = s[1][0]; out[2] = s[2][0]; }
}

// Deterministic FP64 sum of n quadruples.
__global__ void k_reduce4(const double* __restrict__ part, int64_t n, double* __restrict__ out) {
  __shared__ double s[4][256];
  const int t = threadIdx.x;
  double a[4] = {0, 0, 0, 0};
  for (int64_t i = t; i < n; i += 256)
    for (int c = 0; c < 4; ++c) a[c] += part[4 * i + c];
  for (int c = 0; c < 4; ++c) s[c][t] = a[c];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w)
      for (int c = 0; c < 4; ++c) s[c][t] += s[c][t + w];
    __syncthreads();
  }
  if (t == 0)
    for (int c = 0; c < 4; ++c) out[c] = s[c][0];
}

// Per-block FP64 mass and momentum of the fluid cells (state.jl:614-637): one CTA per block.
template <class S, class R>
__global__ void k_mass_momentum(const S* __restrict__ f, PopIndex pi, const uint32_t* __restrict__ bflags,
                                const int32_t* __restrict__ mslot, const uint32_t* __restrict__ cmask,
                                double* __restrict__ part) {
  __shared__ double s[4][16];
  const int b = blockIdx.x, t = threadIdx.x;
  double m = 0, px = 0, py = 0, pz = 0;
  const bool ns = (bflags[b] & BF_NEAR_SOLID) != 0;
  for (int cell = t; cell < kCells; cell += blockDim.x) {
    if (ns && ((cmask[(int64_t)mslot[b] * kCells + cell] >> 13) & 1u)) continue;
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      const double v = (double)Codec<S>::dec(f[pi(b, cell, k)], R(q27_w(k)), R(1.0 / q27_w(k)));
      m += v; px += v * q27_cx(k); py += v * q27_cy(k); pz += v * q27_cz(k);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    m += __shfl_down_sync(0xffffffffu, m, o);
    px += __shfl_down_sync(0xffffffffu, px, o);
    py += __shfl_down_sync(0xffffffffu, py, o);
    pz += __shfl_down_sync(0xffffffffu, pz, o);
  }
  if ((t & 31) == 0) { s[0][t >> 5] = m; s[1][t >> 5] = px; s[2][t >> 5] = py; s[3][t >> 5] = pz; }
  __syncthreads();
  if (t < 4) {
    double acc = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) acc += s[t][w];
    part[4 * (int64_t)b + t] = acc;
  }
}

// Equilibrium start (physics_utils.jl:30-35 / 65-95) from reference-layout double rho / vel.
template <class S, class R>
__global__ void k_init_feq(const double* __restrict__ rho, const double* __restrict__ vel, int64_t ncell, int comp,
                           S* __restrict__ f, PopIndex pi, R* __restrict__ rho_out, R* __restrict__ vel_out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  const int64_t b = i >> 9, cell = i & 511;
  const R r = R(rho[i]), ux = R(vel[i]), uy = R(vel[i + ncell]), uz = R(vel[i + 2 * ncell]);
  const R usq = ux * ux + uy * uy + uz * uz;
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R w = R(q27_w(k));
    const R cu = R(q27_cx(k)) * ux + R(q27_cy(k)) * uy + R(q27_cz(k)) * uz;
    R val = R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq;
    if (comp) {
      const R cu2 = cu * cu;
      val += (R(4.5) * cu2 * cu - R(4.5) * cu * usq) + (R(3.375) * cu2 * cu2 - R(6.75) * cu2 * usq + R(1.125) * usq * usq);
    }
    f[pi(b, (int)cell, k)] = Codec<S>::enc(r * w * val, w, R(1.0 / q27_w(k)));
  }
  rho_out[i] = r;
  vel_out[i] = ux; vel_out[i + ncell] = uy; vel_out[i + 2 * ncell] = uz;
}

// Reference-layout double -> storage layout.
template <class S, class R>
__global__ void k_import_f(const double* __restrict__ src, int64_t ncell, S* __restrict__ f, PopIndex pi) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  const int64_t b = i >> 9, cell = i & 511;
#pragma unroll
  for (int k = 0; k < kQ27; ++k)
    f[pi(b, (int)cell, k)] = Codec<S>::enc(R(src[i + ncell * k]), R(q27_w(k)), R(1.0 / q27_w(k)));
}
// Storage layout -> reference-layout double.
template <class S, class R>
__global__ void k_export_f(const S* __restrict__ f, PopIndex pi, int64_t ncell, double* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  const int64_t b = i >> 9, cell = i & 511;
#pragma unroll
  for (int k = 0; k < kQ27; ++k)
    dst[i + ncell * k] = (double)Codec<S>::dec(f[pi(b, (int)cell, k)], R(q27_w(k)), R(1.0 / q27_w(k)));
}
template <class R>
__global__ void k_to_double(const R* __restrict__ src, int64_t n, double* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}
template <class R>
__global__ void k_from_double(const double* __restrict__ src, int64_t n, R* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = R(src[i]);
}

// Non-equilibrium stress of the stored state (compute_pi_neq_kernel!, kernel_pi_neq.jl:39-180):
// one thread per cell, f decoded from the current buffer, rho and u from the level's macros.
template <class S, class R, class O>
__global__ void k_pi_neq(const S* __restrict__ f, PopIndex pi, const R* __restrict__ rho, const R* __restrict__ vel,
                         const uint32_t* __restrict__ bflags, const int32_t* __restrict__ mslot,
                         const uint32_t* __restrict__ cmask, int64_t ncell, int comp, O* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  const int64_t b = i >> 9;
  const int cell = (int)(i & 511);
  const bool obs = (bflags[b] & BF_NEAR_SOLID) && ((cmask[(int64_t)mslot[b] * kCells + cell] >> 13) & 1u);
  const R r = rho[i], ux = vel[i], uy = vel[i + ncell], uz = vel[i + 2 * ncell];
  const bool skip = obs || !isfinite(r) || r < R(0.01) || r > R(10) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz);
  R fk[kQ27];
#pragma unroll
  for (int k = 0; k < kQ27; ++k) fk[k] = Codec<S>::dec(f[pi(b, cell, k)], R(q27_w(k)), R(1.0 / q27_w(k)));
  R p[6];
  pi_neq_of<R>(fk, r, ux, uy, uz, comp != 0, skip, p);
#pragma unroll
  for (int m = 0; m < 6; ++m) out[i + m * ncell] = O(p[m]);
}

// Characteristic (NSCBC) outlet, apply_nscbc_outlet_kernel! (kernel_nscbc_outlet.jl:80-340),
// athermal: one thread per (y, z) of the x = 8 plane of a listed block, face cell x = 8 and its
// interior neighbour x = 7; both fluid. Macros in, new macros and face populations out (the
// library is compiled without FMA contraction, so each operation rounds as written).
struct NscbcArgs {
  float p_target, k_relax, neq_blend;
  int32_t ny, nz;  // global cells of the domain (the corner test)
};
template <class S, class R>
__global__ void __launch_bounds__(64) k_nscbc(S* __restrict__ f, PopIndex pi, R* __restrict__ rho, R* __restrict__ vel,
                                              int64_t vcs, const int32_t* __restrict__ blocks, int32_t n,
                                              const int4* __restrict__ binfo, const uint32_t* __restrict__ bflags,
                                              const int32_t* __restrict__ mslot, const uint32_t* __restrict__ cmask,
                                              NscbcArgs na) {
  if ((int)blockIdx.x >= n) return;
  const int64_t b = blocks[blockIdx.x];
  const int y = threadIdx.x & 7, z = threadIdx.x >> 3;
  const int cf = 7 | (y << 3) | (z << 6), ci = 6 | (y << 3) | (z << 6);
  if (bflags[b] & BF_NEAR_SOLID) {
    const uint32_t* m = cmask + (int64_t)mslot[b] * kCells;
    if (((m[cf] >> 13) & 1u) || ((m[ci] >> 13) & 1u)) return;
  }
  const int4 bi = binfo[b];
  const int gy = (bi.y - 1) * kBS + y + 1, gz = (bi.z - 1) * kBS + z + 1;
  const bool corner = gy == 1 || gy == na.ny || gz == 1 || gz == na.nz;
  const int64_t vf = b * kCells + cf, vi = b * kCells + ci;
  const R rf = rho[vf], uf = vel[vf], vff = vel[vf + vcs], wf = vel[vf + 2 * vcs];
  const R ri = rho[vi], ui = vel[vi], vi_ = vel[vi + vcs], wi = vel[vi + 2 * vcs];
  const R Ru = R(1) / R(3), T = R(1);  // p = rho R T with R = cs^2 and T = 1
  const R pf = rf * Ru * T, pint = ri * Ru * T;
  const R g = R(1);
  const R c = sqrt(fmax(g * Ru * T, R(1e-12)));
  const R drho = rf - ri, du = uf - ui, dv = vff - vi_, dw = wf - wi, dp = pf - pint;
  const R un = uf;
  const R mach = un / fmax(c, R(1e-6));
  R L1 = (un - c) * (dp - rf * c * du);
  const R L2 = un * (c * c * drho - dp);
  const R L3 = corner ? R(0) : un * dv;
  const R L4 = corner ? R(0) : un * dw;
  const R L5 = (un + c) * (dp + rf * c * du);
  if (mach < R(1) && un > R(0)) {
    const R mc = fmin(fmax(mach, R(0.05f)), R(0.95f));
    L1 = R(na.k_relax) * (R(1) - mc * mc) * (pf - R(na.p_target));
  }
  const R d1 = (R(1) / (c * c)) * (L2 + R(0.5) * (L5 + L1));
  const R d2 = R(0.5) * (L5 + L1);
  const R d3 = (L5 - L1) / (R(2) * rf * c + R(1e-12));
  auto cl = [](R x, R lo, R hi) { return x > hi ? hi : (x < lo ? lo : x); };
  const R cap = corner ? R(0.10f) : R(0.20f);
  const R d1c = cl(d1, -cap * rf, cap * rf), d2c = cl(d2, R(-0.10f) * pf, R(0.10f) * pf);
  const R d3c = cl(d3, R(-0.10f) * c, R(0.10f) * c);
  const R L3c = cl(L3, R(-0.10f) * c, R(0.10f) * c), L4c = cl(L4, R(-0.10f) * c, R(0.10f) * c);
  R rn = rf - d1c;
  const R un2 = uf - d3c;
  const R vn = corner ? vi_ : vff - L3c;
  const R wn = corner ? wi : wf - L4c;
  R pn = pf - d2c;
  rn = cl(rn, R(0.1f), R(10));
  pn = fmax(pn, R(1e-6));
  const R Tn = cl(pn / (rn * Ru + R(1e-12)), R(0.1f), R(10));
  rho[vf] = rn;
  vel[vf] = un2; vel[vf + vcs] = vn; vel[vf + 2 * vcs] = wn;
  const R inv_n = R(1) / fmax(Ru * Tn, R(1e-12)), inv_i = R(1) / fmax(Ru * T, R(1e-12));
  const R usq_n = un2 * un2 + vn * vn + wn * wn, usq_i = ui * ui + vi_ * vi_ + wi * wi;
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R cx = R(q27_cx(k)), cy = R(q27_cy(k)), cz = R(q27_cz(k)), w = R(q27_w(k));
    const R cun = cx * un2 + cy * vn + cz * wn;
    const R fen = fmax(rn * w * (R(1) + cun * inv_n + R(0.5) * cun * cun * inv_n * inv_n - R(0.5) * usq_n * inv_n), R(1e-15));
    const R cui = cx * ui + cy * vi_ + cz * wi;
    const R fei = fmax(ri * w * (R(1) + cui * inv_i + R(0.5) * cui * cui * inv_i * inv_i - R(0.5) * usq_i * inv_i), R(1e-15));
    const R fi = Codec<S>::dec(f[pi(b, ci, k)], w, R(1.0 / q27_w(k)));
    f[pi(b, cf, k)] = Codec<S>::enc(fen + R(na.neq_blend) * (fi - fei), w, R(1.0 / q27_w(k)));
  }
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

size_t storage_bytes(int32_t storage) {
  switch (storage) {
    case OAL_STORE_F32: return 4;
    case OAL_STORE_F16_DEV: return 2;
    case OAL_STORE_BF16_DEV: return 2;
    case OAL_STORE_F64: return 8;
  }
  return 0;
}
size_t macro_bytes(int32_t storage) { return storage == OAL_STORE_F64 ? 8 : 4; }

}  // namespace

// ------------------------------------------------------------------------------------------------
// objects
// ------------------------------------------------------------------------------------------------
struct oal_geometry {
  int device = 0;
  int32_t nb = 0, nx = 0, ny = 0, nz = 0;
  int32_t n_ghost = 0;             // ghost blocks appended after the real ones (library-owned levels)
  int32_t* d_nbr = nullptr;        // [nb*27] 0-based, -1 = none (caller-owned arrays)
  int32_t* d_nbr_ghost = nullptr;  // [nb*27] missing neighbours point at ghost blocks
  uint2* d_gentries = nullptr;     // ghost fill entries (block, cell | k << 9)
  int64_t n_gentries = 0;
  int32_t* d_fast = nullptr;       // blocks for the uniform kernel
  int32_t* d_fast_rec = nullptr;   // their 32-int records (neighbour row, coordinates, index)
  int32_t n_fast_in = 0;           // the first n_fast_in fast blocks read no ghost slot
  int32_t* d_general = nullptr;    // blocks for the general kernel
  int32_t n_fast = 0, n_general = 0;
  // ghost fill split by face conditions (one entry per key of fill_key_of, kept until the
  // geometry is destroyed: captured graphs may hold the pointers)
  struct FillLists {
    uint32_t key;
    uint2* copy;   // raw copies, inlet and weight values (k_fill_copy)
    int64_t n_copy;
    uint2* rest;   // entries for the general fill kernel
    int64_t n_rest;
    std::vector<uint2> h_copies;  // host: the raw copies alone (dst, src) (batches rebase them)
    std::vector<uint2> h_other;   // host: every other entry as a fill entry (block, cell | k << 9)
  };
  std::vector<FillLists> fills;
  int4* d_binfo = nullptr;
  uint32_t* d_bflags = nullptr;
  int32_t* d_mslot = nullptr;
  uint32_t* d_cmask = nullptr;
  float* d_sponge = nullptr;
  float* d_wdist = nullptr;
  double* d_force_part = nullptr;  // scratch of oal_stream_collide
  double* d_force = nullptr;
  int64_t n_fluid = 0, n_solid = 0, n_boundary = 0, n_slots = 0;
  // box levels (every block of a bx x by x bz box): dense padded population layout
  bool box = false;
  int32_t bdim[3] = {0, 0, 0};
  uint32_t pmask = 0;              // CF_PERIODIC_* bits
  uint2* d_dense_gentries = nullptr;  // (block, cell | k << 9 | wrap << 31)
  int64_t n_dense_gentries = 0;
  int32_t* d_dense_fast = nullptr;    // uniform blocks, x fastest
  // host copies of the block-layout tables (batches remap them into a shared block pool)
  std::vector<int32_t> h_nbrg;       // [nb*27], ghost-indexed
  std::vector<int4> h_binfo;
  std::vector<uint32_t> h_bflags;
  std::vector<int32_t> h_mslot;
  std::vector<uint32_t> h_cmask;
  std::vector<uint2> h_gentries;
  std::vector<int32_t> h_fast, h_general;
  std::vector<float> h_sponge, h_wdist;
  std::vector<int32_t> h_box_at;     // box levels: block index at ((bx-1)*by + by-1)*bz + bz-1
  bool dense_tables = false;
  // levels built on this geometry; destroying the geometry while levels live defers the release
  // to the last level's destroy
  int32_t n_levels = 0;
  bool destroy_requested = false;
};

// Stream resources of an overlapped step: the general kernel (blocks at solids, sponge, wall
// model) runs on `side` while the uniform kernel runs on the caller's stream.
struct Overlap {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

struct GraphCache {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  int32_t n = 0;
  int parity = -1;
  oal_step_params p{};
};

struct oal_level {
  const oal_geometry* g = nullptr;
  int device = 0;
  int32_t op = 0, storage = 0;
  // dense padded layout (box levels, FP32/FP16/BF16)
  bool dense = false;
  bool round_nearest = false;  // OAL_LEVEL_ROUND_NEAREST
  int32_t PX = 0, PY = 0, PZ = 0;
  int32_t dense_grid = 0;
  uint32_t* d_err = nullptr;
  void* f[2] = {nullptr, nullptr};
  void* vel[2] = {nullptr, nullptr};
  void* rho = nullptr;
  double* d_force_part = nullptr;
  double* d_force = nullptr;
  uint32_t* d_ticket = nullptr;  // the general kernel's last-CTA ticket (fused drag sum)
  double* d_mm_part = nullptr;
  double* d_mm = nullptr;
  int parity = 0;
  int64_t bytes = 0;
  cudaStream_t cap = nullptr;
  Overlap ov;
  GraphCache gc;
  bool forces_valid = false;
  KbcLevel* kbc = nullptr;  // D3Q39 entropic levels: the whole state lives here
  ParentView par{};         // refined level of a block-AMR hierarchy: its parent (set per step)
  BouzidiSet bz;            // linear Bouzidi boundary cells (oal_level_set_bouzidi)
  // surface-stress mapping (oal_level_set_surface): triangles, block pointer, outputs
  float* s_tri = nullptr;
  int32_t s_n = 0;
  int32_t* s_ptr = nullptr;
  float* s_out = nullptr;
  double* s_part = nullptr;
  double* s_sum = nullptr;
  uint32_t bz_gen = 0;      // bumped by every oal_level_set_bouzidi (hierarchy graphs compare it)
  // variable nu_sgs from Pi_neq: the post-collision non-equilibrium stress of the previous step,
  // 6 components x n_blocks x 512 in the compute type, refreshed in place by the general kernel
  void* pi_neq = nullptr;
  bool comp = false;        // the last step's compressible equilibrium (oal_level_pi_neq)
  int32_t prefetch_ctas = 0;  // launch tuning (OAL_TUNE_PREFETCH_CTAS)
  int32_t persistent = 0;     // launch tuning (OAL_TUNE_PERSISTENT)
  // spectral vanishing viscosity of the step being enqueued (oal_step_params svv_*_epsilon)
  float svv_x = 0.0f, svv_yz = 0.0f;
  // characteristic outlet (oal_level_set_nscbc): settings and the listed blocks
  oal_nscbc_params nscbc{};
  int32_t* d_nscbc_blocks = nullptr;
  int32_t n_nscbc = 0;
};

// ------------------------------------------------------------------------------------------------
// parameter resolution
// ------------------------------------------------------------------------------------------------
static oal_status resolve_params(const oal_step_params* p, const oal_geometry* g, CaseParams* cp) {
  if (!p) return set_error(OAL_E_INVALID_ARG, "null step params");
  if (p->abi_version != OAL_ABI_VERSION)
    return set_error(OAL_E_ABI_MISMATCH, "oal_step_params.abi_version %u != %d", p->abi_version, OAL_ABI_VERSION);
  if (p->operator_id != OAL_OP_CUMULANT_D3Q27)
    return set_error(OAL_E_UNSUPPORTED, "operator %d has no level-step kernel in this build", p->operator_id);
  if (!(p->tau > 0.5f) || !std::isfinite(p->tau)) return set_error(OAL_E_INVALID_ARG, "tau must be > 0.5 (got %g)", p->tau);
  if (p->limiter_type < 0 || p->limiter_type > 2) return set_error(OAL_E_INVALID_ARG, "limiter_type %d", p->limiter_type);
  if (p->zwall_bc < 0 || p->zwall_bc > 2) return set_error(OAL_E_INVALID_ARG, "zwall_bc %d", p->zwall_bc);
  if (p->solid_bc != OAL_SOLID_FULLWAY && p->solid_bc != OAL_SOLID_HALFWAY && p->solid_bc != OAL_SOLID_GRAD &&
      p->solid_bc != OAL_SOLID_BOUZIDI)
    return set_error(OAL_E_INVALID_ARG, "solid_bc %d", p->solid_bc);
  if (p->variable_nu_sgs < 0 || p->variable_nu_sgs > 2)
    return set_error(OAL_E_INVALID_ARG, "variable_nu_sgs %d (0 off, 1 Pi_neq, 2 dynamic)", p->variable_nu_sgs);
  if (!(p->svv_x_epsilon >= 0.0f) || !std::isfinite(p->svv_x_epsilon) || !(p->svv_yz_epsilon >= 0.0f) ||
      !std::isfinite(p->svv_yz_epsilon))
    return set_error(OAL_E_INVALID_ARG, "svv_x_epsilon and svv_yz_epsilon must be finite and >= 0");
  if (p->solid_bc == OAL_SOLID_BOUZIDI && p->collect_forces)
    return set_error(OAL_E_UNSUPPORTED, "collect_forces with OAL_SOLID_BOUZIDI: the momentum exchange would be the full-way "
                                        "wall's, computed before the Bouzidi correction; use the surface-stress forces");
  std::memset(cp, 0, sizeof *cp);
  cp->tau = p->tau;
  cp->c_wale = p->c_wale;
  cp->nu_sgs_bg = p->nu_sgs_background;
  cp->amr_sgs_scale = p->amr_sgs_scale;
  cp->omega_bulk = p->omega_bulk;
  cp->omega3 = p->omega3;
  cp->omega4 = p->omega4;
  cp->lambda_param = p->lambda_param;
  cp->u_inlet = p->u_inlet;
  cp->inlet_turbulence = p->inlet_turbulence;
  cp->wall_model_max_distance = p->wall_model_max_distance;
  cp->transverse_blend = p->transverse_freestream_blend;
  cp->time_step_seed = p->time_step_seed;
  cp->nx = g->nx; cp->ny = g->ny; cp->nz = g->nz;
  uint32_t f = 0;
  if (p->adaptive_omega4 == 1) f |= CF_ADAPTIVE_OMEGA4;
  if (p->limiter_type == OAL_LIMITER_FACTORED) f |= CF_LIMITER_FACTORED;
  if (p->limiter_type == OAL_LIMITER_POSITIVITY) f |= CF_LIMITER_POSITIVITY;
  if (p->compressible_corr == 1) f |= CF_COMPRESSIBLE;
  if (p->ymin_wall_bc == 1) f |= CF_YMIN_WALL;
  if (p->zwall_bc == 1) f |= CF_ZWALL_SLIP;
  if (p->zwall_bc == 2) f |= CF_ZWALL_NOSLIP;
  if (p->wall_model_active == 1) f |= CF_WALL_MODEL;
  if (p->sponge_blend_distributions == 1) f |= CF_SPONGE_BLEND;
  if (p->transverse_freestream == 1) f |= CF_TRANSVERSE_FS;
  if (p->solid_bc == OAL_SOLID_HALFWAY) f |= CF_HALFWAY;
  if (p->solid_bc == OAL_SOLID_GRAD) f |= CF_GRAD_WALL;
  if (p->solid_bc == OAL_SOLID_BOUZIDI) f |= CF_BOUZIDI;
  cp->grad_pineq_scale = p->grad_pineq_scale;
  if (p->collect_forces) f |= CF_COLLECT;
  if (p->store_post_collision == 1) f |= CF_STORE_POST;
  if (p->c_wale != 0.0f) f |= CF_GRADIENTS;
  if (p->inlet_turbulence > 0.0f) f |= CF_INLET_NOISE;
  if (p->omega_bulk != 1.0f || p->omega3 != 1.0f || p->omega4 != 1.0f) f |= CF_GENERAL_RATES;
  if (p->variable_nu_sgs == 1) f |= CF_SGS_PI;
  if (p->variable_nu_sgs == 2) f |= CF_SGS_DYNAMIC | CF_GRADIENTS;
  cp->c_pi = p->c_pi;
  cp->nu_sgs_floor = p->nu_sgs_floor;
  cp->flags = f;
  return OAL_OK;
}

// The case flags that decide where a ghost value comes from.
static uint32_t fill_key_of(uint32_t flags) {
  return flags & (CF_YMIN_WALL | CF_ZWALL_SLIP | CF_ZWALL_NOSLIP | CF_TRANSVERSE_FS | CF_INLET_NOISE);
}

// Split the ghost fill entries for the face conditions of `flags` (the branches of
// face_population_impl for a level without parent): a stored word of a real cell of the same
// lattice weight (outlet, mirrors, walls, the slip image), the inlet equilibrium without noise,
// the lattice weight, or anything else (transverse freestream blend, inlet noise), which stays on
// the general fill. Built on the host once per key, outside any stream capture.
static oal_status build_fill_lists(oal_geometry* g, uint32_t flags) {
  const uint32_t key = fill_key_of(flags);
  for (const auto& c : g->fills)
    if (c.key == key) return OAL_OK;
  const int64_t bst = 27 * kCells, kst = kCells;
  if ((int64_t)(g->nb + g->n_ghost) * bst >= (1ll << 31)) return OAL_OK;  // element index must fit 31 bits
  std::vector<uint2> copy, rest, copies, other;
  copy.reserve(g->h_gentries.size());
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  for (const uint2& en : g->h_gentries) {
    const int64_t b = en.x;
    const int cell = (int)(en.y & 511u), k = (int)((en.y >> 9) & 31u);
    const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
    const int4 bi = g->h_binfo[(size_t)b];
    const int gx = (bi.x - 1) * kBS + x + 1, gy = (bi.y - 1) * kBS + y + 1, gz = (bi.z - 1) * kBS + z + 1;
    const int cx = q27_cx(k), cy = q27_cy(k), cz = q27_cz(k);
    const int sx = x - cx, sy = y - cy, sz = z - cz;
    const int32_t gblk = g->h_nbrg[(size_t)b * 27 + nbr_dir(sx >> 3, sy >> 3, sz >> 3)];
    const uint32_t dst = (uint32_t)((int64_t)gblk * bst + k * kst + ((sx & 7) | ((sy & 7) << 3) | ((sz & 7) << 6)));
    const int sgx = gx - cx, sgy = gy - cy, sgz = gz - cz;
    const bool zmin = sgz < 1, zmax = sgz > nz, ymin = sgy < 1, ymax = sgy > ny;
    int j = k;
    int64_t src = -1;
    uint32_t code = 0;
    bool general = false, constant = false;
    if (sgx < 1) {
      if (flags & CF_INLET_NOISE) general = true;
      else { code = 0x80000000u | (uint32_t)k; constant = true; }
    } else if (sgx > nx) {
      j = k;
    } else if ((flags & (CF_ZWALL_SLIP | CF_ZWALL_NOSLIP)) && (zmin || zmax)) {
      if (flags & CF_ZWALL_NOSLIP) {
        j = q27_opp(k);
      } else {
        j = q27_mir_z(k);
        const int ix = x - cx, iy = y - cy;
        if (ix >= 0 && ix < kBS && iy >= 0 && iy < kBS) {
          src = b * bst + j * kst + (ix + 8 * iy + 64 * z);
        } else {
          const int32_t nb2 = g->h_nbrg[(size_t)b * 27 + nbr_dir(ix >> 3, iy >> 3, 0)];
          if (nb2 >= 0 && nb2 < g->nb) src = (int64_t)nb2 * bst + j * kst + ((ix & 7) + 8 * (iy & 7) + 64 * z);
        }
      }
    } else if ((flags & CF_TRANSVERSE_FS) && (ymin || ymax || zmin || zmax)) {
      general = true;
    } else if (ymin && (flags & CF_YMIN_WALL)) {
      j = q27_opp(k);
    } else if (ymin || ymax) {
      j = q27_mir_y(k);
    } else if (zmin || zmax) {
      j = q27_mir_z(k);
    } else {
      code = 0xC0000000u | (uint32_t)k;
      constant = true;
    }
    if (general) { rest.push_back(en); other.push_back(en); continue; }
    if (!constant) code = (uint32_t)(src >= 0 ? src : b * bst + j * kst + cell);
    copy.push_back(make_uint2(dst, code));
    if (constant) other.push_back(en);
    else copies.push_back(make_uint2(dst, code));
  }
  // consecutive threads write consecutive slots
  std::sort(copy.begin(), copy.end(), [](const uint2& p, const uint2& q) { return p.x < q.x; });
  std::sort(copies.begin(), copies.end(), [](const uint2& p, const uint2& q) { return p.x < q.x; });
  oal_geometry::FillLists fl{key, nullptr, (int64_t)copy.size(), nullptr, (int64_t)rest.size(), std::move(copies),
                             std::move(other)};
  cudaError_t e = cudaSuccess;
  if (!copy.empty()) {
    e = cudaMalloc(&fl.copy, copy.size() * sizeof(uint2));
    if (e == cudaSuccess) e = cudaMemcpy(fl.copy, copy.data(), copy.size() * sizeof(uint2), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !rest.empty()) {
    e = cudaMalloc(&fl.rest, rest.size() * sizeof(uint2));
    if (e == cudaSuccess) e = cudaMemcpy(fl.rest, rest.data(), rest.size() * sizeof(uint2), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(fl.copy); cudaFree(fl.rest);
    OAL_CUDA_TRY(e);
  }
  g->fills.push_back(std::move(fl));
  return OAL_OK;
}

// Builds the fill lists of the level's face conditions when the stream is not being captured
// (a level with a parent or a dense layout keeps the general fill).
static oal_status prepare_fill(oal_level* L, const CaseParams& cp, cudaStream_t st) {
  if (L->dense || L->par.ptr || L->g->n_gentries == 0) return OAL_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  OAL_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return OAL_OK;
  return build_fill_lists(const_cast<oal_geometry*>(L->g), cp.flags);
}

// The Pi_neq field of variable nu_sgs mode 1, zero at first use (allocated outside a capture).
static oal_status prepare_sgs(oal_level* L, const CaseParams& cp, cudaStream_t st) {
  if (!(cp.flags & CF_SGS_PI) || L->pi_neq) return OAL_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  OAL_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return set_error(OAL_E_UNSUPPORTED, "variable_nu_sgs 1: first step inside a stream capture");
  const size_t bytes = (size_t)L->g->nb * 512 * 6 * macro_bytes(L->storage);
  OAL_CUDA_TRY(cudaMalloc(&L->pi_neq, bytes));
  OAL_CUDA_TRY(cudaMemset(L->pi_neq, 0, bytes));
  L->bytes += (int64_t)bytes;
  return OAL_OK;
}

// Which kernels one step launches.
enum StepPath { PATH_PLAIN = 0, PATH_GHOSTED = 1 };

// x-pair blocks [first, first + count) of a fast list and its records
template <class S, class R>
static cudaError_t launch_fast_range(const StepArgs& a, const int32_t* work, int first, int count, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  StepArgs b = a;
  if (b.fast_rec) b.fast_rec += (int64_t)first * 32;
  return launch_fast<S, R>(b, work + first, count, st);
}

template <class S, class R>
static cudaError_t launch_step_t(const oal_geometry* g, const StepArgs& a0, StepPath path, cudaStream_t st,
                                 const Overlap* ov) {
  cudaError_t e;
  if (path == PATH_PLAIN) return launch_general<S, R>(a0, nullptr, g->nb, st);
  StepArgs a = a0;
  a.fast_rec = g->d_fast_rec;
  const oal_geometry::FillLists* fl = nullptr;
  if (!a.par.ptr && !a.dense && !a.cases)
    for (const auto& c : g->fills)
      if (c.key == fill_key_of(a.p0.flags)) fl = &c;
  auto fill = [&](cudaStream_t s) -> cudaError_t {
    cudaError_t r;
    if (!fl) return launch_fill_ghosts<S, R>(a, g->d_gentries, g->n_gentries, s);
    if ((r = launch_fill_copy<S, R>(a, fl->copy, fl->n_copy, s)) != cudaSuccess) return r;
    return launch_fill_ghosts<S, R>(a, fl->rest, fl->n_rest, s);
  };
  if (a.flags_any & (CF_SGS_PI | CF_SGS_DYNAMIC)) {
    // variable nu_sgs: every block in the general kernel (per-cell test filter / Pi_neq refresh)
    if ((e = fill(st)) != cudaSuccess) return e;
    return launch_general<S, R>(a, nullptr, g->nb, st);
  }
  // high-priority side stream: ghost fill, then the blocks that read ghost slots (general kernel,
  // boundary x-pair blocks); main stream: the interior x-pair blocks, which read none
  const int n_in = g->n_fast_in, n_bd = g->n_fast - g->n_fast_in;
  const bool fork = ov && ov->side && n_in > 0 && (g->n_general > 0 || n_bd > 0);
  if (fork) {
    if ((e = cudaEventRecord(ov->fork, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ov->side, ov->fork, 0)) != cudaSuccess) return e;
    if ((e = fill(ov->side)) != cudaSuccess) return e;
    if ((e = launch_general<S, R>(a, g->d_general, g->n_general, ov->side)) != cudaSuccess) return e;
    if ((e = launch_fast_range<S, R>(a, g->d_fast, n_in, n_bd, ov->side)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ov->join, ov->side)) != cudaSuccess) return e;
    if ((e = launch_fast_range<S, R>(a, g->d_fast, 0, n_in, st)) != cudaSuccess) return e;
    return cudaStreamWaitEvent(st, ov->join, 0);
  }
  if ((e = fill(st)) != cudaSuccess) return e;
  if ((e = launch_fast<S, R>(a, g->d_fast, g->n_fast, st)) != cudaSuccess) return e;
  return launch_general<S, R>(a, g->d_general, g->n_general, st);
}

static cudaError_t launch_by_storage(int32_t storage, const oal_geometry* g, const StepArgs& a, StepPath path,
                                     cudaStream_t st, const Overlap* ov = nullptr) {
  switch (storage) {
    case OAL_STORE_F32: return launch_step_t<float, float>(g, a, path, st, ov);
    case OAL_STORE_F16_DEV: return launch_step_t<__half, float>(g, a, path, st, ov);
    case OAL_STORE_BF16_DEV: return launch_step_t<__nv_bfloat16, float>(g, a, path, st, ov);
    case OAL_STORE_F64: return launch_step_t<double, double>(g, a, path, st, ov);
  }
  return cudaErrorInvalidValue;
}

static void fill_geometry_args(const oal_geometry* g, StepArgs* a) {
  a->nbr = g->d_nbr;
  a->binfo = g->d_binfo;
  a->bflags = g->d_bflags;
  a->mslot = g->d_mslot;
  a->cmask = g->d_cmask;
  a->sponge = g->d_sponge;
  a->wall_dist = g->d_wdist;
  a->n_blocks = g->nb;
  a->block_base = 0;
  a->cases = nullptr;
}

static void level_layout(const oal_level* L, int64_t* bst, int64_t* kst) {
  if (L->dense) {
    *bst = 0;
    *kst = (int64_t)L->PX * L->PY * L->PZ;  // dense: f[k][Z][Y][X]
  } else {
    *bst = 27 * 512;  // block-major: f[b][k][cell]
    *kst = 512;
  }
}

static PopIndex pop_index(const oal_level* L) {
  PopIndex pi{};
  pi.binfo = L->g->d_binfo;
  pi.dense = L->dense ? 1 : 0;
  pi.PX = L->PX;
  pi.PY = L->PY;
  level_layout(L, &pi.bst, &pi.kst);
  return pi;
}

template <class S, class R>
static cudaError_t init_feq_t(oal_level* L, const double* d_rho, const double* d_vel, int comp) {
  const int64_t ncell = (int64_t)L->g->nb * 512;
  k_init_feq<S, R><<<nblk(ncell, 256), 256>>>(d_rho, d_vel, ncell, comp, static_cast<S*>(L->f[0]), pop_index(L),
                                              static_cast<R*>(L->rho), static_cast<R*>(L->vel[0]));
  return cudaGetLastError();
}

template <class S, class R>
static cudaError_t import_t(oal_level* L, const double* d_f, const double* d_rho, const double* d_vel) {
  const int64_t ncell = (int64_t)L->g->nb * 512;
  k_import_f<S, R><<<nblk(ncell, 256), 256>>>(d_f, ncell, static_cast<S*>(L->f[L->parity]), pop_index(L));
  if (d_rho) k_from_double<R><<<nblk(ncell, 256), 256>>>(d_rho, ncell, static_cast<R*>(L->rho));
  if (d_vel) k_from_double<R><<<nblk(3 * ncell, 256), 256>>>(d_vel, 3 * ncell, static_cast<R*>(L->vel[L->parity]));
  return cudaGetLastError();
}
template <class S, class R>
static cudaError_t export_t(oal_level* L, double* d_f, double* d_rho, double* d_vel) {
  const int64_t ncell = (int64_t)L->g->nb * 512;
  if (d_f) k_export_f<S, R><<<nblk(ncell, 256), 256>>>(static_cast<const S*>(L->f[L->parity]), pop_index(L), ncell, d_f);
  if (d_rho) k_to_double<R><<<nblk(ncell, 256), 256>>>(static_cast<const R*>(L->rho), ncell, d_rho);
  if (d_vel) k_to_double<R><<<nblk(3 * ncell, 256), 256>>>(static_cast<const R*>(L->vel[L->parity]), 3 * ncell, d_vel);
  return cudaGetLastError();
}

template <class S, class R>
static cudaError_t mm_t(oal_level* L) {
  const oal_geometry* g = L->g;
  k_mass_momentum<S, R><<<g->nb, 128>>>(static_cast<const S*>(L->f[L->parity]), pop_index(L), g->d_bflags, g->d_mslot,
                                        g->d_cmask, L->d_mm_part);
  k_reduce4<<<1, 256>>>(L->d_mm_part, g->nb, L->d_mm);
  return cudaGetLastError();
}

template <class S, class R>
static cudaError_t dense_step_t(oal_level* L, const StepArgs& a, cudaStream_t st) {
  const oal_geometry* g = L->g;
  cudaError_t e;
  if ((e = launch_fill_ghosts<S, R>(a, g->d_dense_gentries, g->n_dense_gentries, st)) != cudaSuccess) return e;
  if (a.flags_any & (CF_SGS_PI | CF_SGS_DYNAMIC)) return launch_general<S, R>(a, nullptr, g->nb, st);
  const int n_fast = (int)(g->nb - g->n_general);
  if (g->n_general > 0) {
    if ((e = cudaEventRecord(L->ov.fork, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(L->ov.side, L->ov.fork, 0)) != cudaSuccess) return e;
    if ((e = launch_general<S, R>(a, g->d_general, g->n_general, L->ov.side)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(L->ov.join, L->ov.side)) != cudaSuccess) return e;
  }
  if ((e = launch_dense_fast<S>(a, g->d_dense_fast, n_fast, L->dense_grid, st)) != cudaSuccess) return e;
  if (g->n_general > 0) return cudaStreamWaitEvent(st, L->ov.join, 0);
  return cudaSuccess;
}

// Pi_neq of the state in buffer `parity` into d_out (6 x n_blocks x 512, type O).
template <class S, class R, class O>
static cudaError_t pi_neq_t(oal_level* L, int parity, O* d_out, cudaStream_t st) {
  const oal_geometry* g = L->g;
  const int64_t ncell = (int64_t)g->nb * 512;
  k_pi_neq<S, R, O><<<nblk(ncell, 128), 128, 0, st>>>(static_cast<const S*>(L->f[parity]), pop_index(L),
                                                      static_cast<const R*>(L->rho), static_cast<const R*>(L->vel[parity]),
                                                      g->d_bflags, g->d_mslot, g->d_cmask, ncell, L->comp ? 1 : 0, d_out);
  return cudaGetLastError();
}

template <class S, class R>
static cudaError_t nscbc_t(oal_level* L, void* f, void* vel, cudaStream_t st) {
  const oal_geometry* g = L->g;
  NscbcArgs na;
  na.p_target = L->nscbc.p_target;
  na.neq_blend = L->nscbc.neq_blend;
  // K = sigma c_ref / L_ref with c_ref = sqrt(gamma R) at gamma 1, R 2/3 (the driver's athermal
  // defaults, kernel_nscbc_outlet.jl:366-368) and L_ref the domain length in x
  const float c_ref = std::sqrt(1.0f * float(2.0 / 3.0));
  na.k_relax = L->nscbc.sigma_relax * c_ref / std::max((float)g->nx, 1.0f);
  na.ny = g->ny; na.nz = g->nz;
  k_nscbc<S, R><<<(unsigned)L->n_nscbc, 64, 0, st>>>(static_cast<S*>(f), pop_index(L), static_cast<R*>(L->rho),
                                                      static_cast<R*>(vel), (int64_t)g->nb * 512, L->d_nscbc_blocks,
                                                      L->n_nscbc, g->d_binfo, g->d_bflags, g->d_mslot, g->d_cmask, na);
  return cudaGetLastError();
}

// Reads (and clears) the level's device error word after a synchronisation.
static oal_status check_level_error(oal_level* L) {
  uint32_t w = 0;
  OAL_CUDA_TRY(cudaMemcpy(&w, L->d_err, sizeof w, cudaMemcpyDeviceToHost));
  if (w == 0) return OAL_OK;
  OAL_CUDA_TRY(cudaMemset(L->d_err, 0, sizeof w));
  return set_error(OAL_E_TIMEOUT, "a bounded device wait gave up (code 0x%x); the step's results are invalid", w);
}

// Dense ghost-frame slots and the x-fastest uniform work order of a box geometry (first dense level).
static oal_status build_dense_tables(oal_geometry* g) {
  if (g->dense_tables) return OAL_OK;
  const int64_t nb = g->nb;
  const int bxm = g->bdim[0], bym = g->bdim[1], bzm = g->bdim[2];
  const int N[3] = {8 * bxm, 8 * bym, 8 * bzm};
  const bool per[3] = {(g->pmask & CF_PERIODIC_X) != 0, (g->pmask & CF_PERIODIC_Y) != 0, (g->pmask & CF_PERIODIC_Z) != 0};
  std::vector<uint2> dentries;
  // every (cell, k) whose source leaves the box; a crossing of periodic axes only is a copy of the
  // wrapped interior cell, any other goes through the face rules
  for (int64_t b = 0; b < nb; ++b) {
    const int4 bi = g->h_binfo[(size_t)b];
    const int g0[3] = {(bi.x - 1) * 8, (bi.y - 1) * 8, (bi.z - 1) * 8};
    const bool edge = g0[0] == 0 || g0[1] == 0 || g0[2] == 0 || g0[0] + 8 == N[0] || g0[1] + 8 == N[1] || g0[2] + 8 == N[2];
    if (!edge) continue;
    for (int cell = 0; cell < 512; ++cell) {
      const int c3[3] = {g0[0] + (cell & 7), g0[1] + ((cell >> 3) & 7), g0[2] + (cell >> 6)};
      for (int k = 0; k < 27; ++k) {
        const int ck[3] = {q27_cx(k), q27_cy(k), q27_cz(k)};
        bool out = false, face = false;
        for (int ax = 0; ax < 3; ++ax) {
          const int sc = c3[ax] - ck[ax];
          if (sc < 0 || sc >= N[ax]) { out = true; if (!per[ax]) face = true; }
        }
        if (out) dentries.push_back(make_uint2((uint32_t)b, (uint32_t)cell | ((uint32_t)k << 9) | (face ? 0u : (1u << 31))));
      }
    }
  }
  std::vector<uint8_t> gen((size_t)nb, 0);
  for (int32_t b : g->h_general) gen[(size_t)b] = 1;
  std::vector<int32_t> dfast;
  // uniform blocks ordered x fastest, so CTAs running together write neighbouring rows
  for (int bz = 1; bz <= bzm; ++bz)
    for (int by = 1; by <= bym; ++by)
      for (int bx = 1; bx <= bxm; ++bx) {
        const int32_t b = g->h_box_at[((size_t)(bx - 1) * bym + (by - 1)) * bzm + (bz - 1)];
        if (!gen[(size_t)b]) dfast.push_back(b);
      }
  OAL_CUDA_TRY(cudaSetDevice(g->device));
  if (!dentries.empty()) {
    OAL_CUDA_TRY(cudaMalloc(&g->d_dense_gentries, dentries.size() * sizeof(uint2)));
    OAL_CUDA_TRY(cudaMemcpy(g->d_dense_gentries, dentries.data(), dentries.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  }
  if (!dfast.empty()) {
    OAL_CUDA_TRY(cudaMalloc(&g->d_dense_fast, dfast.size() * sizeof(int32_t)));
    OAL_CUDA_TRY(cudaMemcpy(g->d_dense_fast, dfast.data(), dfast.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  g->n_dense_gentries = (int64_t)dentries.size();
  g->dense_tables = true;
  return OAL_OK;
}

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------
extern "C" {

int32_t oal_abi_version(void) { return OAL_ABI_VERSION; }

const char* oal_status_string(oal_status s) {
  switch (s) {
    case OAL_OK: return "ok";
    case OAL_E_INVALID_ARG: return "invalid argument";
    case OAL_E_UNKNOWN_OPERATOR: return "unknown collision operator";
    case OAL_E_CUDA: return "CUDA error";
    case OAL_E_OUT_OF_MEMORY: return "out of device memory";
    case OAL_E_UNSUPPORTED: return "unsupported";
    case OAL_E_ABI_MISMATCH: return "ABI version mismatch";
    case OAL_E_ADMISSION: return "request exceeds the memory budget";
    case OAL_E_TOO_LARGE: return "size exceeds the supported maximum";
    case OAL_E_NOT_FOUND: return "not found";
    case OAL_E_TIMEOUT: return "timeout";
    case OAL_E_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

const char* oal_last_error(void) { return g_last_error.c_str(); }

int32_t oal_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
  return n;
}

oal_status oal_lookup_operator(const char* name, int32_t* out) {
  if (!name || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  std::string s(name);
  if (!s.empty() && s[0] == ':') s = s.substr(1);
  if (s == "cumulant") { *out = OAL_OP_CUMULANT_D3Q27; return OAL_OK; }
  if (s == "entropic") { *out = OAL_OP_ENTROPIC_D3Q39; return OAL_OK; }
  if (s == "hrr" || s == "octree_q19") { *out = OAL_OP_HRR_D3Q19; return OAL_OK; }
  return set_error(OAL_E_UNKNOWN_OPERATOR,
                   "Unknown or retired operator: :%s. Valid options: :cumulant (D3Q27), :entropic (D3Q39), :hrr (D3Q19 octree).",
                   s.c_str());
}

void oal_default_step_params(oal_step_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->abi_version = OAL_ABI_VERSION;
  p->operator_id = OAL_OP_CUMULANT_D3Q27;
  p->tau = 0.6f;
  p->tau_parent = 0.6f;
  p->c_wale = 0.20f;              // config_loader.jl:1305
  p->nu_sgs_background = 0.0f;    // :1310
  p->amr_sgs_scale = 1.0f;        // timestep.jl:1127
  p->omega_bulk = 1.0f;           // :1373
  p->omega3 = 1.0f;               // :1374
  p->omega4 = 1.0f;               // :1375
  p->adaptive_omega4 = 1;         // :1376
  p->lambda_param = 1.0f / 6.0f;  // :1377
  p->limiter_type = OAL_LIMITER_FACTORED;  // :1379
  p->compressible_corr = 0;
  p->u_inlet = 0.05f;
  p->inlet_turbulence = 0.0f;
  p->time_step_seed = 0;
  p->ymin_wall_bc = 0;
  p->zwall_bc = 0;
  p->wall_model_active = 0;       // :1870
  p->wall_model_max_distance = 10.0f;  // :1873
  p->sponge_blend_distributions = 0;
  p->transverse_freestream = 0;
  p->transverse_freestream_blend = 1.0f;
  p->solid_bc = OAL_SOLID_FULLWAY;
  p->collect_forces = 0;
  p->store_post_collision = 0;
  p->temporal_weight = 1.0f;
  p->use_temporal_interp = 0;
  p->level_visc_physical = 0;
  p->hrr_hybrid = 0;
  p->hrr_sigma = 1.0f;            // :2283
  p->nu_sgs_lattice_floor = 0.0f; // :733
  p->shock_nu_max = 0.0f;
  p->grad_pineq_scale = 1.0f;     // config_loader.jl:898
  p->variable_nu_sgs = 0;         // VARIABLE_NU_SGS, config_loader.jl:237
  p->c_pi = 0.2f;                 // :238
  p->nu_sgs_floor = 0.002f;       // :239
}

void oal_default_entropic_params(oal_step_params* p) {
  oal_default_step_params(p);
  if (!p) return;
  p->operator_id = OAL_OP_ENTROPIC_D3Q39;
  p->lambda_param = 0.0f;         // ENTROPIC_SIGMA, config_loader.jl:1391
  p->adaptive_omega4 = 0;         // alpha_solver "bisection", config_loader.jl:1386
  p->omega_bulk = p->omega3 = p->omega4 = 0.0f;  // timestep.jl:1136-1138
  p->limiter_type = 0;
}

oal_status oal_build_box_blocks(int32_t bxm, int32_t bym, int32_t bzm, int32_t periodic_mask, int32_t* coords,
                                int32_t* nbr) {
  if (bxm <= 0 || bym <= 0 || bzm <= 0 || !coords || !nbr) return set_error(OAL_E_INVALID_ARG, "bad box");
  const int64_t n = (int64_t)bxm * bym * bzm;
  // sorted tuples (bx, by, bz): bx most significant (domain.jl:785)
  auto index_of = [&](int bx, int by, int bz) -> int64_t { return ((int64_t)(bx - 1) * bym + (by - 1)) * bzm + (bz - 1); };
  for (int bx = 1; bx <= bxm; ++bx)
    for (int by = 1; by <= bym; ++by)
      for (int bz = 1; bz <= bzm; ++bz) {
        const int64_t i = index_of(bx, by, bz);
        coords[3 * i] = bx; coords[3 * i + 1] = by; coords[3 * i + 2] = bz;
      }
  const bool px = periodic_mask & 1, py = periodic_mask & 2, pz = periodic_mask & 4;
  for (int64_t i = 0; i < n; ++i) {
    const int bx = coords[3 * i], by = coords[3 * i + 1], bz = coords[3 * i + 2];
    for (int d = 0; d < 27; ++d) {
      int nx = bx + d % 3 - 1, ny = by + (d / 3) % 3 - 1, nz = bz + d / 9 - 1;
      if (px) nx = nx < 1 ? bxm : (nx > bxm ? 1 : nx);
      if (py) ny = ny < 1 ? bym : (ny > bym ? 1 : ny);
      if (pz) nz = nz < 1 ? bzm : (nz > bzm ? 1 : nz);
      const bool in = nx >= 1 && nx <= bxm && ny >= 1 && ny <= bym && nz >= 1 && nz <= bzm;
      nbr[i + n * d] = in ? (int32_t)(index_of(nx, ny, nz) + 1) : 0;
    }
  }
  return OAL_OK;
}

oal_status oal_build_sphere_obstacle(int32_t nb, const int32_t* coords, double cx, double cy, double cz, double radius,
                                     uint8_t* obst, int64_t* n_solid) {
  if (nb <= 0 || !coords || !obst) return set_error(OAL_E_INVALID_ARG, "bad sphere arguments");
  const double r2 = radius * radius;
  int64_t count = 0;
  for (int64_t b = 0; b < nb; ++b)
    for (int lz = 1; lz <= 8; ++lz)
      for (int ly = 1; ly <= 8; ++ly)
        for (int lx = 1; lx <= 8; ++lx) {
          const double px = (coords[3 * b] - 1) * 8 + lx - 0.5;
          const double py = (coords[3 * b + 1] - 1) * 8 + ly - 0.5;
          const double pz = (coords[3 * b + 2] - 1) * 8 + lz - 0.5;
          const double d = (px - cx) * (px - cx) + (py - cy) * (py - cy) + (pz - cz) * (pz - cz);
          const uint8_t s = d <= r2;
          obst[(lx - 1) + 8 * (ly - 1) + 64 * (lz - 1) + 512 * b] = s;
          count += s;
        }
  if (n_solid) *n_solid = count;
  return OAL_OK;
}

oal_status oal_geometry_create(const oal_geometry_desc* d, int32_t device, oal_geometry** out) {
  if (!d || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  *out = nullptr;
  if (d->n_blocks <= 0 || !d->active_coords || !d->neighbor_table)
    return set_error(OAL_E_INVALID_ARG, "geometry needs n_blocks > 0, active_coords and neighbor_table");
  if (d->nx_global <= 0 || d->ny_global <= 0 || d->nz_global <= 0)
    return set_error(OAL_E_INVALID_ARG, "global sizes must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(OAL_E_NO_DEVICE, "no CUDA device visible");
  }
  if (device < 0 || device >= ndev) return set_error(OAL_E_INVALID_ARG, "device %d out of range", device);
  OAL_CUDA_TRY(cudaSetDevice(device));

  const int64_t nb = d->n_blocks;
  std::vector<int32_t> nbr0((size_t)nb * 27);
  std::vector<int4> binfo((size_t)nb);
  std::vector<uint32_t> bflags((size_t)nb, 0);
  for (int64_t b = 0; b < nb; ++b) {
    bool interior = true;
    for (int dir = 0; dir < 27; ++dir) {
      const int32_t v = d->neighbor_table[b + nb * dir];
      if (v < 0 || v > nb) return set_error(OAL_E_INVALID_ARG, "neighbor_table[%lld,%d] = %d out of range", (long long)b, dir, v);
      nbr0[(size_t)b * 27 + dir] = v - 1;
      if (v == 0) interior = false;
    }
    if (nbr0[(size_t)b * 27 + 13] != b)
      return set_error(OAL_E_INVALID_ARG, "neighbor_table[%lld, self] must be the block itself", (long long)b);
    binfo[(size_t)b] = make_int4(d->active_coords[3 * b], d->active_coords[3 * b + 1], d->active_coords[3 * b + 2], 0);
    if (interior) bflags[(size_t)b] |= BF_INTERIOR;
  }
  auto* g = new oal_geometry();
  g->device = device;
  g->nb = d->n_blocks; g->nx = d->nx_global; g->ny = d->ny_global; g->nz = d->nz_global;

  // per-cell solid masks: bit k = source cell x - c_k is solid, bit 13 = own cell solid
  std::vector<int32_t> mslot((size_t)nb, -1);
  std::vector<uint32_t> cmask;
  int64_t n_solid = 0;
  if (d->obstacle) {
    // only blocks with a solid cell in their 27-block neighbourhood can carry mask bits
    std::vector<uint8_t> has_solid((size_t)nb, 0);
    for (int64_t b = 0; b < nb; ++b)
      for (int c = 0; c < 512 && !has_solid[(size_t)b]; ++c) has_solid[(size_t)b] = d->obstacle[b * 512 + c] != 0;
    std::vector<uint32_t> m(512);
    for (int64_t b = 0; b < nb; ++b) {
      bool near = false;
      for (int dir = 0; dir < 27 && !near; ++dir) {
        const int32_t sb = nbr0[(size_t)b * 27 + dir];
        near = sb >= 0 && has_solid[(size_t)sb];
      }
      if (!near) continue;
      bool any = false;
      for (int cell = 0; cell < 512; ++cell) {
        const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
        uint32_t bits = 0;
        for (int k = 0; k < 27; ++k) {
          const int sx = x - q27_cx(k), sy = y - q27_cy(k), sz = z - q27_cz(k);
          const int dir = nbr_dir(sx >> 3, sy >> 3, sz >> 3);
          const int32_t sb = nbr0[(size_t)b * 27 + dir];
          if (sb < 0) continue;
          const int sc = (sx & 7) | ((sy & 7) << 3) | ((sz & 7) << 6);
          if (d->obstacle[(int64_t)sb * 512 + sc]) bits |= 1u << k;
        }
        m[cell] = bits;
        if (bits) any = true;
        if (bits & (1u << 13)) ++n_solid;
      }
      if (any) {
        mslot[(size_t)b] = (int32_t)(cmask.size() / 512);
        cmask.insert(cmask.end(), m.begin(), m.end());
        bflags[(size_t)b] |= BF_NEAR_SOLID;
      }
    }
  }
  g->n_solid = n_solid;
  g->n_fluid = nb * 512 - n_solid;
  g->n_slots = (int64_t)cmask.size() / 512;
  for (int64_t b = 0; b < nb; ++b)
    if (!(bflags[(size_t)b] & BF_INTERIOR)) ++g->n_boundary;

  // Ghost blocks: every missing neighbour position gets a block appended after the real ones; the
  // fill kernel writes into it, before each step, exactly the populations that real cells pull
  // from it, so the step kernels pull uniformly. A ghost slot (cell g, direction k) feeds the
  // single destination g + c_k, so no two entries write the same slot.
  std::vector<int32_t> nbrg(nbr0);
  std::vector<uint2> gentries;
  {
    std::vector<int64_t> keys;  // packed ghost block coordinates, index = ghost id
    auto pack = [](int64_t bx, int64_t by, int64_t bz) { return ((bx + 4) << 42) | ((by + 4) << 21) | (bz + 4); };
    std::vector<std::pair<int64_t, int32_t>> lookup;
    for (int64_t b = 0; b < nb; ++b)
      for (int dir = 0; dir < 27; ++dir) {
        if (nbr0[(size_t)b * 27 + dir] >= 0) continue;
        const int64_t key = pack(binfo[b].x + dir % 3 - 1, binfo[b].y + (dir / 3) % 3 - 1, binfo[b].z + dir / 9 - 1);
        keys.push_back(key);
      }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    g->n_ghost = (int32_t)keys.size();
    for (int64_t b = 0; b < nb; ++b)
      for (int dir = 0; dir < 27; ++dir) {
        if (nbr0[(size_t)b * 27 + dir] >= 0) continue;
        const int64_t key = pack(binfo[b].x + dir % 3 - 1, binfo[b].y + (dir / 3) % 3 - 1, binfo[b].z + dir / 9 - 1);
        const int64_t gi = std::lower_bound(keys.begin(), keys.end(), key) - keys.begin();
        nbrg[(size_t)b * 27 + dir] = (int32_t)(nb + gi);
      }
    for (int64_t b = 0; b < nb; ++b) {
      if (bflags[(size_t)b] & BF_INTERIOR) continue;
      for (int cell = 0; cell < 512; ++cell) {
        const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
        for (int k = 0; k < 27; ++k) {
          const int sx = x - q27_cx(k), sy = y - q27_cy(k), sz = z - q27_cz(k);
          if (nbr0[(size_t)b * 27 + nbr_dir(sx >> 3, sy >> 3, sz >> 3)] < 0)
            gentries.push_back(make_uint2((uint32_t)b, (uint32_t)cell | ((uint32_t)k << 9)));
        }
      }
    }
  }
  // direction-major order: consecutive fill threads read and write the same direction plane of
  // neighbouring cells (coalesced), instead of 27 planes of one cell
  std::stable_sort(gentries.begin(), gentries.end(), [](const uint2& p, const uint2& q) {
    const uint32_t kp = (p.y >> 9) & 31u, kq = (q.y >> 9) & 31u;
    return kp != kq ? kp < kq : p.x < q.x;
  });
  g->n_gentries = (int64_t)gentries.size();
  // Work lists: blocks near solids, with sponge cells or with wall distances take the general kernel.
  std::vector<int32_t> fast, general;
  for (int64_t b = 0; b < nb; ++b) {
    bool gen = (bflags[(size_t)b] & BF_NEAR_SOLID) != 0;
    for (int c = 0; c < 512 && !gen; ++c) {
      if (d->sponge && d->sponge[b * 512 + c] > 0.0f) gen = true;
      if (d->wall_dist && d->wall_dist[b * 512 + c] > 0.0f) gen = true;
    }
    (gen ? general : fast).push_back((int32_t)b);
  }
  // interior blocks first: they pull no ghost slot, so their step need not wait for the fill
  std::stable_partition(fast.begin(), fast.end(), [&](int32_t b) { return (bflags[(size_t)b] & BF_INTERIOR) != 0; });
  g->n_fast_in = (int32_t)std::count_if(fast.begin(), fast.end(), [&](int32_t b) { return (bflags[(size_t)b] & BF_INTERIOR) != 0; });
  g->n_fast = (int32_t)fast.size();
  g->n_general = (int32_t)general.size();

  // Box levels: every block of the bx x by x bz box present -> a dense padded population layout
  // is available. Periodic axes are read from the neighbour table (a first block that has a
  // neighbour across the low face of an axis wraps on that axis). The dense ghost-frame entries
  // and work order are built by the first dense level (build_dense_tables).
  {
    int bxm = 0, bym = 0, bzm = 0;
    bool ok = true;
    for (int64_t b = 0; b < nb; ++b) {
      if (binfo[b].x < 1 || binfo[b].y < 1 || binfo[b].z < 1) ok = false;
      bxm = std::max(bxm, binfo[b].x); bym = std::max(bym, binfo[b].y); bzm = std::max(bzm, binfo[b].z);
    }
    ok = ok && (int64_t)bxm * bym * bzm == nb && d->nx_global == 8 * bxm && d->ny_global == 8 * bym &&
         d->nz_global == 8 * bzm;
    if (ok) {
      std::vector<int32_t> at((size_t)nb, -1);
      for (int64_t b = 0; b < nb && ok; ++b) {
        const int64_t key = ((int64_t)(binfo[b].x - 1) * bym + (binfo[b].y - 1)) * bzm + (binfo[b].z - 1);
        if (at[(size_t)key] >= 0) ok = false; else at[(size_t)key] = (int32_t)b;
      }
      if (ok) {
        g->box = true;
        g->bdim[0] = bxm; g->bdim[1] = bym; g->bdim[2] = bzm;
        const int64_t first = at[0];  // block (1,1,1)
        if (nbr0[(size_t)first * 27 + nbr_dir(-1, 0, 0)] >= 0) g->pmask |= CF_PERIODIC_X;
        if (nbr0[(size_t)first * 27 + nbr_dir(0, -1, 0)] >= 0) g->pmask |= CF_PERIODIC_Y;
        if (nbr0[(size_t)first * 27 + nbr_dir(0, 0, -1)] >= 0) g->pmask |= CF_PERIODIC_Z;
        g->h_box_at = at;
      }
    }
  }

  g->h_nbrg = nbrg;
  g->h_binfo = binfo;
  g->h_bflags = bflags;
  g->h_mslot = mslot;
  g->h_cmask = cmask;
  g->h_gentries = gentries;
  g->h_fast = fast;
  g->h_general = general;
  if (d->sponge) g->h_sponge.assign(d->sponge, d->sponge + nb * 512);
  if (d->wall_dist) g->h_wdist.assign(d->wall_dist, d->wall_dist + nb * 512);

  auto fail = [&](oal_status s) { oal_geometry_destroy(g); return s; };
#define GTRY(expr)                                                                         \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess)                                                                 \
      return fail(set_error(_e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "%s: %s", #expr, \
                            cudaGetErrorString(_e)));                                      \
  } while (0)
  GTRY(cudaMalloc(&g->d_nbr, nbr0.size() * sizeof(int32_t)));
  GTRY(cudaMemcpy(g->d_nbr, nbr0.data(), nbr0.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  GTRY(cudaMalloc(&g->d_binfo, binfo.size() * sizeof(int4)));
  GTRY(cudaMemcpy(g->d_binfo, binfo.data(), binfo.size() * sizeof(int4), cudaMemcpyHostToDevice));
  GTRY(cudaMalloc(&g->d_bflags, bflags.size() * sizeof(uint32_t)));
  GTRY(cudaMemcpy(g->d_bflags, bflags.data(), bflags.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  GTRY(cudaMalloc(&g->d_mslot, mslot.size() * sizeof(int32_t)));
  GTRY(cudaMemcpy(g->d_mslot, mslot.data(), mslot.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (!cmask.empty()) {
    GTRY(cudaMalloc(&g->d_cmask, cmask.size() * sizeof(uint32_t)));
    GTRY(cudaMemcpy(g->d_cmask, cmask.data(), cmask.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  }
  if (d->sponge) {
    GTRY(cudaMalloc(&g->d_sponge, (size_t)nb * 512 * sizeof(float)));
    GTRY(cudaMemcpy(g->d_sponge, d->sponge, (size_t)nb * 512 * sizeof(float), cudaMemcpyHostToDevice));
  }
  if (d->wall_dist) {
    GTRY(cudaMalloc(&g->d_wdist, (size_t)nb * 512 * sizeof(float)));
    GTRY(cudaMemcpy(g->d_wdist, d->wall_dist, (size_t)nb * 512 * sizeof(float), cudaMemcpyHostToDevice));
  }
  GTRY(cudaMalloc(&g->d_nbr_ghost, nbrg.size() * sizeof(int32_t)));
  GTRY(cudaMemcpy(g->d_nbr_ghost, nbrg.data(), nbrg.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (!gentries.empty()) {
    GTRY(cudaMalloc(&g->d_gentries, gentries.size() * sizeof(uint2)));
    GTRY(cudaMemcpy(g->d_gentries, gentries.data(), gentries.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  }
  if (!fast.empty()) {
    GTRY(cudaMalloc(&g->d_fast, fast.size() * sizeof(int32_t)));
    GTRY(cudaMemcpy(g->d_fast, fast.data(), fast.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (!general.empty()) {
    GTRY(cudaMalloc(&g->d_general, general.size() * sizeof(int32_t)));
    GTRY(cudaMemcpy(g->d_general, general.data(), general.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (!fast.empty()) {
    GTRY(cudaMalloc(&g->d_fast_rec, fast.size() * 32 * sizeof(int32_t)));
    GTRY(build_fast_records(g->d_fast, (int)fast.size(), g->d_nbr_ghost, g->d_binfo, g->d_fast_rec, nullptr));
    GTRY(cudaDeviceSynchronize());
  }
  GTRY(cudaMalloc(&g->d_force_part, (size_t)nb * 4 * 3 * sizeof(double)));
  GTRY(cudaMalloc(&g->d_force, 3 * sizeof(double)));
  GTRY(cudaMemset(g->d_force, 0, 3 * sizeof(double)));
#undef GTRY
  *out = g;
  return OAL_OK;
}

static void geometry_release(oal_geometry* g) {
  cudaSetDevice(g->device);
  cudaFree(g->d_nbr_ghost); cudaFree(g->d_gentries); cudaFree(g->d_fast); cudaFree(g->d_general);
  cudaFree(g->d_fast_rec);
  for (auto& c : g->fills) { cudaFree(c.copy); cudaFree(c.rest); }
  g->fills.clear();
  cudaFree(g->d_dense_gentries); cudaFree(g->d_dense_fast);
  cudaFree(g->d_nbr); cudaFree(g->d_binfo); cudaFree(g->d_bflags); cudaFree(g->d_mslot);
  cudaFree(g->d_cmask); cudaFree(g->d_sponge); cudaFree(g->d_wdist);
  cudaFree(g->d_force_part); cudaFree(g->d_force);
  cudaGetLastError();
  delete g;
}

void oal_geometry_destroy(oal_geometry* g) {
  if (!g) return;
  if (g->n_levels > 0) { g->destroy_requested = true; return; }
  geometry_release(g);
}

oal_status oal_geometry_info(const oal_geometry* g, int64_t out[5]) {
  if (!g || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  out[0] = g->nb; out[1] = g->n_fluid; out[2] = g->n_solid; out[3] = g->n_boundary; out[4] = g->n_slots;
  return OAL_OK;
}

oal_status oal_stream_collide(const oal_geometry* g, const oal_level_fields* fl, const oal_step_params* p, void* stream) {
  if (!g || !fl) return set_error(OAL_E_INVALID_ARG, "null argument");
  CaseParams cp;
  oal_status s = resolve_params(p, g, &cp);
  if (s != OAL_OK) return s;
  if (cp.flags & (CF_SGS_PI | CF_SGS_DYNAMIC))
    return set_error(OAL_E_UNSUPPORTED, "variable_nu_sgs: the Pi_neq field and the test filter belong to plain levels, not to caller-owned arrays (oal_stream_collide)");
  if (!fl->f_in || !fl->f_out || !fl->rho_out || !fl->vel_out || !fl->vel_in)
    return set_error(OAL_E_INVALID_ARG, "f_in, f_out, rho_out, vel_out and vel_in are required");
  if (fl->f_in == fl->f_out) return set_error(OAL_E_INVALID_ARG, "f_in and f_out must differ (pull scheme)");
  if (fl->storage < OAL_STORE_F32 || fl->storage > OAL_STORE_F64) return set_error(OAL_E_INVALID_ARG, "storage %d", fl->storage);
  if (fl->f_block_stride < 512 || fl->f_dir_stride < 512) return set_error(OAL_E_INVALID_ARG, "bad population strides");
  OAL_CUDA_TRY(cudaSetDevice(g->device));
  StepArgs a{};
  fill_geometry_args(g, &a);
  a.f_in = fl->f_in; a.f_out = fl->f_out; a.f_post = fl->f_post_collision;
  a.rho_out = fl->rho_out; a.vel_out = fl->vel_out; a.vel_in = fl->vel_in;
  a.f_bstride = fl->f_block_stride; a.f_kstride = fl->f_dir_stride;
  a.v_bstride = 512; a.v_cstride = fl->vel_comp_stride > 0 ? fl->vel_comp_stride : 512 * (int64_t)g->nb;
  a.force_part = g->d_force_part;
  a.p0 = cp;
  a.flags_any = cp.flags;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  OAL_CUDA_TRY(launch_by_storage(fl->storage, g, a, PATH_PLAIN, st));
  if (p->svv_x_epsilon > 0.0f || p->svv_yz_epsilon > 0.0f) {
    // the filter on the caller's output, and on its f_post_collision when given (the reference's
    // filter writes both on a level with boundary cells, timestep.jl:1584-1594)
    PopIndex pi{};
    pi.binfo = g->d_binfo;
    pi.bst = fl->f_block_stride;
    pi.kst = fl->f_dir_stride;
    const int64_t n_el = (int64_t)(g->nb - 1) * pi.bst + 26 * pi.kst + 512;
    OAL_CUDA_TRY(svv_enqueue(fl->storage, fl->f_in, fl->f_out, pi, g->nb, n_el, g->d_nbr, g->nb, g->d_mslot, g->d_cmask,
                             p->svv_x_epsilon, p->svv_yz_epsilon, st, fl->f_post_collision));
  }
  if ((cp.flags & CF_COLLECT) && fl->force_out) {
    k_reduce3<<<1, 256, 0, st>>>(g->d_force_part, (int64_t)g->nb * 4, fl->force_out);
    OAL_CUDA_TRY(cudaGetLastError());
  }
  return OAL_OK;
}

struct oal_bouzidi {
  const oal_geometry* g = nullptr;
  int32_t storage = 0;
  BouzidiSet bz;
};

oal_status oal_bouzidi_create(const oal_geometry* g, int32_t storage, int32_t n_cells, const int32_t* cell_block,
                              const int32_t* cell_x, const int32_t* cell_y, const int32_t* cell_z,
                              const uint16_t* q_half, float q_min_threshold, int32_t ff_fallback,
                              float limiter_rel_cap, float limiter_abs_cap, oal_bouzidi** out) {
  if (!g || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (storage < OAL_STORE_F32 || storage > OAL_STORE_F64) return set_error(OAL_E_INVALID_ARG, "storage %d", storage);
  *out = nullptr;
  OAL_CUDA_TRY(cudaSetDevice(g->device));
  auto* B = new oal_bouzidi();
  B->g = g;
  B->storage = storage;
  oal_status s = bouzidi_upload(&B->bz, storage, g->nb, 0, n_cells, cell_block, cell_x, cell_y, cell_z, q_half,
                                q_min_threshold, ff_fallback, limiter_rel_cap, limiter_abs_cap);
  if (s != OAL_OK) {
    bouzidi_free(&B->bz);
    delete B;
    return s;
  }
  *out = B;
  return OAL_OK;
}

void oal_bouzidi_destroy(oal_bouzidi* B) {
  if (!B) return;
  cudaSetDevice(B->g->device);
  bouzidi_free(&B->bz);
  delete B;
}

oal_status oal_bouzidi_apply(const oal_geometry* g, oal_bouzidi* B, const oal_level_fields* fl, void* stream) {
  if (!g || !B || !fl || !fl->f_out) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (B->g != g) return set_error(OAL_E_INVALID_ARG, "the boundary cells belong to another geometry");
  if (fl->storage != B->storage) return set_error(OAL_E_INVALID_ARG, "storage %d, the set was built for %d", fl->storage, B->storage);
  if (fl->f_block_stride < 512 || fl->f_dir_stride < 512) return set_error(OAL_E_INVALID_ARG, "bad population strides");
  OAL_CUDA_TRY(cudaSetDevice(g->device));
  PopIndex pix{};
  pix.binfo = g->d_binfo;
  pix.bst = fl->f_block_stride;
  pix.kst = fl->f_dir_stride;
  OAL_CUDA_TRY(bouzidi_enqueue(B->bz, B->storage, fl->f_out, pix, g->d_nbr, g->d_mslot, g->d_cmask,
                               static_cast<cudaStream_t>(stream)));
  return OAL_OK;
}

// ---- levels ----
// D3Q39 entropic level: FP32 populations on a library-built geometry (faces, solids, sponge and
// wall distance as the geometry carries them; the wall model is not built for it)
static oal_status create_entropic_level(const oal_geometry* g, int32_t storage, uint32_t flags, oal_level** out) {
  if (storage != OAL_STORE_F32)
    return set_error(OAL_E_UNSUPPORTED, "the D3Q39 entropic level stores FP32 populations (storage %d)", storage);
  if (!g->d_nbr_ghost || g->h_nbrg.size() != (size_t)g->nb * 27 || g->h_binfo.size() != (size_t)g->nb)
    return set_error(OAL_E_UNSUPPORTED, "the D3Q39 entropic level needs a library-built geometry");
  KbcGeometry G;
  G.nb = g->nb; G.n_ghost = g->n_ghost; G.nx = g->nx; G.ny = g->ny; G.nz = g->nz;
  G.d_nbr = g->d_nbr_ghost; G.h_nbr = g->h_nbrg.data();
  G.d_binfo = g->d_binfo; G.h_bflags = g->h_bflags.data();
  G.d_bflags = g->d_bflags; G.d_mslot = g->d_mslot; G.d_cmask = g->d_cmask;
  G.has_solid = g->n_solid > 0;
  G.d_sponge = g->d_sponge;
  G.d_wdist = g->d_wdist;
  KbcLevel* k = nullptr;
  oal_status s = kbc_create(g->device, G, &k);
  if (s != OAL_OK) return s;
  kbc_set_exact_math(k, (flags & OAL_LEVEL_EXACT_MATH) != 0);
  auto* L = new oal_level();
  L->g = g; L->device = g->device; L->op = OAL_OP_ENTROPIC_D3Q39; L->storage = storage; L->kbc = k;
  ++const_cast<oal_geometry*>(g)->n_levels;
  *out = L;
  return OAL_OK;
}

oal_status oal_level_create(const oal_geometry* g, int32_t op, int32_t storage, oal_level** out) {
  return oal_level_create_ex(g, op, storage, 0u, out);
}

oal_status oal_level_create_ex(const oal_geometry* g, int32_t op, int32_t storage, uint32_t flags, oal_level** out) {
  if (!g || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  *out = nullptr;
  if (op == OAL_OP_ENTROPIC_D3Q39) return create_entropic_level(g, storage, flags, out);
  if (op != OAL_OP_CUMULANT_D3Q27) return set_error(OAL_E_UNSUPPORTED, "operator %d has no level state in this build", op);
  if (storage < OAL_STORE_F32 || storage > OAL_STORE_F64) return set_error(OAL_E_INVALID_ARG, "storage %d", storage);
  OAL_CUDA_TRY(cudaSetDevice(g->device));
  auto* L = new oal_level();
  L->g = g; L->device = g->device; L->op = op; L->storage = storage;
  ++const_cast<oal_geometry*>(g)->n_levels;
  const int64_t ncell = (int64_t)g->nb * 512;
  // box levels in FP32/FP16/BF16: dense padded grid; otherwise the real blocks followed by the
  // ghost blocks
  L->dense = (flags & OAL_LEVEL_DENSE) && g->box && storage != OAL_STORE_F64;
  L->round_nearest = (flags & OAL_LEVEL_ROUND_NEAREST) != 0;
  if (L->dense) {
    oal_status ds = build_dense_tables(const_cast<oal_geometry*>(g));
    if (ds != OAL_OK) { delete L; return ds; }
  }
  if (L->dense) {
    L->PX = 8 * g->bdim[0] + 16;
    L->PY = 8 * g->bdim[1] + 2;
    L->PZ = 8 * g->bdim[2] + 2;
  }
  const size_t fbytes = L->dense ? (size_t)27 * L->PX * L->PY * L->PZ * storage_bytes(storage)
                                 : (size_t)(g->nb + g->n_ghost) * 512 * 27 * storage_bytes(storage);
  const size_t mb = macro_bytes(storage);
  auto fail = [&](cudaError_t e) {
    oal_level_destroy(L);
    return set_error(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "level allocation: %s",
                     cudaGetErrorString(e));
  };
  cudaError_t e;
  for (int i = 0; i < 2; ++i) {
    if ((e = cudaMalloc(&L->f[i], fbytes)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(L->f[i], 0, fbytes)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&L->vel[i], (size_t)ncell * 3 * mb)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(L->vel[i], 0, (size_t)ncell * 3 * mb)) != cudaSuccess) return fail(e);
  }
  if ((e = cudaMalloc(&L->rho, (size_t)ncell * mb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&L->d_force_part, (size_t)g->nb * 4 * 3 * sizeof(double))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&L->d_force, 3 * sizeof(double))) != cudaSuccess) return fail(e);
  if ((e = cudaMemset(L->d_force, 0, 3 * sizeof(double))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&L->d_ticket, sizeof(uint32_t))) != cudaSuccess) return fail(e);
  if ((e = cudaMemset(L->d_ticket, 0, sizeof(uint32_t))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&L->d_mm_part, (size_t)g->nb * 4 * sizeof(double))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&L->d_mm, 4 * sizeof(double))) != cudaSuccess) return fail(e);
  if ((e = cudaStreamCreateWithFlags(&L->cap, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
  // the general kernel's side stream at the highest priority: its few, long CTAs (blocks at solids)
  // start first instead of trailing the uniform kernel's
  int prio_least = 0, prio_greatest = 0;
  if ((e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest)) != cudaSuccess) return fail(e);
  if ((e = cudaStreamCreateWithPriority(&L->ov.side, cudaStreamNonBlocking, prio_greatest)) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&L->ov.fork, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&L->ov.join, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&L->d_err, sizeof(uint32_t))) != cudaSuccess) return fail(e);
  if ((e = cudaMemset(L->d_err, 0, sizeof(uint32_t))) != cudaSuccess) return fail(e);
  if (L->dense) {
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device)) != cudaSuccess) return fail(e);
    int per = 1;
    if (storage == OAL_STORE_F32) per = dense_ctas_per_sm<float>();
    else if (storage == OAL_STORE_F16_DEV) per = dense_ctas_per_sm<__half>();
    else per = dense_ctas_per_sm<__nv_bfloat16>();
    L->dense_grid = sms * per;
  }
  L->bytes = (int64_t)(2 * fbytes + ncell * 7 * mb + g->nb * 16 * 8 + 60);
  *out = L;
  return OAL_OK;
}

static void release_graph(oal_level* L) {
  if (L->gc.exec) cudaGraphExecDestroy(L->gc.exec);
  if (L->gc.graph) cudaGraphDestroy(L->gc.graph);
  L->gc = GraphCache{};
}

void oal_level_destroy(oal_level* L) {
  if (!L) return;
  if (L->kbc) {
    kbc_destroy(L->kbc);
    auto* g = const_cast<oal_geometry*>(L->g);
    delete L;
    if (g && --g->n_levels == 0 && g->destroy_requested) geometry_release(g);
    return;
  }
  cudaSetDevice(L->device);
  release_graph(L);
  bouzidi_free(&L->bz);
  for (int i = 0; i < 2; ++i) { cudaFree(L->f[i]); cudaFree(L->vel[i]); }
  cudaFree(L->rho); cudaFree(L->d_force_part); cudaFree(L->d_force); cudaFree(L->d_mm_part); cudaFree(L->d_mm);
  cudaFree(L->d_ticket); cudaFree(L->pi_neq); cudaFree(L->d_nscbc_blocks);
  cudaFree(L->s_tri); cudaFree(L->s_ptr); cudaFree(L->s_out); cudaFree(L->s_part); cudaFree(L->s_sum);
  if (L->cap) cudaStreamDestroy(L->cap);
  if (L->ov.side) cudaStreamDestroy(L->ov.side);
  if (L->ov.fork) cudaEventDestroy(L->ov.fork);
  if (L->ov.join) cudaEventDestroy(L->ov.join);
  cudaFree(L->d_err);
  cudaGetLastError();  // teardown leaves no error behind for the next call
  auto* g = const_cast<oal_geometry*>(L->g);
  delete L;
  if (g && --g->n_levels == 0 && g->destroy_requested) geometry_release(g);
}

oal_status oal_level_init_equilibrium(oal_level* L, const double* rho, const double* vel, int32_t comp) {
  if (!L || !rho || !vel) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) return kbc_init_equilibrium(L->kbc, rho, vel);
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  const int64_t ncell = (int64_t)L->g->nb * 512;
  double *d_rho = nullptr, *d_vel = nullptr;
  OAL_CUDA_TRY(cudaMalloc(&d_rho, ncell * sizeof(double)));
  cudaError_t e = cudaMalloc(&d_vel, 3 * ncell * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(d_rho, rho, ncell * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_vel, vel, 3 * ncell * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    switch (L->storage) {
      case OAL_STORE_F32: e = init_feq_t<float, float>(L, d_rho, d_vel, comp); break;
      case OAL_STORE_F16_DEV: e = init_feq_t<__half, float>(L, d_rho, d_vel, comp); break;
      case OAL_STORE_BF16_DEV: e = init_feq_t<__nv_bfloat16, float>(L, d_rho, d_vel, comp); break;
      case OAL_STORE_F64: e = init_feq_t<double, double>(L, d_rho, d_vel, comp); break;
    }
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(d_rho); cudaFree(d_vel);
  if (e == cudaSuccess && L->pi_neq) e = cudaMemset(L->pi_neq, 0, (size_t)ncell * 6 * macro_bytes(L->storage));
  if (e != cudaSuccess) return set_error(OAL_E_CUDA, "init_equilibrium: %s", cudaGetErrorString(e));
  L->parity = 0;
  L->forces_valid = false;
  release_graph(L);
  return OAL_OK;
}

oal_status oal_level_set_state(oal_level* L, const double* f, const double* rho, const double* vel) {
  if (!L || !f) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) return kbc_set_state(L->kbc, f, rho, vel);
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  const int64_t ncell = (int64_t)L->g->nb * 512;
  double *d_f = nullptr, *d_r = nullptr, *d_v = nullptr;
  cudaError_t e = cudaMalloc(&d_f, 27 * ncell * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(d_f, f, 27 * ncell * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && rho) {
    e = cudaMalloc(&d_r, ncell * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(d_r, rho, ncell * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && vel) {
    e = cudaMalloc(&d_v, 3 * ncell * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(d_v, vel, 3 * ncell * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) {
    switch (L->storage) {
      case OAL_STORE_F32: e = import_t<float, float>(L, d_f, d_r, d_v); break;
      case OAL_STORE_F16_DEV: e = import_t<__half, float>(L, d_f, d_r, d_v); break;
      case OAL_STORE_BF16_DEV: e = import_t<__nv_bfloat16, float>(L, d_f, d_r, d_v); break;
      case OAL_STORE_F64: e = import_t<double, double>(L, d_f, d_r, d_v); break;
    }
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(d_f); cudaFree(d_r); cudaFree(d_v);
  if (e != cudaSuccess) return set_error(OAL_E_CUDA, "set_state: %s", cudaGetErrorString(e));
  release_graph(L);
  return OAL_OK;
}

oal_status oal_level_get_state(oal_level* L, double* f, double* rho, double* vel) {
  if (!L) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) return kbc_get_state(L->kbc, f, rho, vel);
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  OAL_CUDA_TRY(cudaDeviceSynchronize());
  const int64_t ncell = (int64_t)L->g->nb * 512;
  double *d_f = nullptr, *d_r = nullptr, *d_v = nullptr;
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMalloc(&d_f, 27 * ncell * sizeof(double));
  if (e == cudaSuccess && rho) e = cudaMalloc(&d_r, ncell * sizeof(double));
  if (e == cudaSuccess && vel) e = cudaMalloc(&d_v, 3 * ncell * sizeof(double));
  if (e == cudaSuccess) {
    switch (L->storage) {
      case OAL_STORE_F32: e = export_t<float, float>(L, d_f, d_r, d_v); break;
      case OAL_STORE_F16_DEV: e = export_t<__half, float>(L, d_f, d_r, d_v); break;
      case OAL_STORE_BF16_DEV: e = export_t<__nv_bfloat16, float>(L, d_f, d_r, d_v); break;
      case OAL_STORE_F64: e = export_t<double, double>(L, d_f, d_r, d_v); break;
    }
  }
  if (e == cudaSuccess && f) e = cudaMemcpy(f, d_f, 27 * ncell * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && rho) e = cudaMemcpy(rho, d_r, ncell * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && vel) e = cudaMemcpy(vel, d_v, 3 * ncell * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d_f); cudaFree(d_r); cudaFree(d_v);
  if (e != cudaSuccess) return set_error(OAL_E_CUDA, "get_state: %s", cudaGetErrorString(e));
  return check_level_error(L);
}

static_assert(sizeof(oal_step_params) == 160, "oal_step_params: 40 four-byte scalars");

// The filter strengths of the steps about to be enqueued on L.
static oal_status set_svv(oal_level* L, const oal_step_params* p) {
  L->svv_x = p->svv_x_epsilon;
  L->svv_yz = p->svv_yz_epsilon;
  return OAL_OK;
}

// Enqueue one step of L on st (no host synchronisation).
static oal_status enqueue_step(oal_level* L, const CaseParams& cp, cudaStream_t st) {
  const oal_geometry* g = L->g;
  StepArgs a{};
  fill_geometry_args(g, &a);
  int64_t bst, kst;
  level_layout(L, &bst, &kst);
  const int p = L->parity;
  a.nbr = g->d_nbr_ghost;
  a.n_total_blocks = g->nb + g->n_ghost;
  a.f_in = L->f[p]; a.f_out = L->f[p ^ 1]; a.f_post = nullptr;
  a.rho_out = L->rho; a.vel_out = L->vel[p ^ 1]; a.vel_in = L->vel[p];
  a.f_bstride = bst; a.f_kstride = kst;
  a.v_bstride = 512; a.v_cstride = 512 * (int64_t)g->nb;
  a.force_part = L->d_force_part;
  a.err = L->d_err;
  a.p0 = cp;
  a.flags_any = cp.flags;
  a.round_nearest = L->round_nearest ? 1 : 0;
  a.prefetch_ctas = L->prefetch_ctas;
  a.persistent = L->persistent;
  a.pi_neq = L->pi_neq;
  if ((cp.flags & CF_SGS_PI) && !L->pi_neq) return set_error(OAL_E_UNSUPPORTED, "variable_nu_sgs 1 without its Pi_neq field");
  if (!L->dense) { a.force_out = L->d_force; a.force_ticket = L->d_ticket; }
  a.par = L->par;
  if (L->dense) {
    a.dense = 1;
    a.PX = L->PX; a.PY = L->PY; a.PZ = L->PZ;
    a.f_bstride = 0;
    a.p0.flags |= g->pmask;
    cudaError_t e = cudaErrorInvalidValue;
    switch (L->storage) {
      case OAL_STORE_F32: e = dense_step_t<float, float>(L, a, st); break;
      case OAL_STORE_F16_DEV: e = dense_step_t<__half, float>(L, a, st); break;
      case OAL_STORE_BF16_DEV: e = dense_step_t<__nv_bfloat16, float>(L, a, st); break;
    }
    OAL_CUDA_TRY(e);
  } else {
    OAL_CUDA_TRY(launch_by_storage(L->storage, g, a, PATH_GHOSTED, st, &L->ov));
  }
  const bool svv = L->svv_x > 0.0f || L->svv_yz > 0.0f;
  if (svv) {
    // spectral vanishing viscosity right after the step kernels (timestep.jl:1576-1611)
    const int64_t n_el = L->dense ? 27 * kst : (int64_t)(g->nb + g->n_ghost) * 27 * 512;
    OAL_CUDA_TRY(svv_enqueue(L->storage, a.f_in, a.f_out, pop_index(L), g->nb, n_el, g->d_nbr, g->nb, g->d_mslot,
                             g->d_cmask, L->svv_x, L->svv_yz, st));
  }
  if (L->nscbc.enabled && L->n_nscbc > 0) {
    // characteristic outlet after the step, before the wall corrections (timestep.jl:1617-1664)
    cudaError_t e = cudaErrorInvalidValue;
    switch (L->storage) {
      case OAL_STORE_F32: e = nscbc_t<float, float>(L, a.f_out, a.vel_out, st); break;
      case OAL_STORE_F16_DEV: e = nscbc_t<__half, float>(L, a.f_out, a.vel_out, st); break;
      case OAL_STORE_BF16_DEV: e = nscbc_t<__nv_bfloat16, float>(L, a.f_out, a.vel_out, st); break;
      case OAL_STORE_F64: e = nscbc_t<double, double>(L, a.f_out, a.vel_out, st); break;
    }
    OAL_CUDA_TRY(e);
  }
  if ((cp.flags & CF_BOUZIDI) && L->bz.n > 0)
    OAL_CUDA_TRY(bouzidi_enqueue(L->bz, L->storage, a.f_out, pop_index(L), g->d_nbr, g->d_mslot, g->d_cmask, st));
  if ((cp.flags & CF_SGS_PI) && (((cp.flags & CF_BOUZIDI) && L->bz.n > 0) || (L->nscbc.enabled && L->n_nscbc > 0) || svv)) {
    // the filter, the Bouzidi correction or the outlet rewrote populations after the fused
    // refresh: refresh Pi_neq again from the corrected state (timestep.jl:1818-1834)
    cudaError_t e = cudaErrorInvalidValue;
    switch (L->storage) {
      case OAL_STORE_F32: e = pi_neq_t<float, float, float>(L, p ^ 1, static_cast<float*>(L->pi_neq), st); break;
      case OAL_STORE_F16_DEV: e = pi_neq_t<__half, float, float>(L, p ^ 1, static_cast<float*>(L->pi_neq), st); break;
      case OAL_STORE_BF16_DEV: e = pi_neq_t<__nv_bfloat16, float, float>(L, p ^ 1, static_cast<float*>(L->pi_neq), st); break;
      case OAL_STORE_F64: e = pi_neq_t<double, double, double>(L, p ^ 1, static_cast<double*>(L->pi_neq), st); break;
    }
    OAL_CUDA_TRY(e);
  }
  if (cp.flags & CF_COLLECT) {
    // the momentum exchange lives on the general kernel's CTAs (blocks near solids); in the
    // block layout the last of them sums the partials (a.force_out)
    const bool all_general = (cp.flags & (CF_SGS_PI | CF_SGS_DYNAMIC)) != 0;
    const int64_t n_gen = all_general ? g->nb : g->n_general;
    if (n_gen > 0 && L->dense) {
      k_reduce3<<<1, 256, 0, st>>>(L->d_force_part, n_gen * 4, L->d_force);
      OAL_CUDA_TRY(cudaGetLastError());
    } else if (n_gen == 0) {
      OAL_CUDA_TRY(cudaMemsetAsync(L->d_force, 0, 3 * sizeof(double), st));
    }
    L->forces_valid = true;
  }
  L->parity ^= 1;
  return OAL_OK;
}

oal_status oal_level_step(oal_level* L, const oal_step_params* p, void* stream) {
  if (!L) return set_error(OAL_E_INVALID_ARG, "null level");
  if (L->kbc) return kbc_step(L->kbc, p, stream);
  CaseParams cp;
  oal_status s = resolve_params(p, L->g, &cp);
  if (s != OAL_OK) return s;
  if (cp.flags & CF_STORE_POST) return set_error(OAL_E_UNSUPPORTED, "store_post_collision needs caller-owned arrays (oal_stream_collide)");
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  if ((s = prepare_fill(L, cp, static_cast<cudaStream_t>(stream))) != OAL_OK) return s;
  if ((s = prepare_sgs(L, cp, static_cast<cudaStream_t>(stream))) != OAL_OK) return s;
  if ((s = set_svv(L, p)) != OAL_OK) return s;
  L->comp = (cp.flags & CF_COMPRESSIBLE) != 0;
  return enqueue_step(L, cp, static_cast<cudaStream_t>(stream));
}

oal_status oal_level_advance(oal_level* L, const oal_step_params* p, int32_t n, void* stream) {
  if (!L) return set_error(OAL_E_INVALID_ARG, "null level");
  if (L->kbc) return kbc_advance(L->kbc, p, n, stream);
  if (n <= 0) return set_error(OAL_E_INVALID_ARG, "n_steps must be positive");
  CaseParams cp;
  oal_status s = resolve_params(p, L->g, &cp);
  if (s != OAL_OK) return s;
  if (cp.flags & CF_STORE_POST) return set_error(OAL_E_UNSUPPORTED, "store_post_collision needs caller-owned arrays");
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((s = prepare_fill(L, cp, st)) != OAL_OK) return s;
  if ((s = prepare_sgs(L, cp, st)) != OAL_OK) return s;
  if ((s = set_svv(L, p)) != OAL_OK) return s;
  L->comp = (cp.flags & CF_COMPRESSIBLE) != 0;
  oal_step_params key = *p;
  if (!(cp.flags & CF_INLET_NOISE)) key.time_step_seed = 0;  // the seed only matters with inlet noise
  const bool hit = L->gc.exec && L->gc.n == n && L->gc.parity == L->parity && std::memcmp(&L->gc.p, &key, sizeof key) == 0;
  if (!hit) {
    release_graph(L);
    const int start_parity = L->parity;
    OAL_CUDA_TRY(cudaStreamBeginCapture(L->cap, cudaStreamCaptureModeThreadLocal));
    oal_status es = OAL_OK;
    for (int i = 0; i < n && es == OAL_OK; ++i) {
      CaseParams ci = cp;
      ci.time_step_seed = p->time_step_seed + i;
      es = enqueue_step(L, ci, L->cap);
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(L->cap, &graph);
    L->parity = start_parity;
    if (es != OAL_OK) { if (graph) cudaGraphDestroy(graph); return es; }
    if (e != cudaSuccess) return set_error(OAL_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(graph); return set_error(OAL_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    L->gc.exec = exec; L->gc.graph = graph; L->gc.n = n; L->gc.parity = start_parity; L->gc.p = key;
  }
  OAL_CUDA_TRY(cudaGraphLaunch(L->gc.exec, st));
  if (n & 1) L->parity ^= 1;
  if (cp.flags & CF_COLLECT) L->forces_valid = true;
  return OAL_OK;
}

oal_status oal_level_set_bouzidi(oal_level* L, int32_t n_cells, const int32_t* cell_block, const int32_t* cell_x,
                                 const int32_t* cell_y, const int32_t* cell_z, const uint16_t* q_half,
                                 float q_min_threshold, int32_t ff_fallback, float limiter_rel_cap,
                                 float limiter_abs_cap) {
  if (!L) return set_error(OAL_E_INVALID_ARG, "null level");
  if (L->kbc) return set_error(OAL_E_UNSUPPORTED, "linear Bouzidi walls are a D3Q27 level path");
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  OAL_CUDA_TRY(cudaDeviceSynchronize());  // a step in flight may still read the old set
  release_graph(L);
  ++L->bz_gen;
  return bouzidi_upload(&L->bz, L->storage, L->g->nb, 0, n_cells, cell_block, cell_x, cell_y, cell_z, q_half,
                        q_min_threshold, ff_fallback, limiter_rel_cap, limiter_abs_cap);
}

void oal_default_surface_params(oal_surface_params* sp) {
  if (!sp) return;
  std::memset(sp, 0, sizeof *sp);
  sp->abi_version = OAL_ABI_VERSION;
  sp->search_radius = 8;      // map_surface_stresses! default (surface.jl:1335)
  sp->recover_normal = 1;     // :1336
  sp->tau = 0.6f;
  sp->c_wale = 0.20f;         // C_SMAGO, config_loader.jl:82
  sp->nu_sgs_background = 0.0f;
  sp->pressure_scale = 1.0f;
  sp->stress_scale = 1.0f;
}

oal_status oal_level_set_surface(oal_level* L, int32_t n_tri, const float* tri) {
  if (!L) return set_error(OAL_E_INVALID_ARG, "null level");
  if (n_tri < 0 || (n_tri > 0 && !tri)) return set_error(OAL_E_INVALID_ARG, "n_tri %d", n_tri);
  for (int64_t i = 0; i < (int64_t)n_tri * 7; ++i)
    if (!std::isfinite(tri[i])) return set_error(OAL_E_INVALID_ARG, "triangle value %lld is not finite", (long long)i);
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  OAL_CUDA_TRY(cudaDeviceSynchronize());
  cudaFree(L->s_tri); cudaFree(L->s_out); cudaFree(L->s_part);
  L->s_tri = nullptr; L->s_out = nullptr; L->s_part = nullptr; L->s_n = 0;
  if (n_tri == 0) return OAL_OK;
  const oal_geometry* g = L->g;
  if (!L->s_ptr) {
    // block pointer of the level's block grid (get_cell_at_position, surface.jl:271-307)
    const int dx = g->nx / kBS, dy = g->ny / kBS, dz = g->nz / kBS;
    std::vector<int32_t> ptr((size_t)dx * dy * dz, 0);
    for (int32_t b = 0; b < g->nb; ++b) {
      const int4 bi = g->h_binfo[(size_t)b];
      if (bi.x < 1 || bi.y < 1 || bi.z < 1 || bi.x > dx || bi.y > dy || bi.z > dz)
        return set_error(OAL_E_UNSUPPORTED, "block %d lies outside the level's %dx%dx%d block grid", b, dx, dy, dz);
      ptr[(size_t)(bi.x - 1) + (size_t)dx * ((bi.y - 1) + (size_t)dy * (bi.z - 1))] = b + 1;
    }
    OAL_CUDA_TRY(cudaMalloc(&L->s_ptr, ptr.size() * sizeof(int32_t)));
    OAL_CUDA_TRY(cudaMemcpy(L->s_ptr, ptr.data(), ptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    OAL_CUDA_TRY(cudaMalloc(&L->s_sum, 9 * sizeof(double)));
  }
  OAL_CUDA_TRY(cudaMalloc(&L->s_tri, (size_t)n_tri * 7 * sizeof(float)));
  OAL_CUDA_TRY(cudaMemcpy(L->s_tri, tri, (size_t)n_tri * 7 * sizeof(float), cudaMemcpyHostToDevice));
  OAL_CUDA_TRY(cudaMalloc(&L->s_out, (size_t)n_tri * 6 * sizeof(float)));
  OAL_CUDA_TRY(cudaMalloc(&L->s_part, (size_t)n_tri * 9 * sizeof(double)));
  L->s_n = n_tri;
  return OAL_OK;
}

oal_status oal_level_surface_forces(oal_level* L, const oal_surface_params* sp, double out[9], float* per_tri) {
  if (!L || !sp || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (sp->abi_version != OAL_ABI_VERSION) return set_error(OAL_E_ABI_MISMATCH, "oal_surface_params.abi_version %u", sp->abi_version);
  if (sp->search_radius < 1 || sp->search_radius > 64) return set_error(OAL_E_INVALID_ARG, "search_radius %d (1..64)", sp->search_radius);
  if (!(sp->tau > 0.5f)) return set_error(OAL_E_INVALID_ARG, "tau must exceed 1/2");
  for (int c = 0; c < 9; ++c) out[c] = 0.0;
  if (L->s_n == 0) return OAL_OK;
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  const oal_geometry* g = L->g;
  SurfArgs a{};
  a.tri = L->s_tri; a.n = L->s_n;
  a.rho = L->rho; a.vel = L->vel[L->parity]; a.vcs = (int64_t)g->nb * kCells;
  float cs2 = 1.0f / 3.0f;
  bool f64 = L->storage == OAL_STORE_F64;
  if (L->kbc) {
    // a D3Q39 level: its FP32 macros and the lattice's cs^2 = 2/3 (CS2_PHYSICS)
    void* r = nullptr;
    void* v = nullptr;
    oal_status ks = kbc_device_state(L->kbc, nullptr, &r, &v);
    if (ks != OAL_OK) return ks;
    a.rho = r; a.vel = v;
    cs2 = 2.0f / 3.0f;
    f64 = false;
  }
  a.ptr = L->s_ptr; a.dim_x = g->nx / kBS; a.dim_y = g->ny / kBS; a.dim_z = g->nz / kBS;
  a.mslot = g->d_mslot; a.cmask = g->d_cmask;
  a.radius = sp->search_radius; a.recover = sp->recover_normal ? 1 : 0;
  a.tau = sp->tau; a.c_wale = sp->c_wale; a.nu_bg = sp->nu_sgs_background;
  a.pscale = sp->pressure_scale; a.sscale = sp->stress_scale; a.cs2 = cs2;
  a.mcx = sp->moment_center[0]; a.mcy = sp->moment_center[1]; a.mcz = sp->moment_center[2];
  a.out = L->s_out; a.part = L->s_part;
  OAL_CUDA_TRY(launch_surface(a, f64, L->s_sum, nullptr));
  OAL_CUDA_TRY(cudaMemcpy(out, L->s_sum, 9 * sizeof(double), cudaMemcpyDeviceToHost));
  if (per_tri) OAL_CUDA_TRY(cudaMemcpy(per_tri, L->s_out, (size_t)L->s_n * 6 * sizeof(float), cudaMemcpyDeviceToHost));
  return L->kbc ? OAL_OK : check_level_error(L);
}

oal_status oal_level_get_forces(oal_level* L, double out[3]) {
  if (!L || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) { out[0] = out[1] = out[2] = 0.0; return OAL_OK; }  // no solid cells
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  if (!L->forces_valid) { out[0] = out[1] = out[2] = 0.0; return check_level_error(L); }
  OAL_CUDA_TRY(cudaMemcpy(out, L->d_force, 3 * sizeof(double), cudaMemcpyDeviceToHost));
  return check_level_error(L);
}

oal_status oal_level_get_forces_async(oal_level* L, double* host_out3, void* stream) {
  if (!L || !host_out3) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) { host_out3[0] = host_out3[1] = host_out3[2] = 0.0; return OAL_OK; }
  OAL_CUDA_TRY(cudaMemcpyAsync(host_out3, L->d_force, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                               static_cast<cudaStream_t>(stream)));
  return OAL_OK;
}

oal_status oal_level_mass_momentum(oal_level* L, double out[4]) {
  if (!L || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) return kbc_mass_momentum(L->kbc, out);
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  cudaError_t e = cudaSuccess;
  switch (L->storage) {
    case OAL_STORE_F32: e = mm_t<float, float>(L); break;
    case OAL_STORE_F16_DEV: e = mm_t<__half, float>(L); break;
    case OAL_STORE_BF16_DEV: e = mm_t<__nv_bfloat16, float>(L); break;
    case OAL_STORE_F64: e = mm_t<double, double>(L); break;
  }
  if (e != cudaSuccess) return set_error(OAL_E_CUDA, "mass_momentum: %s", cudaGetErrorString(e));
  OAL_CUDA_TRY(cudaMemcpy(out, L->d_mm, 4 * sizeof(double), cudaMemcpyDeviceToHost));
  return check_level_error(L);
}

oal_status oal_level_pi_neq(oal_level* L, float* out) {
  if (!L || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) return set_error(OAL_E_UNSUPPORTED, "oal_level_pi_neq: D3Q27 levels");
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  const int64_t ncell = (int64_t)L->g->nb * 512;
  float* d_out = nullptr;
  OAL_CUDA_TRY(cudaMalloc(&d_out, (size_t)ncell * 6 * sizeof(float)));
  cudaError_t e = cudaErrorInvalidValue;
  switch (L->storage) {
    case OAL_STORE_F32: e = pi_neq_t<float, float, float>(L, L->parity, d_out, 0); break;
    case OAL_STORE_F16_DEV: e = pi_neq_t<__half, float, float>(L, L->parity, d_out, 0); break;
    case OAL_STORE_BF16_DEV: e = pi_neq_t<__nv_bfloat16, float, float>(L, L->parity, d_out, 0); break;
    case OAL_STORE_F64: e = pi_neq_t<double, double, float>(L, L->parity, d_out, 0); break;
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d_out, (size_t)ncell * 6 * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  if (e != cudaSuccess) return set_error(OAL_E_CUDA, "pi_neq: %s", cudaGetErrorString(e));
  return OAL_OK;
}

// ---- launch tuning and the autotuner --------------------------------------------------------
}  // extern "C"

// Device copies of a level's or pool's state buffers: the autotuner restores them between
// candidates, so that tuning leaves the simulation where it was.
struct StateSnapshot {
  std::vector<void*> live, copy;
  std::vector<size_t> bytes;
  cudaError_t add(void* p, size_t n) {
    if (!p || !n) return cudaSuccess;
    void* c = nullptr;
    cudaError_t e = cudaMalloc(&c, n);
    if (e != cudaSuccess) return e;
    live.push_back(p); copy.push_back(c); bytes.push_back(n);
    return cudaMemcpy(c, p, n, cudaMemcpyDeviceToDevice);
  }
  cudaError_t restore() const {
    for (size_t i = 0; i < live.size(); ++i) {
      cudaError_t e = cudaMemcpy(live[i], copy[i], bytes[i], cudaMemcpyDeviceToDevice);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  ~StateSnapshot() { for (void* c : copy) cudaFree(c); }
};

// The settings the autotuner tries: the plain and the persistent launch, each with the prefetch
// distances {0, 4, 8, 16} x the SM count of the device.
static cudaError_t tune_candidates(int device, int64_t* cand, int32_t* pers) {
  int nsm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  const int64_t mult[4] = {0, 4, 8, 16};
  for (int c = 0; c < OAL_TUNE_CANDIDATES; ++c) {
    cand[c] = mult[c % 4] * nsm;
    pers[c] = c / 4;
  }
  return e;
}

// Times `run` (n steps) once untimed, then once between two events on `st`, after `reset`.
template <class Run, class Reset>
static oal_status time_candidate(Run run, Reset reset, int32_t n, cudaStream_t st, double* ms) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  OAL_CUDA_TRY(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  oal_status s = ce == cudaSuccess ? OAL_OK : set_error(OAL_E_CUDA, "autotune: %s", cudaGetErrorString(ce));
  if (s == OAL_OK) s = reset();
  if (s == OAL_OK) s = run(st);
  if (s == OAL_OK && (ce = cudaStreamSynchronize(st)) != cudaSuccess) s = set_error(OAL_E_CUDA, "autotune: %s", cudaGetErrorString(ce));
  if (s == OAL_OK) s = reset();
  if (s == OAL_OK && (ce = cudaEventRecord(e0, st)) != cudaSuccess) s = set_error(OAL_E_CUDA, "autotune: %s", cudaGetErrorString(ce));
  if (s == OAL_OK) s = run(st);
  if (s == OAL_OK && (ce = cudaEventRecord(e1, st)) != cudaSuccess) s = set_error(OAL_E_CUDA, "autotune: %s", cudaGetErrorString(ce));
  if (s == OAL_OK && (ce = cudaEventSynchronize(e1)) != cudaSuccess) s = set_error(OAL_E_CUDA, "autotune: %s", cudaGetErrorString(ce));
  float t = 0.0f;
  if (s == OAL_OK && (ce = cudaEventElapsedTime(&t, e0, e1)) != cudaSuccess) s = set_error(OAL_E_CUDA, "autotune: %s", cudaGetErrorString(ce));
  *ms = (double)t / n;
  cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return s;
}

extern "C" {

void oal_default_nscbc_params(oal_nscbc_params* np) {
  if (!np) return;
  std::memset(np, 0, sizeof *np);
  np->enabled = 0;          // OUTLET_NSCBC_ENABLED, config_loader.jl:751
  np->p_target = 1.0f;      // :752
  np->sigma_relax = 0.27f;  // :753
  np->neq_blend = 0.5f;     // :754
}

oal_status oal_level_set_nscbc(oal_level* L, const oal_nscbc_params* np) {
  if (!L || !np) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) return set_error(OAL_E_UNSUPPORTED, "the characteristic outlet is built for D3Q27 levels");
  if (L->par.ptr) return set_error(OAL_E_UNSUPPORTED, "the characteristic outlet acts on the coarsest level only");
  if (np->enabled && !(np->sigma_relax >= 0.0f && std::isfinite(np->p_target) && std::isfinite(np->neq_blend)))
    return set_error(OAL_E_INVALID_ARG, "nscbc: sigma_relax >= 0 and finite p_target, neq_blend");
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  std::vector<int32_t> list;
  if (np->enabled) {
    const oal_geometry* g = L->g;
    int32_t bxmax = 0;
    for (const int4& bi : g->h_binfo) bxmax = std::max(bxmax, bi.x);
    for (int32_t b = 0; b < g->nb; ++b)
      if (np->all_blocks || g->h_binfo[(size_t)b].x == bxmax) list.push_back(b);
  }
  cudaFree(L->d_nscbc_blocks);
  L->d_nscbc_blocks = nullptr;
  L->n_nscbc = 0;
  if (!list.empty()) {
    OAL_CUDA_TRY(cudaMalloc(&L->d_nscbc_blocks, list.size() * sizeof(int32_t)));
    OAL_CUDA_TRY(cudaMemcpy(L->d_nscbc_blocks, list.data(), list.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    L->n_nscbc = (int32_t)list.size();
  }
  L->nscbc = *np;
  release_graph(L);  // the captured steps hold the old setting
  return OAL_OK;
}

oal_status oal_level_set_tuning(oal_level* L, int32_t key, int64_t value) {
  if (!L) return set_error(OAL_E_INVALID_ARG, "null level");
  int32_t* slot = key == OAL_TUNE_PREFETCH_CTAS ? &L->prefetch_ctas : key == OAL_TUNE_PERSISTENT ? &L->persistent : nullptr;
  if (!slot) return set_error(OAL_E_INVALID_ARG, "unknown tuning key %d", key);
  if (value < 0 || value > (key == OAL_TUNE_PERSISTENT ? 1 : (1 << 24)))
    return set_error(OAL_E_INVALID_ARG, "tuning key %d: value %lld", key, (long long)value);
  if (*slot != (int32_t)value) {
    *slot = (int32_t)value;
    release_graph(L);  // the captured launches hold the old value
  }
  return OAL_OK;
}

oal_status oal_level_get_tuning(const oal_level* L, int32_t key, int64_t* value) {
  if (!L || !value) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (key == OAL_TUNE_PREFETCH_CTAS) *value = L->prefetch_ctas;
  else if (key == OAL_TUNE_PERSISTENT) *value = L->persistent;
  else return set_error(OAL_E_INVALID_ARG, "unknown tuning key %d", key);
  return OAL_OK;
}

oal_status oal_level_autotune(oal_level* L, const oal_step_params* p, int32_t n_steps, int64_t* prefetch,
                              int32_t* persistent, double* ms_per_step) {
  if (!L || !p) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (n_steps <= 0) return set_error(OAL_E_INVALID_ARG, "n_steps must be positive");
  if (L->kbc) return set_error(OAL_E_UNSUPPORTED, "autotune: D3Q27 levels (the D3Q39 kernel has no tuning key)");
  OAL_CUDA_TRY(cudaSetDevice(L->g->device));
  OAL_CUDA_TRY(cudaDeviceSynchronize());
  const oal_geometry* g = L->g;
  const size_t ncell = (size_t)g->nb * 512, mb = macro_bytes(L->storage);
  const size_t fbytes = L->dense ? (size_t)27 * L->PX * L->PY * L->PZ * storage_bytes(L->storage)
                                 : (size_t)(g->nb + g->n_ghost) * 512 * 27 * storage_bytes(L->storage);
  StateSnapshot snap;
  cudaError_t e = snap.add(L->f[L->parity], fbytes);
  if (e == cudaSuccess) e = snap.add(L->vel[L->parity], ncell * 3 * mb);
  if (e == cudaSuccess) e = snap.add(L->rho, ncell * mb);
  if (e == cudaSuccess) e = snap.add(L->pi_neq, ncell * 6 * mb);
  if (e != cudaSuccess)
    return set_error(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "autotune snapshot: %s", cudaGetErrorString(e));
  int64_t cand[OAL_TUNE_CANDIDATES];
  int32_t pers[OAL_TUNE_CANDIDATES];
  OAL_CUDA_TRY(tune_candidates(L->g->device, cand, pers));
  const int parity0 = L->parity;
  const int32_t keep = L->prefetch_ctas, keep_p = L->persistent;
  cudaStream_t st = nullptr;
  OAL_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  oal_status s = OAL_OK;
  double best = 0.0;
  int best_c = -1;
  for (int c = 0; c < OAL_TUNE_CANDIDATES && s == OAL_OK; ++c) {
    if ((s = oal_level_set_tuning(L, OAL_TUNE_PREFETCH_CTAS, cand[c])) != OAL_OK) break;
    if ((s = oal_level_set_tuning(L, OAL_TUNE_PERSISTENT, pers[c])) != OAL_OK) break;
    double ms = 0.0;
    s = time_candidate([&](cudaStream_t q) { return oal_level_advance(L, p, n_steps, q); },
                       [&]() -> oal_status {
                         cudaError_t re = snap.restore();
                         L->parity = parity0;
                         return re == cudaSuccess ? OAL_OK : set_error(OAL_E_CUDA, "autotune restore: %s", cudaGetErrorString(re));
                       },
                       n_steps, st, &ms);
    if (prefetch) prefetch[c] = cand[c];
    if (persistent) persistent[c] = pers[c];
    if (ms_per_step) ms_per_step[c] = ms;
    if (s == OAL_OK && (best_c < 0 || ms < best)) { best = ms; best_c = c; }
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cudaError_t re = snap.restore();
  L->parity = parity0;
  L->forces_valid = false;
  oal_level_set_tuning(L, OAL_TUNE_PREFETCH_CTAS, s == OAL_OK && best_c >= 0 ? cand[best_c] : keep);
  oal_level_set_tuning(L, OAL_TUNE_PERSISTENT, s == OAL_OK && best_c >= 0 ? pers[best_c] : keep_p);
  if (s != OAL_OK) return s;
  if (re != cudaSuccess) return set_error(OAL_E_CUDA, "autotune restore: %s", cudaGetErrorString(re));
  return OAL_OK;
}

oal_status oal_level_device_state(oal_level* L, void** f, void** rho, void** vel) {
  if (!L) return set_error(OAL_E_INVALID_ARG, "null level");
  if (L->kbc) return kbc_device_state(L->kbc, f, rho, vel);
  if (f) *f = L->f[L->parity];
  if (rho) *rho = L->rho;
  if (vel) *vel = L->vel[L->parity];
  return OAL_OK;
}

int64_t oal_level_device_bytes(const oal_level* L) { return L ? (L->kbc ? kbc_device_bytes(L->kbc) : L->bytes) : 0; }

oal_status oal_level_entropic_lambda(oal_level* L, float* get_host, const float* set_host) {
  if (!L) return set_error(OAL_E_INVALID_ARG, "null level");
  if (!L->kbc) return set_error(OAL_E_INVALID_ARG, "not a D3Q39 entropic level");
  return kbc_lambda(L->kbc, get_host, set_host);
}

oal_status oal_level_layout(const oal_level* L, int64_t out[6]) {
  if (!L || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (L->kbc) return kbc_layout(L->kbc, out);
  int64_t bst, kst;
  level_layout(L, &bst, &kst);
  out[0] = L->dense ? 1 : 0; out[1] = L->PX; out[2] = L->PY; out[3] = L->PZ; out[4] = bst; out[5] = kst;
  return OAL_OK;
}

}  // extern "C"

// ================================================================================================
// Block AMR: a hierarchy of D3Q27 levels with 2:1 refinement in space and time
// (recursive_step! / recursive_step_temporal!, src/solver/solver_control.jl:55-560, default flags)
// ================================================================================================
struct AmrLevel {
  oal_level* L = nullptr;
  const oal_geometry* g = nullptr;
  int32_t dim[3] = {0, 0, 0};
  int32_t* d_ptr = nullptr;       // block pointer [dim_x*dim_y*dim_z], x fastest, 1-based
  int32_t* d_covered = nullptr;   // this level's blocks that have children
  int32_t n_covered = 0;
  void* d_f_old = nullptr;        // snapshot before the level's step (levels with children)
  void* d_rho_old = nullptr;
  void* d_vel_old = nullptr;
  // refined levels: the parent nodes their interpolation stencils touch, evaluated once per substep
  int32_t* d_nodes = nullptr;     // parent cell ids (block * 512 + cell)
  int32_t n_nodes = 0;
  int32_t* d_node_map = nullptr;  // [parent cells] -> record index, -1
  void* d_node_vals = nullptr;    // [n_nodes * 32] compute type
  // interpolation positions: the ghost cells whose pulls interpolate from the parent
  int32_t n_pos = 0;
  int4* d_pos_xyz = nullptr;      // fine global coordinates of each position
  int32_t* d_slot_pos = nullptr;  // [ghost blocks * 512] -> position, -1
  int32_t* d_pos_nodes = nullptr; // [n_pos * 64] stencil records, -1 = absent parent cell
  void* d_pos_macro = nullptr;    // [n_pos * 4] compute type
};

struct oal_amr {
  int device = 0;
  int32_t storage = 0;
  std::vector<AmrLevel> lv;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  int32_t g_n = 0;
  int g_parity = -1;
  std::vector<oal_step_params> g_p;
  std::vector<uint32_t> g_bz;  // the levels' Bouzidi generations the graph was captured with
};

static void amr_release_graph(oal_amr* A) {
  if (A->exec) cudaGraphExecDestroy(A->exec);
  if (A->graph) cudaGraphDestroy(A->graph);
  A->exec = nullptr; A->graph = nullptr; A->g_n = 0; A->g_parity = -1; A->g_p.clear();
}

template <class R>
static double restrict_ratio(R tau_p, R tau_c, int physical) {
  const R tpc = std::max(tau_p - R(0.5), R(1e-6)), tcc = std::max(tau_c - R(0.5), R(1e-6));
  R r = std::min(std::max(tpc / tcc, R(0.01)), R(100));
  if (physical == 1) r = std::min(std::max(R(2) * tau_p / std::max(tau_c, R(0.500001)), R(0.01)), R(100));
  const R omega_p = R(1) / std::max(tau_p, R(0.500001)), omega_c = R(1) / std::max(tau_c, R(0.500001));
  const R one_m_wp = R(1) - omega_p, one_m_wc = R(1) - omega_c;
  if (std::fabs(one_m_wc) > R(1e-6)) r = std::min(std::max(r * (one_m_wp / one_m_wc), R(0.01)), R(100));
  return (double)r;
}

// One step of level l (0-based) and, recursively, two substeps of each finer level, then the
// restriction onto l. t_sub: the level's step index (noise seed); tw: temporal weight of l's parent.
static oal_status amr_step(oal_amr* A, int l, const std::vector<CaseParams>& cps, const oal_step_params* P,
                           int64_t t_sub, double tw, cudaStream_t st) {
  AmrLevel& me = A->lv[(size_t)l];
  oal_level* L = me.L;
  const oal_geometry* g = me.g;
  const bool has_children = l + 1 < (int)A->lv.size();
  const size_t sb = storage_bytes(A->storage), mb = macro_bytes(A->storage);
  const size_t ncell = (size_t)g->nb * 512;
  if (has_children) {  // copy_to_old! (src/geometry/blocks.jl:604-640)
    const int p = L->parity;
    OAL_CUDA_TRY(cudaMemcpyAsync(me.d_f_old, L->f[p], ncell * 27 * sb, cudaMemcpyDeviceToDevice, st));
    OAL_CUDA_TRY(cudaMemcpyAsync(me.d_rho_old, L->rho, ncell * mb, cudaMemcpyDeviceToDevice, st));
    OAL_CUDA_TRY(cudaMemcpyAsync(me.d_vel_old, L->vel[p], ncell * 3 * mb, cudaMemcpyDeviceToDevice, st));
  }
  if (l > 0) {
    const AmrLevel& pa = A->lv[(size_t)l - 1];
    ParentView v{};
    v.f_new = pa.L->f[pa.L->parity];
    v.f_old = pa.d_f_old;
    v.rho_new = pa.L->rho;
    v.rho_old = pa.d_rho_old;
    v.vel_new = pa.L->vel[pa.L->parity];
    v.vel_old = pa.d_vel_old;
    v.ptr = pa.d_ptr;
    v.dim_x = pa.dim[0]; v.dim_y = pa.dim[1]; v.dim_z = pa.dim[2];
    v.nb = pa.g->nb;
    v.tau_parent = P[l - 1].tau;
    v.tau_fine = P[l].tau;
    v.tw = tw;
    v.use_temporal = 1;  // TEMPORAL_INTERPOLATION (config_loader.jl:90)
    v.level_visc_physical = P[l].level_visc_physical;
    v.node_map = me.d_node_map;
    v.node_vals = me.d_node_vals;
    v.slot_pos = me.n_pos > 0 ? me.d_slot_pos : nullptr;
    v.pos_nodes = me.d_pos_nodes;
    v.pos_macro = me.d_pos_macro;
    v.n_pos = me.n_pos;
    v.n_real = me.g->nb;
    L->par = v;
    if (me.n_nodes > 0) {
      cudaError_t e = cudaErrorInvalidValue;
      const int32_t comp = P[l].compressible_corr;
      switch (A->storage) {
        case OAL_STORE_F32: e = launch_parent_nodes<float, float>(v, me.d_nodes, me.n_nodes, me.d_node_vals, comp, st); break;
        case OAL_STORE_F16_DEV: e = launch_parent_nodes<__half, float>(v, me.d_nodes, me.n_nodes, me.d_node_vals, comp, st); break;
        case OAL_STORE_BF16_DEV: e = launch_parent_nodes<__nv_bfloat16, float>(v, me.d_nodes, me.n_nodes, me.d_node_vals, comp, st); break;
        case OAL_STORE_F64: e = launch_parent_nodes<double, double>(v, me.d_nodes, me.n_nodes, me.d_node_vals, comp, st); break;
      }
      OAL_CUDA_TRY(e);
      if (me.n_pos > 0) {
        e = A->storage == OAL_STORE_F64 ? launch_parent_positions<double>(v, me.d_pos_xyz, me.n_pos, me.d_pos_macro, st)
                                        : launch_parent_positions<float>(v, me.d_pos_xyz, me.n_pos, me.d_pos_macro, st);
        OAL_CUDA_TRY(e);
      }
    }
  }
  CaseParams cp = cps[(size_t)l];
  cp.time_step_seed = (int32_t)(P[l].time_step_seed + t_sub);
  oal_status s = enqueue_step(L, cp, st);
  if (s != OAL_OK) return s;
  if (has_children) {
    const double bias = 0.0;  // INTERFACE_TEMPORAL_WEIGHT_BIAS (config_loader.jl:146)
    s = amr_step(A, l + 1, cps, P, 2 * t_sub, std::min(std::max(0.0 + bias, 0.0), 1.0), st);
    if (s != OAL_OK) return s;
    s = amr_step(A, l + 1, cps, P, 2 * t_sub + 1, std::min(std::max(0.5 + bias, 0.0), 1.0), st);
    if (s != OAL_OK) return s;
    // restrict_fine_to_parent! (amr_coupling.jl:7562-7640)
    const AmrLevel& ch = A->lv[(size_t)l + 1];
    RestrictArgs r{};
    r.pf = L->f[L->parity];
    r.prho = L->rho;
    r.pvel = L->vel[L->parity];
    r.pbinfo = g->d_binfo;
    r.covered = me.d_covered;
    r.n_covered = me.n_covered;
    r.pnb = g->nb;
    r.cf = ch.L->f[ch.L->parity];
    r.cptr = ch.d_ptr;
    r.cdx = ch.dim[0]; r.cdy = ch.dim[1]; r.cdz = ch.dim[2];
    r.cbflags = ch.g->d_bflags;
    r.cmslot = ch.g->d_mslot;
    r.ccmask = ch.g->d_cmask;
    r.comp = P[l].compressible_corr;
    cudaError_t e = cudaErrorInvalidValue;
    switch (A->storage) {
      case OAL_STORE_F32:
        r.ratio = restrict_ratio<float>(P[l].tau, P[l + 1].tau, P[l].level_visc_physical);
        e = launch_restrict<float, float>(r, st); break;
      case OAL_STORE_F16_DEV:
        r.ratio = restrict_ratio<float>(P[l].tau, P[l + 1].tau, P[l].level_visc_physical);
        e = launch_restrict<__half, float>(r, st); break;
      case OAL_STORE_BF16_DEV:
        r.ratio = restrict_ratio<float>(P[l].tau, P[l + 1].tau, P[l].level_visc_physical);
        e = launch_restrict<__nv_bfloat16, float>(r, st); break;
      case OAL_STORE_F64:
        r.ratio = restrict_ratio<double>((double)P[l].tau, (double)P[l + 1].tau, P[l].level_visc_physical);
        e = launch_restrict<double, double>(r, st); break;
    }
    OAL_CUDA_TRY(e);
  }
  return OAL_OK;
}

extern "C" {

void oal_amr_destroy(oal_amr* A) {
  if (!A) return;
  cudaSetDevice(A->device);
  amr_release_graph(A);
  for (AmrLevel& l : A->lv) {
    if (l.L) oal_level_destroy(l.L);
    cudaFree(l.d_ptr); cudaFree(l.d_covered); cudaFree(l.d_f_old); cudaFree(l.d_rho_old); cudaFree(l.d_vel_old);
    cudaFree(l.d_nodes); cudaFree(l.d_node_map); cudaFree(l.d_node_vals);
    cudaFree(l.d_pos_xyz); cudaFree(l.d_slot_pos); cudaFree(l.d_pos_nodes); cudaFree(l.d_pos_macro);
  }
  if (A->cap) cudaStreamDestroy(A->cap);
  cudaGetLastError();
  delete A;
}

oal_status oal_amr_create(int32_t nlevels, const oal_amr_level_desc* levels, int32_t storage, oal_amr** out) {
  if (!out || !levels || nlevels < 1) return set_error(OAL_E_INVALID_ARG, "oal_amr_create: bad arguments");
  *out = nullptr;
  if (storage < OAL_STORE_F32 || storage > OAL_STORE_F64) return set_error(OAL_E_INVALID_ARG, "storage %d", storage);
  const int device = levels[0].geometry ? levels[0].geometry->device : 0;
  for (int l = 0; l < nlevels; ++l) {
    const oal_geometry* g = levels[l].geometry;
    const int32_t* d = levels[l].dim;
    if (!g) return set_error(OAL_E_INVALID_ARG, "level %d has no geometry", l);
    if (g->device != device) return set_error(OAL_E_INVALID_ARG, "levels on different devices");
    if (d[0] < 1 || d[1] < 1 || d[2] < 1) return set_error(OAL_E_INVALID_ARG, "level %d: block grid extent", l);
    if (g->nx != 8 * d[0] || g->ny != 8 * d[1] || g->nz != 8 * d[2])
      return set_error(OAL_E_INVALID_ARG, "level %d: geometry extent %dx%dx%d is not 8 x the block grid %dx%dx%d", l,
                       g->nx, g->ny, g->nz, d[0], d[1], d[2]);
    for (int32_t b = 0; b < g->nb; ++b) {
      const int4 c = g->h_binfo[(size_t)b];
      if (c.x < 1 || c.y < 1 || c.z < 1 || c.x > d[0] || c.y > d[1] || c.z > d[2])
        return set_error(OAL_E_INVALID_ARG, "level %d: block %d at (%d,%d,%d) outside the block grid", l, b, c.x, c.y, c.z);
    }
    if (l > 0) {
      const int32_t* pd = levels[l - 1].dim;
      if (d[0] != 2 * pd[0] || d[1] != 2 * pd[1] || d[2] != 2 * pd[2])
        return set_error(OAL_E_INVALID_ARG, "level %d: block grid must be twice its parent's", l);
    }
  }
  OAL_CUDA_TRY(cudaSetDevice(device));
  auto* A = new oal_amr();
  A->device = device;
  A->storage = storage;
  A->lv.resize((size_t)nlevels);
  auto fail = [&](oal_status s) { oal_amr_destroy(A); return s; };
  // host block pointers (x fastest) and the nesting check
  std::vector<std::vector<int32_t>> ptrs((size_t)nlevels);
  for (int l = 0; l < nlevels; ++l) {
    const oal_geometry* g = levels[l].geometry;
    const int32_t* d = levels[l].dim;
    std::vector<int32_t>& ptr = ptrs[(size_t)l];
    ptr.assign((size_t)d[0] * d[1] * d[2], 0);
    for (int32_t b = 0; b < g->nb; ++b) {
      const int4 c = g->h_binfo[(size_t)b];
      int32_t& slot = ptr[(size_t)(c.x - 1) + (size_t)d[0] * ((c.y - 1) + (size_t)d[1] * (c.z - 1))];
      if (slot != 0) { set_error(OAL_E_INVALID_ARG, "level %d: two blocks at (%d,%d,%d)", l, c.x, c.y, c.z); return fail(OAL_E_INVALID_ARG); }
      slot = b + 1;
    }
    if (l > 0) {
      const int32_t* pd = levels[l - 1].dim;
      const std::vector<int32_t>& pp = ptrs[(size_t)l - 1];
      for (int32_t b = 0; b < g->nb; ++b) {
        const int4 c = g->h_binfo[(size_t)b];
        const int px = (c.x + 1) / 2, py = (c.y + 1) / 2, pz = (c.z + 1) / 2;
        if (pp[(size_t)(px - 1) + (size_t)pd[0] * ((py - 1) + (size_t)pd[1] * (pz - 1))] == 0) {
          set_error(OAL_E_INVALID_ARG, "level %d: block (%d,%d,%d) lies outside its parent level", l, c.x, c.y, c.z);
          return fail(OAL_E_INVALID_ARG);
        }
      }
    }
  }
  for (int l = 0; l < nlevels; ++l) {
    AmrLevel& me = A->lv[(size_t)l];
    me.g = levels[l].geometry;
    std::memcpy(me.dim, levels[l].dim, sizeof me.dim);
    oal_status s = oal_level_create_ex(me.g, OAL_OP_CUMULANT_D3Q27, storage, 0u, &me.L);
    if (s != OAL_OK) return fail(s);
    const std::vector<int32_t>& ptr = ptrs[(size_t)l];
    cudaError_t e = cudaMalloc(&me.d_ptr, ptr.size() * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemcpy(me.d_ptr, ptr.data(), ptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && l + 1 < nlevels) {
      // blocks with children: the covered band of the restriction (_restrict_covered_block_list)
      const oal_geometry* cg = levels[l + 1].geometry;
      std::vector<uint8_t> has((size_t)me.g->nb, 0);
      for (int32_t b = 0; b < cg->nb; ++b) {
        const int4 c = cg->h_binfo[(size_t)b];
        const int px = (c.x + 1) / 2, py = (c.y + 1) / 2, pz = (c.z + 1) / 2;
        has[(size_t)ptr[(size_t)(px - 1) + (size_t)me.dim[0] * ((py - 1) + (size_t)me.dim[1] * (pz - 1))] - 1] = 1;
      }
      std::vector<int32_t> cov;
      for (int32_t b = 0; b < me.g->nb; ++b)
        if (has[(size_t)b]) cov.push_back(b);
      me.n_covered = (int32_t)cov.size();
      e = cudaMalloc(&me.d_covered, std::max<size_t>(cov.size(), 1) * sizeof(int32_t));
      if (e == cudaSuccess && !cov.empty())
        e = cudaMemcpy(me.d_covered, cov.data(), cov.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      const size_t ncell = (size_t)me.g->nb * 512;
      if (e == cudaSuccess) e = cudaMalloc(&me.d_f_old, ncell * 27 * storage_bytes(storage));
      if (e == cudaSuccess) e = cudaMalloc(&me.d_rho_old, ncell * macro_bytes(storage));
      if (e == cudaSuccess) e = cudaMalloc(&me.d_vel_old, ncell * 3 * macro_bytes(storage));
    }
    if (e == cudaSuccess && l > 0) {
      // parent nodes of every interpolation stencil this level's ghost pulls can use: the 4x4x4
      // parent cells around the bracket of each pull source inside the domain (and of the z-wall
      // slip image of sources beyond the z faces)
      const oal_geometry* g = me.g;
      const AmrLevel& pa = A->lv[(size_t)l - 1];
      const std::vector<int32_t>& pptr = ptrs[(size_t)l - 1];
      const int pnx = pa.dim[0] * 8, pny = pa.dim[1] * 8, pnz = pa.dim[2] * 8;
      std::vector<int32_t> map((size_t)pa.g->nb * 512, -1);
      std::vector<int32_t> nodes;
      auto bracket = [](double p, int n) {
        if (n <= 1) return 1;
        const double pc = std::min(std::max(p, 1.0), (double)n);
        return std::min(std::max((int)std::floor(pc), 1), n - 1);
      };
      auto add_stencil = [&](int fgx, int fgy, int fgz) {
        const int px0 = bracket(fgx * 0.5 + 0.25, pnx), py0 = bracket(fgy * 0.5 + 0.25, pny),
                  pz0 = bracket(fgz * 0.5 + 0.25, pnz);
        for (int a = -1; a <= 2; ++a)
          for (int b2 = -1; b2 <= 2; ++b2)
            for (int c2 = -1; c2 <= 2; ++c2) {
              const int gx = px0 + a, gy = py0 + b2, gz = pz0 + c2;
              if (gx < 1 || gy < 1 || gz < 1) continue;
              const int bx = (gx - 1) / 8 + 1, by = (gy - 1) / 8 + 1, bz = (gz - 1) / 8 + 1;
              if (bx > pa.dim[0] || by > pa.dim[1] || bz > pa.dim[2]) continue;
              const int32_t pb = pptr[(size_t)(bx - 1) + (size_t)pa.dim[0] * ((by - 1) + (size_t)pa.dim[1] * (bz - 1))];
              if (pb <= 0) continue;
              const int32_t cid = (pb - 1) * 512 + (((gx - 1) % 8) | (((gy - 1) % 8) << 3) | (((gz - 1) % 8) << 6));
              if (map[(size_t)cid] < 0) { map[(size_t)cid] = (int32_t)nodes.size(); nodes.push_back(cid); }
            }
      };
      // interpolation positions: every ghost cell that an in-domain pull reads (its slot in the
      // ghost blocks), with the record of each of its 64 stencil nodes
      std::vector<int32_t> slot_pos((size_t)std::max(g->n_ghost, 1) * 512, -1);
      std::vector<int4> pos_xyz;
      for (const uint2& en : g->h_gentries) {
        const int4 bi = g->h_binfo[en.x];
        const int cell = (int)(en.y & 511u), k = (int)((en.y >> 9) & 31u);
        const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
        const int gx = (bi.x - 1) * 8 + x + 1, gy = (bi.y - 1) * 8 + y + 1, gz = (bi.z - 1) * 8 + z + 1;
        const int sx = gx - q27_cx(k), sy = gy - q27_cy(k), sz = gz - q27_cz(k);
        const bool in_x = sx >= 1 && sx <= g->nx, in_y = sy >= 1 && sy <= g->ny, in_z = sz >= 1 && sz <= g->nz;
        if (in_x && in_y && in_z) {
          add_stencil(sx, sy, sz);
          const int lx = x - q27_cx(k), ly = y - q27_cy(k), lz = z - q27_cz(k);
          const int ox = lx < 0 ? -1 : (lx > 7 ? 1 : 0), oy = ly < 0 ? -1 : (ly > 7 ? 1 : 0),
                    oz = lz < 0 ? -1 : (lz > 7 ? 1 : 0);
          const int32_t gb = g->h_nbrg[(size_t)en.x * 27 + nbr_dir(ox, oy, oz)];
          if (gb >= g->nb && gb < g->nb + g->n_ghost) {
            const size_t slot = (size_t)(gb - g->nb) * 512 + ((lx & 7) | ((ly & 7) << 3) | ((lz & 7) << 6));
            if (slot_pos[slot] < 0) { slot_pos[slot] = (int32_t)pos_xyz.size(); pos_xyz.push_back(make_int4(sx, sy, sz, 0)); }
          }
        } else if (in_x && in_y && !in_z) {
          add_stencil(sx, sy, gz);
        }
      }
      std::vector<int32_t> pos_nodes(pos_xyz.size() * 64, -1);
      for (size_t i = 0; i < pos_xyz.size(); ++i) {
        const int px0 = bracket(pos_xyz[i].x * 0.5 + 0.25, pnx), py0 = bracket(pos_xyz[i].y * 0.5 + 0.25, pny),
                  pz0 = bracket(pos_xyz[i].z * 0.5 + 0.25, pnz);
        for (int a = -1; a <= 2; ++a)
          for (int b2 = -1; b2 <= 2; ++b2)
            for (int c2 = -1; c2 <= 2; ++c2) {
              const int gx = px0 + a, gy = py0 + b2, gz = pz0 + c2;
              if (gx < 1 || gy < 1 || gz < 1) continue;
              const int bx = (gx - 1) / 8 + 1, by = (gy - 1) / 8 + 1, bz = (gz - 1) / 8 + 1;
              if (bx > pa.dim[0] || by > pa.dim[1] || bz > pa.dim[2]) continue;
              const int32_t pb = pptr[(size_t)(bx - 1) + (size_t)pa.dim[0] * ((by - 1) + (size_t)pa.dim[1] * (bz - 1))];
              if (pb <= 0) continue;
              const int32_t cid = (pb - 1) * 512 + (((gx - 1) % 8) | (((gy - 1) % 8) << 3) | (((gz - 1) % 8) << 6));
              pos_nodes[i * 64 + (size_t)(16 * (a + 1) + 4 * (b2 + 1) + (c2 + 1))] = map[(size_t)cid];
            }
      }
      me.n_nodes = (int32_t)nodes.size();
      const size_t rb = A->storage == OAL_STORE_F64 ? 8 : 4;
      e = cudaMalloc(&me.d_nodes, std::max<size_t>(nodes.size(), 1) * sizeof(int32_t));
      if (e == cudaSuccess && !nodes.empty()) e = cudaMemcpy(me.d_nodes, nodes.data(), nodes.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMalloc(&me.d_node_map, map.size() * sizeof(int32_t));
      if (e == cudaSuccess) e = cudaMemcpy(me.d_node_map, map.data(), map.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMalloc(&me.d_node_vals, std::max<size_t>(nodes.size(), 1) * 32 * rb);
      me.n_pos = (int32_t)pos_xyz.size();
      const size_t np1 = std::max<size_t>(pos_xyz.size(), 1);
      if (e == cudaSuccess) e = cudaMalloc(&me.d_pos_xyz, np1 * sizeof(int4));
      if (e == cudaSuccess) e = cudaMalloc(&me.d_slot_pos, slot_pos.size() * sizeof(int32_t));
      if (e == cudaSuccess) e = cudaMalloc(&me.d_pos_nodes, np1 * 64 * sizeof(int32_t));
      if (e == cudaSuccess) e = cudaMalloc(&me.d_pos_macro, np1 * 4 * rb);
      if (e == cudaSuccess && me.n_pos > 0) {
        e = cudaMemcpy(me.d_pos_xyz, pos_xyz.data(), pos_xyz.size() * sizeof(int4), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(me.d_pos_nodes, pos_nodes.data(), pos_nodes.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      }
      if (e == cudaSuccess) e = cudaMemcpy(me.d_slot_pos, slot_pos.data(), slot_pos.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      // a refined level's fill runs in cell-major entry order (block, cell, direction): the
      // interpolations of one ghost position's directions then read its stencil records together,
      // which outweighs the coalescing of the direction-major order of plain levels. The order of
      // entries carries no meaning (each writes its own slot), so the level's geometry is re-ordered
      // in place.
      if (e == cudaSuccess && g->n_gentries > 0) {
        oal_geometry* gm = const_cast<oal_geometry*>(g);
        auto key = [](const uint2& v) {
          return ((uint64_t)v.x << 14) | ((uint64_t)(v.y & 511u) << 5) | (uint64_t)((v.y >> 9) & 31u);
        };
        std::stable_sort(gm->h_gentries.begin(), gm->h_gentries.end(),
                         [&](const uint2& p, const uint2& q) { return key(p) < key(q); });
        e = cudaMemcpy(gm->d_gentries, gm->h_gentries.data(), gm->h_gentries.size() * sizeof(uint2), cudaMemcpyHostToDevice);
      }
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "amr allocation: %s", cudaGetErrorString(e));
      return fail(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA);
    }
  }
  if (cudaStreamCreateWithFlags(&A->cap, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    set_error(OAL_E_CUDA, "amr stream");
    return fail(OAL_E_CUDA);
  }
  *out = A;
  return OAL_OK;
}

oal_status oal_amr_level(oal_amr* A, int32_t level, oal_level** out) {
  if (!A || !out || level < 0 || level >= (int32_t)A->lv.size()) return set_error(OAL_E_INVALID_ARG, "bad level");
  *out = A->lv[(size_t)level].L;
  return OAL_OK;
}

oal_status oal_amr_advance(oal_amr* A, const oal_step_params* params, int32_t n, void* stream) {
  if (!A || !params) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (n <= 0) return set_error(OAL_E_INVALID_ARG, "n_coarse_steps must be positive");
  const int nl = (int)A->lv.size();
  std::vector<CaseParams> cps((size_t)nl);
  for (int l = 0; l < nl; ++l) {
    oal_status s = resolve_params(&params[l], A->lv[(size_t)l].g, &cps[(size_t)l]);
    if (s != OAL_OK) return s;
    if (cps[(size_t)l].flags & CF_STORE_POST) return set_error(OAL_E_UNSUPPORTED, "store_post_collision needs caller-owned arrays");
    if (cps[(size_t)l].flags & (CF_SGS_PI | CF_SGS_DYNAMIC))
      return set_error(OAL_E_UNSUPPORTED, "variable_nu_sgs: plain levels only, not the levels of a block-AMR hierarchy");
  }
  OAL_CUDA_TRY(cudaSetDevice(A->device));
  for (int l = 0; l < nl; ++l) {
    oal_status s = set_svv(A->lv[(size_t)l].L, &params[l]);
    if (s != OAL_OK) return s;
  }
  const int start = A->lv[0].L->parity;
  bool hit = A->exec && A->g_n == n && A->g_parity == start && (int)A->g_p.size() == nl;
  for (int l = 0; hit && l < nl; ++l) {
    oal_step_params a = params[l], b = A->g_p[(size_t)l];
    a.time_step_seed = b.time_step_seed = 0;
    hit = std::memcmp(&a, &b, sizeof a) == 0 && !(cps[(size_t)l].flags & CF_INLET_NOISE) &&
          A->g_bz.size() == (size_t)nl && A->g_bz[(size_t)l] == A->lv[(size_t)l].L->bz_gen;
  }
  std::vector<int> parities((size_t)nl);
  for (int l = 0; l < nl; ++l) parities[(size_t)l] = A->lv[(size_t)l].L->parity;
  if (!hit) {
    amr_release_graph(A);
    OAL_CUDA_TRY(cudaStreamBeginCapture(A->cap, cudaStreamCaptureModeThreadLocal));
    oal_status es = OAL_OK;
    for (int i = 0; i < n && es == OAL_OK; ++i) es = amr_step(A, 0, cps, params, i, 0.0, A->cap);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(A->cap, &graph);
    for (int l = 0; l < nl; ++l) A->lv[(size_t)l].L->parity = parities[(size_t)l];
    if (es != OAL_OK) { if (graph) cudaGraphDestroy(graph); return es; }
    if (e != cudaSuccess) { cudaGetLastError(); return set_error(OAL_E_CUDA, "graph capture: %s", cudaGetErrorString(e)); }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(graph); cudaGetLastError(); return set_error(OAL_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    A->exec = exec; A->graph = graph; A->g_n = n; A->g_parity = start;
    A->g_p.assign(params, params + nl);
    A->g_bz.resize((size_t)nl);
    for (int l = 0; l < nl; ++l) A->g_bz[(size_t)l] = A->lv[(size_t)l].L->bz_gen;
  }
  OAL_CUDA_TRY(cudaGraphLaunch(A->exec, static_cast<cudaStream_t>(stream)));
  // level l takes n * 2^l steps: only the coarsest level can end on the other buffer
  if (n & 1) A->lv[0].L->parity ^= 1;
  for (int l = 0; l < nl; ++l) A->lv[(size_t)l].L->forces_valid = true;
  return OAL_OK;
}

}  // extern "C"

// ================================================================================================
// Batches: a block pool shared by many cases
// ================================================================================================
namespace {

// first-fit allocator of index ranges
struct RangeAlloc {
  int64_t cap = 0;
  std::vector<std::pair<int64_t, int64_t>> free_;  // (begin, length), sorted by begin
  void init(int64_t c) { cap = c; free_.clear(); if (c > 0) free_.push_back({0, c}); }
  int64_t alloc(int64_t n) {
    if (n == 0) return 0;
    for (size_t i = 0; i < free_.size(); ++i)
      if (free_[i].second >= n) {
        const int64_t b = free_[i].first;
        free_[i].first += n; free_[i].second -= n;
        if (free_[i].second == 0) free_.erase(free_.begin() + (long)i);
        return b;
      }
    return -1;
  }
  void release(int64_t b, int64_t n) {
    if (n == 0) return;
    auto it = std::lower_bound(free_.begin(), free_.end(), std::make_pair(b, (int64_t)0));
    it = free_.insert(it, {b, n});
    // coalesce with neighbours
    size_t i = (size_t)(it - free_.begin());
    if (i + 1 < free_.size() && free_[i].first + free_[i].second == free_[i + 1].first) {
      free_[i].second += free_[i + 1].second; free_.erase(free_.begin() + (long)i + 1);
    }
    if (i > 0 && free_[i - 1].first + free_[i - 1].second == free_[i].first) {
      free_[i - 1].second += free_[i].second; free_.erase(free_.begin() + (long)i);
    }
  }
  int64_t used() const { int64_t f = 0; for (auto& r : free_) f += r.second; return cap - f; }
};

// Equilibrium start of one member's real blocks inside the pool.
template <class S, class R>
__global__ void k_pool_init(const double* __restrict__ rho, const double* __restrict__ vel, int64_t ncell, int comp,
                            S* __restrict__ f, R* __restrict__ rho_out, R* __restrict__ vel_out, int64_t vcs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  const int64_t b = i >> 9, cell = i & 511;
  const R r = R(rho[i]), ux = R(vel[i]), uy = R(vel[i + ncell]), uz = R(vel[i + 2 * ncell]);
  const R usq = ux * ux + uy * uy + uz * uz;
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R w = R(q27_w(k));
    const R cu = R(q27_cx(k)) * ux + R(q27_cy(k)) * uy + R(q27_cz(k)) * uz;
    R val = R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq;
    if (comp) {
      const R cu2 = cu * cu;
      val += (R(4.5) * cu2 * cu - R(4.5) * cu * usq) + (R(3.375) * cu2 * cu2 - R(6.75) * cu2 * usq + R(1.125) * usq * usq);
    }
    f[b * 27 * kCells + k * kCells + cell] = Codec<S>::enc(r * w * val, w, R(1.0 / q27_w(k)));
  }
  rho_out[i] = r;
  vel_out[i] = ux; vel_out[i + vcs] = uy; vel_out[i + 2 * vcs] = uz;
}

// One member's state out of the pool, reference layout (double).
template <class S, class R>
__global__ void k_pool_export(const S* __restrict__ f, const R* __restrict__ rho, const R* __restrict__ vel, int64_t vcs,
                              int64_t ncell, double* __restrict__ fo, double* __restrict__ ro, double* __restrict__ vo) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  const int64_t b = i >> 9, cell = i & 511;
  if (fo)
#pragma unroll
    for (int k = 0; k < kQ27; ++k)
      fo[i + ncell * k] = (double)Codec<S>::dec(f[b * 27 * kCells + k * kCells + cell], R(q27_w(k)), R(1.0 / q27_w(k)));
  if (ro) ro[i] = (double)rho[i];
  if (vo) { vo[i] = (double)vel[i]; vo[i + ncell] = (double)vel[i + vcs]; vo[i + 2 * ncell] = (double)vel[i + 2 * vcs]; }
}

// Per-member FP64 sums of consecutive CTA partial triples: member m owns [seg[m], seg[m+1]).
__global__ void k_reduce3_segments(const double* __restrict__ part, const int32_t* __restrict__ seg, double* __restrict__ out) {
  __shared__ double s[3][256];
  const int m = blockIdx.x, t = threadIdx.x;
  const int64_t b0 = seg[m], b1 = seg[m + 1];
  double a0 = 0, a1 = 0, a2 = 0;
  for (int64_t i = b0 + t; i < b1; i += 256) { a0 += part[3 * i]; a1 += part[3 * i + 1]; a2 += part[3 * i + 2]; }
  s[0][t] = a0; s[1][t] = a1; s[2][t] = a2;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w) { s[0][t] += s[0][t + w]; s[1][t] += s[1][t + w]; s[2][t] += s[2][t + w]; }
    __syncthreads();
  }
  if (t == 0) { out[3 * m] = s[0][0]; out[3 * m + 1] = s[1][0]; out[3 * m + 2] = s[2][0]; }
}

}  // namespace

struct BatchMember {
  bool active = false;
  const oal_geometry* g = nullptr;
  oal_step_params p{};
  CaseParams cp{};
  int64_t rb = 0, gb = 0, mb = 0;  // pool bases: real blocks, ghost blocks, mask slots
  int64_t nb = 0, ng = 0, nm = 0;
  bool forces_valid = false;
  BouzidiSet bz;  // linear Bouzidi boundary cells (oal_batch_set_bouzidi), pool block indices
};

struct oal_batch {
  int device = 0;
  int32_t storage = 0;
  int64_t R = 0, G = 0, M = 0;  // capacities: real blocks, ghost blocks, mask slots
  int32_t max_members = 0;
  RangeAlloc ar, ag, am;
  std::vector<BatchMember> mem;
  void* f[2] = {nullptr, nullptr};
  void* vel[2] = {nullptr, nullptr};
  void* rho = nullptr;
  int32_t* d_nbr = nullptr;      // [R*27] pool indices (ghosts at R + g)
  int4* d_binfo = nullptr;       // [R] coords + member id
  uint32_t* d_bflags = nullptr;  // [R]
  int32_t* d_mslot = nullptr;    // [R]
  uint32_t* d_cmask = nullptr;   // [M*512]
  float* d_sponge = nullptr;     // [R*512] (allocated when a member brings one)
  float* d_wdist = nullptr;
  CaseParams* d_cases = nullptr;  // [max_members]
  uint32_t flags_any = 0;          // OR of the active members' case flags
  // work lists, rebuilt when membership changes
  uint2* d_gentries = nullptr; int64_t n_gentries = 0, cap_gentries = 0;
  uint2* d_fcopy = nullptr; int64_t n_fcopy = 0;  // raw ghost copies of the members (pool elements)
  int32_t* d_fast = nullptr; int64_t n_fast = 0;
  int32_t* d_fast_rec = nullptr;  // x-pair kernel records of d_fast
  int64_t n_fast_in = 0;          // the first n_fast_in fast blocks read no ghost slot
  int32_t* d_general = nullptr; int64_t n_general = 0;
  int32_t* d_seg = nullptr;       // [max_members + 1] general-CTA segments per member
  double* d_part = nullptr;       // [R*4*3]
  double* d_forces = nullptr;     // [max_members*3]
  double* d_mm_part = nullptr;    // [R*4]
  double* d_mm = nullptr;         // [4]
  int parity = 0;
  bool dirty = true;
  cudaStream_t cap = nullptr;
  Overlap ov;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  int32_t graph_n = 0;
  int graph_parity = -1;
  int64_t bytes = 0;
  int32_t prefetch_ctas = 0;  // launch tuning (OAL_TUNE_PREFETCH_CTAS)
  int32_t persistent = 0;     // launch tuning (OAL_TUNE_PERSISTENT)
};

static void batch_release_graph(oal_batch* B) {
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  B->exec = nullptr; B->graph = nullptr; B->graph_n = 0; B->graph_parity = -1;
}

// Combined work lists over the active members (host concatenation, then upload).
static oal_status batch_rebuild(oal_batch* B) {
  std::vector<uint2> ge;
  std::vector<int32_t> fast, fast_bd, general, seg(1, 0);
  std::vector<uint2> fcopy;
  const int64_t pool_elems = (B->R + B->G) * 27 * kCells;
  std::vector<CaseParams> cases((size_t)B->max_members);
  uint32_t flags_any = 0;
  for (int32_t m = 0; m < B->max_members; ++m) {
    const BatchMember& M = B->mem[(size_t)m];
    if (M.active) {
      const oal_geometry* g = M.g;
      // the member's raw ghost copies, rebased into the pool (as a single level of the same
      // geometry copies them); its other fill entries stay with the general fill
      const oal_geometry::FillLists* fl = nullptr;
      if (build_fill_lists(const_cast<oal_geometry*>(g), M.cp.flags) == OAL_OK && pool_elems < (1ll << 32))
        for (const auto& c : g->fills)
          if (c.key == fill_key_of(M.cp.flags)) fl = &c;
      if (fl) {
        const int64_t bst = 27 * kCells;
        for (const uint2& c : fl->h_copies) {
          const int64_t db = c.x / bst, sb = c.y / bst;
          const int64_t dpool = B->R + M.gb + (db - g->nb), spool = M.rb + sb;
          fcopy.push_back(make_uint2((uint32_t)(dpool * bst + c.x % bst), (uint32_t)(spool * bst + c.y % bst)));
        }
        for (const uint2& e : fl->h_other) ge.push_back(make_uint2((uint32_t)(M.rb + e.x), e.y));
      } else {
        for (const uint2& e : g->h_gentries) ge.push_back(make_uint2((uint32_t)(M.rb + e.x), e.y));
      }
      for (int32_t i = 0; i < g->n_fast_in; ++i) fast.push_back((int32_t)(M.rb + g->h_fast[(size_t)i]));
      for (size_t i = (size_t)g->n_fast_in; i < g->h_fast.size(); ++i) fast_bd.push_back((int32_t)(M.rb + g->h_fast[i]));
      for (int32_t b : g->h_general) general.push_back((int32_t)(M.rb + b));
      cases[(size_t)m] = M.cp;
      flags_any |= M.cp.flags;
    }
    seg.push_back((int32_t)(general.size() * 4));
  }
  auto upload = [&](auto*& dptr, const auto& vec, int64_t& n) -> cudaError_t {
    using Tv = typename std::remove_reference<decltype(vec)>::type::value_type;
    cudaFree(dptr); dptr = nullptr; n = (int64_t)vec.size();
    if (vec.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(&dptr, vec.size() * sizeof(Tv));
    if (e == cudaSuccess) e = cudaMemcpy(dptr, vec.data(), vec.size() * sizeof(Tv), cudaMemcpyHostToDevice);
    return e;
  };
  OAL_CUDA_TRY(upload(B->d_gentries, ge, B->n_gentries));
  std::sort(fcopy.begin(), fcopy.end(), [](const uint2& p, const uint2& q) { return p.x < q.x; });
  OAL_CUDA_TRY(upload(B->d_fcopy, fcopy, B->n_fcopy));
  B->n_fast_in = (int64_t)fast.size();
  fast.insert(fast.end(), fast_bd.begin(), fast_bd.end());
  OAL_CUDA_TRY(upload(B->d_fast, fast, B->n_fast));
  cudaFree(B->d_fast_rec);
  B->d_fast_rec = nullptr;
  if (B->n_fast > 0) {
    OAL_CUDA_TRY(cudaMalloc(&B->d_fast_rec, (size_t)B->n_fast * 32 * sizeof(int32_t)));
    OAL_CUDA_TRY(build_fast_records(B->d_fast, (int)B->n_fast, B->d_nbr, B->d_binfo, B->d_fast_rec, nullptr));
    OAL_CUDA_TRY(cudaDeviceSynchronize());
  }
  OAL_CUDA_TRY(upload(B->d_general, general, B->n_general));
  OAL_CUDA_TRY(cudaMemcpy(B->d_seg, seg.data(), seg.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  OAL_CUDA_TRY(cudaMemcpy(B->d_cases, cases.data(), cases.size() * sizeof(CaseParams), cudaMemcpyHostToDevice));
  B->flags_any = flags_any;
  B->dirty = false;
  batch_release_graph(B);
  return OAL_OK;
}

template <class S, class R>
static cudaError_t batch_step_t(oal_batch* B, const StepArgs& a, cudaStream_t st) {
  cudaError_t e;
  // as for a single level: fill, general and boundary blocks on the side stream, interior blocks
  // (no ghost reads) on the main stream
  const int n_in = (int)B->n_fast_in, n_bd = (int)(B->n_fast - B->n_fast_in);
  const bool fork = n_in > 0 && (B->n_general > 0 || n_bd > 0);
  if (fork) {
    if ((e = cudaEventRecord(B->ov.fork, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(B->ov.side, B->ov.fork, 0)) != cudaSuccess) return e;
    if ((e = launch_fill_copy<S, R>(a, B->d_fcopy, B->n_fcopy, B->ov.side, true)) != cudaSuccess) return e;
    if ((e = launch_fill_ghosts<S, R>(a, B->d_gentries, B->n_gentries, B->ov.side)) != cudaSuccess) return e;
    if ((e = launch_general<S, R>(a, B->d_general, (int)B->n_general, B->ov.side)) != cudaSuccess) return e;
    if ((e = launch_fast_range<S, R>(a, B->d_fast, n_in, n_bd, B->ov.side)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(B->ov.join, B->ov.side)) != cudaSuccess) return e;
    if ((e = launch_fast_range<S, R>(a, B->d_fast, 0, n_in, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(st, B->ov.join, 0)) != cudaSuccess) return e;
  } else {
    if ((e = launch_fill_copy<S, R>(a, B->d_fcopy, B->n_fcopy, st, true)) != cudaSuccess) return e;
    if ((e = launch_fill_ghosts<S, R>(a, B->d_gentries, B->n_gentries, st)) != cudaSuccess) return e;
    if ((e = launch_fast<S, R>(a, B->d_fast, (int)B->n_fast, st)) != cudaSuccess) return e;
    if ((e = launch_general<S, R>(a, B->d_general, (int)B->n_general, st)) != cudaSuccess) return e;
  }
  if (B->n_general > 0) {
    k_reduce3_segments<<<B->max_members, 256, 0, st>>>(B->d_part, B->d_seg, B->d_forces);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static oal_status batch_enqueue_step(oal_batch* B, int step_offset, cudaStream_t st) {
  StepArgs a{};
  a.nbr = B->d_nbr;
  a.binfo = B->d_binfo;
  a.bflags = B->d_bflags;
  a.mslot = B->d_mslot;
  a.cmask = B->d_cmask;
  a.sponge = B->d_sponge;
  a.wall_dist = B->d_wdist;
  a.cases = B->d_cases;
  a.flags_any = B->flags_any;
  a.fast_rec = B->d_fast_rec;
  a.prefetch_ctas = B->prefetch_ctas;
  a.persistent = B->persistent;
  a.n_blocks = (int32_t)B->R;
  a.n_total_blocks = (int32_t)(B->R + B->G);
  a.block_base = 0;
  const int p = B->parity;
  a.f_in = B->f[p]; a.f_out = B->f[p ^ 1]; a.f_post = nullptr;
  a.rho_out = B->rho; a.vel_out = B->vel[p ^ 1]; a.vel_in = B->vel[p];
  a.f_bstride = 27 * 512; a.f_kstride = 512;
  a.v_bstride = 512; a.v_cstride = 512 * B->R;
  a.force_part = B->d_part;
  (void)step_offset;
  cudaError_t e = cudaErrorInvalidValue;
  switch (B->storage) {
    case OAL_STORE_F32: e = batch_step_t<float, float>(B, a, st); break;
    case OAL_STORE_F16_DEV: e = batch_step_t<__half, float>(B, a, st); break;
    case OAL_STORE_BF16_DEV: e = batch_step_t<__nv_bfloat16, float>(B, a, st); break;
    case OAL_STORE_F64: e = batch_step_t<double, double>(B, a, st); break;
  }
  OAL_CUDA_TRY(e);
  // the members' linear Bouzidi walls on the step's output (their cells in pool indices)
  PopIndex pix{};
  pix.binfo = B->d_binfo;
  pix.bst = 27 * 512;
  pix.kst = 512;
  for (const auto& M : B->mem)
    if (M.active && (M.cp.flags & CF_BOUZIDI) && M.bz.n > 0)
      OAL_CUDA_TRY(bouzidi_enqueue(M.bz, B->storage, a.f_out, pix, B->d_nbr, B->d_mslot, B->d_cmask, st, (int32_t)B->R));
  B->parity ^= 1;
  return OAL_OK;
}

template <class S, class R>
static cudaError_t pool_init_t(oal_batch* B, const BatchMember& M, const double* d_rho, const double* d_vel, int comp) {
  const int64_t ncell = M.nb * 512;
  k_pool_init<S, R><<<nblk(ncell, 256), 256>>>(d_rho, d_vel, ncell, comp,
                                              static_cast<S*>(B->f[B->parity]) + M.rb * 27 * 512,
                                              static_cast<R*>(B->rho) + M.rb * 512,
                                              static_cast<R*>(B->vel[B->parity]) + M.rb * 512, 512 * B->R);
  return cudaGetLastError();
}

template <class S, class R>
static cudaError_t pool_export_t(oal_batch* B, const BatchMember& M, double* fo, double* ro, double* vo) {
  const int64_t ncell = M.nb * 512;
  k_pool_export<S, R><<<nblk(ncell, 256), 256>>>(static_cast<const S*>(B->f[B->parity]) + M.rb * 27 * 512,
                                                static_cast<const R*>(B->rho) + M.rb * 512,
                                                static_cast<const R*>(B->vel[B->parity]) + M.rb * 512, 512 * B->R,
                                                ncell, fo, ro, vo);
  return cudaGetLastError();
}

template <class S, class R>
static cudaError_t pool_mm_t(oal_batch* B, const BatchMember& M) {
  PopIndex pi{};
  pi.binfo = B->d_binfo + M.rb; pi.dense = 0; pi.bst = 27 * 512; pi.kst = 512;
  k_mass_momentum<S, R><<<(unsigned)M.nb, 128>>>(static_cast<const S*>(B->f[B->parity]) + M.rb * 27 * 512, pi,
                                                B->d_bflags + M.rb, B->d_mslot + M.rb, B->d_cmask, B->d_mm_part);
  k_reduce4<<<1, 256>>>(B->d_mm_part, M.nb, B->d_mm);
  return cudaGetLastError();
}

extern "C" {

oal_status oal_geometry_blocks(const oal_geometry* g, int64_t out[3]) {
  if (!g || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  out[0] = g->nb; out[1] = g->n_ghost; out[2] = g->n_slots;
  return OAL_OK;
}

void oal_batch_destroy(oal_batch* B) {
  if (!B) return;
  cudaSetDevice(B->device);
  batch_release_graph(B);
  for (int i = 0; i < 2; ++i) { cudaFree(B->f[i]); cudaFree(B->vel[i]); }
  cudaFree(B->rho); cudaFree(B->d_nbr); cudaFree(B->d_binfo); cudaFree(B->d_bflags); cudaFree(B->d_mslot);
  cudaFree(B->d_cmask); cudaFree(B->d_sponge); cudaFree(B->d_wdist); cudaFree(B->d_cases);
  cudaFree(B->d_gentries); cudaFree(B->d_fast); cudaFree(B->d_general); cudaFree(B->d_seg);
  cudaFree(B->d_fast_rec); cudaFree(B->d_fcopy);
  cudaFree(B->d_part); cudaFree(B->d_forces); cudaFree(B->d_mm_part); cudaFree(B->d_mm);
  if (B->cap) cudaStreamDestroy(B->cap);
  if (B->ov.side) cudaStreamDestroy(B->ov.side);
  if (B->ov.fork) cudaEventDestroy(B->ov.fork);
  if (B->ov.join) cudaEventDestroy(B->ov.join);
  for (auto& M : B->mem) bouzidi_free(&M.bz);
  for (auto& M : B->mem)
    if (M.active && M.g) {
      auto* g = const_cast<oal_geometry*>(M.g);
      if (--g->n_levels == 0 && g->destroy_requested) geometry_release(g);
    }
  cudaGetLastError();
  delete B;
}

oal_status oal_batch_create(int32_t device, int32_t storage, int32_t max_real, int32_t max_ghost, int32_t max_mask,
                            int32_t max_members, oal_batch** out) {
  if (!out) return set_error(OAL_E_INVALID_ARG, "null argument");
  *out = nullptr;
  if (storage < OAL_STORE_F32 || storage > OAL_STORE_F64) return set_error(OAL_E_INVALID_ARG, "storage %d", storage);
  if (max_real <= 0 || max_ghost < 0 || max_mask < 0 || max_members <= 0 || max_members > 4096)
    return set_error(OAL_E_INVALID_ARG, "bad batch capacities");
  if ((int64_t)(max_real + max_ghost) * 27 * 512 >= (1ll << 32))
    return set_error(OAL_E_TOO_LARGE, "a batch pool holds fewer than 2^32 population elements");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return set_error(OAL_E_NO_DEVICE, "no CUDA device visible"); }
  OAL_CUDA_TRY(cudaSetDevice(device));
  auto* B = new oal_batch();
  B->device = device; B->storage = storage;
  B->R = max_real; B->G = max_ghost; B->M = max_mask; B->max_members = max_members;
  B->ar.init(B->R); B->ag.init(B->G); B->am.init(B->M);
  B->mem.resize((size_t)max_members);
  const size_t fbytes = (size_t)(B->R + B->G) * 27 * 512 * storage_bytes(storage);
  const size_t mb = macro_bytes(storage);
  const size_t ncell = (size_t)B->R * 512;
  cudaError_t e = cudaSuccess;
  auto A = [&](void** p, size_t n) { if (e == cudaSuccess && n) e = cudaMalloc(p, n); };
  for (int i = 0; i < 2; ++i) { A(&B->f[i], fbytes); A(&B->vel[i], ncell * 3 * mb); }
  A(&B->rho, ncell * mb);
  A((void**)&B->d_nbr, (size_t)B->R * 27 * sizeof(int32_t));
  A((void**)&B->d_binfo, (size_t)B->R * sizeof(int4));
  A((void**)&B->d_bflags, (size_t)B->R * sizeof(uint32_t));
  A((void**)&B->d_mslot, (size_t)B->R * sizeof(int32_t));
  A((void**)&B->d_cmask, (size_t)B->M * 512 * sizeof(uint32_t));
  A((void**)&B->d_cases, (size_t)max_members * sizeof(CaseParams));
  A((void**)&B->d_seg, (size_t)(max_members + 1) * sizeof(int32_t));
  A((void**)&B->d_part, (size_t)B->R * 4 * 3 * sizeof(double));
  A((void**)&B->d_forces, (size_t)max_members * 3 * sizeof(double));
  A((void**)&B->d_mm_part, (size_t)B->R * 4 * sizeof(double));
  A((void**)&B->d_mm, 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(B->f[0], 0, fbytes);
  if (e == cudaSuccess) e = cudaMemset(B->f[1], 0, fbytes);
  if (e == cudaSuccess) e = cudaMemset(B->d_forces, 0, (size_t)max_members * 3 * sizeof(double));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->ov.side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->ov.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->ov.join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    oal_batch_destroy(B);
    return set_error(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "batch allocation: %s",
                     cudaGetErrorString(e));
  }
  B->bytes = (int64_t)(2 * fbytes + ncell * 7 * mb + (size_t)B->R * (27 * 4 + 16 + 4 + 4 + 96 + 32) +
                       (size_t)B->M * 2048 + (size_t)max_members * 112);
  *out = B;
  return OAL_OK;
}


oal_status oal_batch_add(oal_batch* B, const oal_geometry* g, const oal_step_params* p, const double* rho,
                         const double* vel, int32_t* member_out) {
  if (!B || !g || !p || !rho || !vel || !member_out) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (g->device != B->device) return set_error(OAL_E_INVALID_ARG, "geometry and batch on different devices");
  CaseParams cp;
  oal_status s = resolve_params(p, g, &cp);
  if (s != OAL_OK) return s;
  if (cp.flags & (CF_SGS_PI | CF_SGS_DYNAMIC))
    return set_error(OAL_E_UNSUPPORTED, "variable_nu_sgs: plain levels only, not batched cases (oal_batch_*)");
  if (p->svv_x_epsilon > 0.0f || p->svv_yz_epsilon > 0.0f)
    return set_error(OAL_E_UNSUPPORTED, "the SVV filter: plain levels and hierarchies only, not batched cases (oal_batch_*)");
  if (cp.flags & CF_STORE_POST) return set_error(OAL_E_UNSUPPORTED, "store_post_collision needs caller-owned arrays");
  int32_t m = -1;
  for (int32_t i = 0; i < B->max_members; ++i)
    if (!B->mem[(size_t)i].active) { m = i; break; }
  if (m < 0) return set_error(OAL_E_ADMISSION, "no free member slot (max_members %d)", B->max_members);
  const int64_t rb = B->ar.alloc(g->nb);
  const int64_t gb = rb >= 0 ? B->ag.alloc(g->n_ghost) : -1;
  const int64_t mbase = gb >= 0 ? B->am.alloc(g->n_slots) : -1;
  if (rb < 0 || gb < 0 || mbase < 0) {
    if (gb >= 0) B->ag.release(gb, g->n_ghost);
    if (rb >= 0) B->ar.release(rb, g->nb);
    return set_error(OAL_E_ADMISSION, "the block pool has no room for %lld real / %lld ghost / %lld mask blocks",
                     (long long)g->nb, (long long)g->n_ghost, (long long)g->n_slots);
  }
  OAL_CUDA_TRY(cudaSetDevice(B->device));
  BatchMember& M = B->mem[(size_t)m];
  M = BatchMember();
  M.active = true; M.g = g; M.p = *p; M.cp = cp;
  M.rb = rb; M.gb = gb; M.mb = mbase; M.nb = g->nb; M.ng = g->n_ghost; M.nm = g->n_slots;
  ++const_cast<oal_geometry*>(g)->n_levels;
  // static tables of the member, remapped into the pool
  const int64_t nb = g->nb;
  std::vector<int32_t> nbr((size_t)nb * 27);
  for (size_t i = 0; i < nbr.size(); ++i) {
    const int32_t v = g->h_nbrg[i];
    nbr[i] = v < 0 ? -1 : (v < g->nb ? (int32_t)(rb + v) : (int32_t)(B->R + gb + (v - g->nb)));
  }
  std::vector<int4> bi(g->h_binfo);
  for (auto& x : bi) x.w = m;
  std::vector<int32_t> ms(g->h_mslot);
  for (auto& x : ms) if (x >= 0) x = (int32_t)(mbase + x);
  cudaError_t e = cudaMemcpy(B->d_nbr + rb * 27, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B->d_binfo + rb, bi.data(), bi.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B->d_bflags + rb, g->h_bflags.data(), (size_t)nb * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B->d_mslot + rb, ms.data(), (size_t)nb * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !g->h_cmask.empty())
    e = cudaMemcpy(B->d_cmask + mbase * 512, g->h_cmask.data(), g->h_cmask.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !g->h_sponge.empty()) {
    if (!B->d_sponge) {
      e = cudaMalloc(&B->d_sponge, (size_t)B->R * 512 * sizeof(float));
      if (e == cudaSuccess) e = cudaMemset(B->d_sponge, 0, (size_t)B->R * 512 * sizeof(float));
    }
    if (e == cudaSuccess) e = cudaMemcpy(B->d_sponge + rb * 512, g->h_sponge.data(), g->h_sponge.size() * 4, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !g->h_wdist.empty()) {
    if (!B->d_wdist) {
      e = cudaMalloc(&B->d_wdist, (size_t)B->R * 512 * sizeof(float));
      if (e == cudaSuccess) e = cudaMemset(B->d_wdist, 0, (size_t)B->R * 512 * sizeof(float));
    }
    if (e == cudaSuccess) e = cudaMemcpy(B->d_wdist + rb * 512, g->h_wdist.data(), g->h_wdist.size() * 4, cudaMemcpyHostToDevice);
  }
  // equilibrium start into the current input buffer
  double *d_rho = nullptr, *d_vel = nullptr;
  const int64_t ncell = nb * 512;
  if (e == cudaSuccess) e = cudaMalloc(&d_rho, ncell * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_vel, 3 * ncell * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(d_rho, rho, ncell * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_vel, vel, 3 * ncell * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    switch (B->storage) {
      case OAL_STORE_F32: e = pool_init_t<float, float>(B, M, d_rho, d_vel, p->compressible_corr); break;
      case OAL_STORE_F16_DEV: e = pool_init_t<__half, float>(B, M, d_rho, d_vel, p->compressible_corr); break;
      case OAL_STORE_BF16_DEV: e = pool_init_t<__nv_bfloat16, float>(B, M, d_rho, d_vel, p->compressible_corr); break;
      case OAL_STORE_F64: e = pool_init_t<double, double>(B, M, d_rho, d_vel, p->compressible_corr); break;
    }
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(d_rho); cudaFree(d_vel);
  if (e != cudaSuccess) {
    oal_batch_remove(B, m);
    return set_error(OAL_E_CUDA, "batch_add: %s", cudaGetErrorString(e));
  }
  B->dirty = true;
  *member_out = m;
  return OAL_OK;
}

oal_status oal_batch_remove(oal_batch* B, int32_t m) {
  if (!B || m < 0 || m >= B->max_members || !B->mem[(size_t)m].active) return set_error(OAL_E_INVALID_ARG, "no such member");
  BatchMember& M = B->mem[(size_t)m];
  B->ar.release(M.rb, M.nb); B->ag.release(M.gb, M.ng); B->am.release(M.mb, M.nm);
  auto* g = const_cast<oal_geometry*>(M.g);
  cudaSetDevice(B->device);
  cudaDeviceSynchronize();  // a step in flight may still read the member's Bouzidi set
  bouzidi_free(&M.bz);
  M = BatchMember();
  if (--g->n_levels == 0 && g->destroy_requested) geometry_release(g);
  B->dirty = true;
  return OAL_OK;
}

oal_status oal_batch_set_bouzidi(oal_batch* B, int32_t m, int32_t n_cells, const int32_t* cell_block,
                                 const int32_t* cell_x, const int32_t* cell_y, const int32_t* cell_z,
                                 const uint16_t* q_half, float q_min_threshold, int32_t ff_fallback,
                                 float limiter_rel_cap, float limiter_abs_cap) {
  if (!B || m < 0 || m >= B->max_members || !B->mem[(size_t)m].active) return set_error(OAL_E_INVALID_ARG, "no such member");
  BatchMember& M = B->mem[(size_t)m];
  OAL_CUDA_TRY(cudaSetDevice(B->device));
  OAL_CUDA_TRY(cudaDeviceSynchronize());  // a step in flight may still read the old set
  batch_release_graph(B);
  return bouzidi_upload(&M.bz, B->storage, M.nb, M.rb, n_cells, cell_block, cell_x, cell_y, cell_z, q_half,
                        q_min_threshold, ff_fallback, limiter_rel_cap, limiter_abs_cap);
}

oal_status oal_batch_set_params(oal_batch* B, int32_t m, const oal_step_params* p) {
  if (!B || m < 0 || m >= B->max_members || !B->mem[(size_t)m].active) return set_error(OAL_E_INVALID_ARG, "no such member");
  CaseParams cp;
  oal_status s = resolve_params(p, B->mem[(size_t)m].g, &cp);
  if (s != OAL_OK) return s;
  if (cp.flags & (CF_SGS_PI | CF_SGS_DYNAMIC))
    return set_error(OAL_E_UNSUPPORTED, "variable_nu_sgs: plain levels only, not batched cases (oal_batch_*)");
  if (p->svv_x_epsilon > 0.0f || p->svv_yz_epsilon > 0.0f)
    return set_error(OAL_E_UNSUPPORTED, "the SVV filter: plain levels and hierarchies only, not batched cases (oal_batch_*)");
  B->mem[(size_t)m].p = *p; B->mem[(size_t)m].cp = cp;
  B->dirty = true;
  return OAL_OK;
}

oal_status oal_batch_advance(oal_batch* B, int32_t n, void* stream) {
  if (!B) return set_error(OAL_E_INVALID_ARG, "null batch");
  if (n <= 0) return set_error(OAL_E_INVALID_ARG, "n_steps must be positive");
  OAL_CUDA_TRY(cudaSetDevice(B->device));
  if (B->dirty) {
    // a rebuild must not race with steps still in flight on the caller's stream
    OAL_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    oal_status s = batch_rebuild(B);
    if (s != OAL_OK) return s;
  }
  if (B->n_fast + B->n_general == 0) return OAL_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // One graph of two steps (both parities) launched n/2 times, plus one single step when n is odd:
  // membership changes then cost one small capture instead of an n-step graph.
  if (!(B->exec && B->graph_parity == B->parity)) {
    batch_release_graph(B);
    const int start = B->parity;
    OAL_CUDA_TRY(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
    oal_status es = OAL_OK;
    for (int i = 0; i < 2 && es == OAL_OK; ++i) es = batch_enqueue_step(B, i, B->cap);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(B->cap, &graph);
    B->parity = start;
    if (es != OAL_OK) { if (graph) cudaGraphDestroy(graph); return es; }
    if (e != cudaSuccess) return set_error(OAL_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(graph); return set_error(OAL_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    B->exec = exec; B->graph = graph; B->graph_n = 2; B->graph_parity = start;
  }
  for (int i = 0; i + 1 < n; i += 2) OAL_CUDA_TRY(cudaGraphLaunch(B->exec, st));
  if (n & 1) {
    oal_status es = batch_enqueue_step(B, n - 1, st);  // flips the parity; the graph is re-made next time
    if (es != OAL_OK) return es;
  }
  for (auto& M : B->mem)
    if (M.active && (M.cp.flags & CF_COLLECT)) M.forces_valid = true;
  return OAL_OK;
}

oal_status oal_batch_set_tuning(oal_batch* B, int32_t key, int64_t value) {
  if (!B) return set_error(OAL_E_INVALID_ARG, "null batch");
  int32_t* slot = key == OAL_TUNE_PREFETCH_CTAS ? &B->prefetch_ctas : key == OAL_TUNE_PERSISTENT ? &B->persistent : nullptr;
  if (!slot) return set_error(OAL_E_INVALID_ARG, "unknown tuning key %d", key);
  if (value < 0 || value > (key == OAL_TUNE_PERSISTENT ? 1 : (1 << 24)))
    return set_error(OAL_E_INVALID_ARG, "tuning key %d: value %lld", key, (long long)value);
  if (*slot != (int32_t)value) {
    *slot = (int32_t)value;
    batch_release_graph(B);
  }
  return OAL_OK;
}

oal_status oal_batch_get_tuning(const oal_batch* B, int32_t key, int64_t* value) {
  if (!B || !value) return set_error(OAL_E_INVALID_ARG, "null argument");
  if (key == OAL_TUNE_PREFETCH_CTAS) *value = B->prefetch_ctas;
  else if (key == OAL_TUNE_PERSISTENT) *value = B->persistent;
  else return set_error(OAL_E_INVALID_ARG, "unknown tuning key %d", key);
  return OAL_OK;
}

oal_status oal_batch_autotune(oal_batch* B, int32_t n_steps, int64_t* prefetch, int32_t* persistent,
                              double* ms_per_step) {
  if (!B) return set_error(OAL_E_INVALID_ARG, "null batch");
  if (n_steps <= 0) return set_error(OAL_E_INVALID_ARG, "n_steps must be positive");
  OAL_CUDA_TRY(cudaSetDevice(B->device));
  OAL_CUDA_TRY(cudaDeviceSynchronize());
  if (B->dirty) {
    oal_status rs = batch_rebuild(B);
    if (rs != OAL_OK) return rs;
  }
  const size_t ncell = (size_t)B->R * 512, mb = macro_bytes(B->storage);
  const size_t fbytes = (size_t)(B->R + B->G) * 27 * 512 * storage_bytes(B->storage);
  StateSnapshot snap;
  cudaError_t e = snap.add(B->f[B->parity], fbytes);
  if (e == cudaSuccess) e = snap.add(B->vel[B->parity], ncell * 3 * mb);
  if (e == cudaSuccess) e = snap.add(B->rho, ncell * mb);
  if (e != cudaSuccess)
    return set_error(e == cudaErrorMemoryAllocation ? OAL_E_OUT_OF_MEMORY : OAL_E_CUDA, "autotune snapshot: %s", cudaGetErrorString(e));
  int64_t cand[OAL_TUNE_CANDIDATES];
  int32_t pers[OAL_TUNE_CANDIDATES];
  OAL_CUDA_TRY(tune_candidates(B->device, cand, pers));
  const int parity0 = B->parity;
  const int32_t keep = B->prefetch_ctas, keep_p = B->persistent;
  cudaStream_t st = nullptr;
  OAL_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  oal_status s = OAL_OK;
  double best = 0.0;
  int best_c = -1;
  for (int c = 0; c < OAL_TUNE_CANDIDATES && s == OAL_OK; ++c) {
    if ((s = oal_batch_set_tuning(B, OAL_TUNE_PREFETCH_CTAS, cand[c])) != OAL_OK) break;
    if ((s = oal_batch_set_tuning(B, OAL_TUNE_PERSISTENT, pers[c])) != OAL_OK) break;
    double ms = 0.0;
    s = time_candidate([&](cudaStream_t q) { return oal_batch_advance(B, n_steps, q); },
                       [&]() -> oal_status {
                         cudaError_t re = snap.restore();
                         B->parity = parity0;
                         return re == cudaSuccess ? OAL_OK : set_error(OAL_E_CUDA, "autotune restore: %s", cudaGetErrorString(re));
                       },
                       n_steps, st, &ms);
    if (prefetch) prefetch[c] = cand[c];
    if (persistent) persistent[c] = pers[c];
    if (ms_per_step) ms_per_step[c] = ms;
    if (s == OAL_OK && (best_c < 0 || ms < best)) { best = ms; best_c = c; }
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cudaError_t re = snap.restore();
  B->parity = parity0;
  for (auto& M : B->mem) M.forces_valid = false;
  oal_batch_set_tuning(B, OAL_TUNE_PREFETCH_CTAS, s == OAL_OK && best_c >= 0 ? cand[best_c] : keep);
  oal_batch_set_tuning(B, OAL_TUNE_PERSISTENT, s == OAL_OK && best_c >= 0 ? pers[best_c] : keep_p);
  if (s != OAL_OK) return s;
  if (re != cudaSuccess) return set_error(OAL_E_CUDA, "autotune restore: %s", cudaGetErrorString(re));
  return OAL_OK;
}


oal_status oal_batch_get_state(oal_batch* B, int32_t m, double* f, double* rho, double* vel) {
  if (!B || m < 0 || m >= B->max_members || !B->mem[(size_t)m].active) return set_error(OAL_E_INVALID_ARG, "no such member");
  OAL_CUDA_TRY(cudaSetDevice(B->device));
  OAL_CUDA_TRY(cudaDeviceSynchronize());
  const BatchMember& M = B->mem[(size_t)m];
  const int64_t ncell = M.nb * 512;
  double *df = nullptr, *dr = nullptr, *dv = nullptr;
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMalloc(&df, 27 * ncell * sizeof(double));
  if (e == cudaSuccess && rho) e = cudaMalloc(&dr, ncell * sizeof(double));
  if (e == cudaSuccess && vel) e = cudaMalloc(&dv, 3 * ncell * sizeof(double));
  if (e == cudaSuccess) {
    switch (B->storage) {
      case OAL_STORE_F32: e = pool_export_t<float, float>(B, M, df, dr, dv); break;
      case OAL_STORE_F16_DEV: e = pool_export_t<__half, float>(B, M, df, dr, dv); break;
      case OAL_STORE_BF16_DEV: e = pool_export_t<__nv_bfloat16, float>(B, M, df, dr, dv); break;
      case OAL_STORE_F64: e = pool_export_t<double, double>(B, M, df, dr, dv); break;
    }
  }
  if (e == cudaSuccess && f) e = cudaMemcpy(f, df, 27 * ncell * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && rho) e = cudaMemcpy(rho, dr, ncell * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && vel) e = cudaMemcpy(vel, dv, 3 * ncell * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(df); cudaFree(dr); cudaFree(dv);
  if (e != cudaSuccess) return set_error(OAL_E_CUDA, "batch_get_state: %s", cudaGetErrorString(e));
  return OAL_OK;
}

oal_status oal_batch_get_forces(oal_batch* B, int32_t m, double out[3]) {
  if (!B || !out || m < 0 || m >= B->max_members || !B->mem[(size_t)m].active) return set_error(OAL_E_INVALID_ARG, "no such member");
  OAL_CUDA_TRY(cudaSetDevice(B->device));
  if (!B->mem[(size_t)m].forces_valid || B->n_general == 0) { out[0] = out[1] = out[2] = 0.0; return OAL_OK; }
  OAL_CUDA_TRY(cudaMemcpy(out, B->d_forces + 3 * m, 3 * sizeof(double), cudaMemcpyDeviceToHost));
  return OAL_OK;
}


oal_status oal_batch_mass_momentum(oal_batch* B, int32_t m, double out[4]) {
  if (!B || !out || m < 0 || m >= B->max_members || !B->mem[(size_t)m].active) return set_error(OAL_E_INVALID_ARG, "no such member");
  OAL_CUDA_TRY(cudaSetDevice(B->device));
  const BatchMember& M = B->mem[(size_t)m];
  cudaError_t e = cudaErrorInvalidValue;
  switch (B->storage) {
    case OAL_STORE_F32: e = pool_mm_t<float, float>(B, M); break;
    case OAL_STORE_F16_DEV: e = pool_mm_t<__half, float>(B, M); break;
    case OAL_STORE_BF16_DEV: e = pool_mm_t<__nv_bfloat16, float>(B, M); break;
    case OAL_STORE_F64: e = pool_mm_t<double, double>(B, M); break;
  }
  OAL_CUDA_TRY(e);
  OAL_CUDA_TRY(cudaMemcpy(out, B->d_mm, 4 * sizeof(double), cudaMemcpyDeviceToHost));
  return OAL_OK;
}

oal_status oal_batch_info(const oal_batch* B, int64_t out[8]) {
  if (!B || !out) return set_error(OAL_E_INVALID_ARG, "null argument");
  int64_t n = 0;
  for (auto& M : B->mem) n += M.active ? 1 : 0;
  out[0] = n; out[1] = B->ar.used(); out[2] = B->ag.used(); out[3] = B->am.used();
  out[4] = B->R; out[5] = B->G; out[6] = B->M; out[7] = B->bytes;
  return OAL_OK;
}

}  // extern "C"
