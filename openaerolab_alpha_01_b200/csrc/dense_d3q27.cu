// dense_d3q27.cu — the uniform D3Q27 cumulant step of box levels with shared-memory-staged
// streaming.
//
// A box level stores its populations on a padded grid f[k][Z][Y][X] (interior cell (i,j,l) at
// X = i + 8, Y = j + 1, Z = l + 1; a one-cell ghost frame, filled before each step with the
// domain-face and periodic values, and 8 cells of x padding so that every row copy starts on a
// 16-byte boundary). For one 8^3 block the pull of direction k reads the block's cells shifted by
// -c_k, i.e. the box [X0-cx, +8) x [Y0-cy, +8) x [Z0-cz, +8). The CTA copies, per block and
// direction, a 16-wide box aligned at X0-8 (cx = +1) or X0 (cx = 0, -1) into shared memory with
// 16-byte cp.async copies spread over all threads, two stages deep: the copies of the next block
// fly while the current one is collided. The pull then is one shared-memory load per population
// at a constant offset.
//
// (Tensor-memory-accelerator box loads were measured first: 27 boxes of 16- or 32-byte rows per
// block ran at one row per ~23 SM cycles and left the CTAs waiting; per-thread async copies keep
// thousands of 16-byte requests in flight per CTA.)
//
// Physics: identical to the uniform kernel of cumulant_d3q27.cu (kernel_cumulant.jl:190-908 with
// zero force) through the shared cumulant_math.cuh; two cells per thread in packed f32x2.
#include <type_traits>

#include "common.cuh"
#include "vmath.cuh"
#include "cumulant_math.cuh"

namespace oal {

// every direction's box is 16 x 8 x 8 in shared memory
__host__ __device__ constexpr int dense_w(int) { return 16; }
// x offset of a thread's source inside the box of direction k
__host__ __device__ constexpr int dense_xo(int k) { return q27_cx(k) == 1 ? 7 : (q27_cx(k) == -1 ? 1 : 0); }
__host__ __device__ constexpr int dense_off(int k) { return k * 1024; }
constexpr int kDenseStageElems = 27 * 1024;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <class S>
__device__ __forceinline__ F2 dec2(S a, S b, int k) {
  if constexpr (std::is_same<S, float>::value) {
    return f2(a, b);
  } else {
    float x, y;
    if constexpr (std::is_same<S, __half>::value) { x = __half2float(a); y = __half2float(b); }
    else { x = __bfloat162float(a); y = __bfloat162float(b); }
    const F2 w = splat<F2>(float(q27_w(k)));
    return vfma(f2(x, y), w, w);
  }
}
template <class S>
__device__ __forceinline__ void enc2_store(S* __restrict__ f, int64_t i0, int64_t i1, F2 v, int k) {
  float a, b;
  if constexpr (std::is_same<S, float>::value) {
    f2split(v, a, b);
    f[i0] = a; f[i1] = b;
  } else {
    f2split(vfma(v, splat<F2>(float(1.0 / q27_w(k))), splat<F2>(-1.0f)), a, b);
    if constexpr (std::is_same<S, __half>::value) { f[i0] = __float2half_rn(a); f[i1] = __float2half_rn(b); }
    else { f[i0] = __float2bfloat16_rn(a); f[i1] = __float2bfloat16_rn(b); }
  }
}

template <class S, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_dense_fast(const StepArgs a, const int32_t* __restrict__ work, int n_work) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // stages on a 128-byte boundary (the launch adds 128 bytes of slack)
  S* stage0 = reinterpret_cast<S*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
  S* stage1 = stage0 + kDenseStageElems;
  __shared__ int32_t s_nbr[2][28];
  __shared__ int4 s_bi[2];
  __shared__ int64_t s_koff[27];
  __shared__ CaseParams s_cp;
  using V = F2;
  using T = float;
  const int tid = threadIdx.x;
  const int64_t PXY = (int64_t)a.PX * a.PY;
  if (tid < 27) {
    // source element of box row 0 of direction k relative to the block's element (X0, Y0, Z0)
    const int k = tid;
    s_koff[k] = k * a.f_kstride - (int64_t)q27_cz(k) * PXY - (int64_t)q27_cy(k) * a.PX - (q27_cx(k) == 1 ? 8 : 0);
  }
  if (tid >= 32 && tid < 32 + (int)(sizeof(CaseParams) / 4))
    reinterpret_cast<uint32_t*>(&s_cp)[tid - 32] = reinterpret_cast<const uint32_t*>(&a.p0)[tid - 32];
  __syncthreads();
  const CaseParams& cp = s_cp;

  // copy assignment: 16-byte chunks, CPR per 16-wide row; thread t copies chunk `part` of rows
  // r, r + RPP, r + 2 RPP, ... of the 27 x 64 rows of a stage
  constexpr int CPR = (int)(16 * sizeof(S)) / 16;
  constexpr int RPP = 256 / CPR;
  constexpr int NPASS = (27 * 64 + RPP - 1) / RPP;
  const int part = tid % CPR, r = tid / CPR;
  const S* __restrict__ fin = static_cast<const S*>(a.f_in);
  auto issue = [&](int w, int s) {
    const int4 bi = a.binfo[work[w]];
    const int64_t base = dense_idx(a, (bi.x - 1) * kBS + 8, (bi.y - 1) * kBS + 1, (bi.z - 1) * kBS + 1);
    const uint32_t sbase = smem_u32(s ? stage1 : stage0);
#pragma unroll
    for (int i = 0; i < NPASS; ++i) {
      const int R = r + RPP * i;
      if (R < 27 * 64) {
        const int k = R >> 6, row = R & 63, y = row & 7, z = row >> 3;
        const S* src = fin + base + s_koff[k] + (int64_t)z * PXY + (int64_t)y * a.PX + part * (16 / (int)sizeof(S));
        cp_async16(sbase + (uint32_t)((k * 1024 + row * 16) * sizeof(S) + part * 16), src);
      }
    }
  };

  S* __restrict__ fout = static_cast<S*>(a.f_out);
  T* __restrict__ rho_out = static_cast<T*>(a.rho_out);
  T* __restrict__ vel_out = static_cast<T*>(a.vel_out);
  const T* __restrict__ vel_in = static_cast<const T*>(a.vel_in);
  const int64_t kst = a.f_kstride, vcs = a.v_cstride;
  const int n_real = a.n_blocks;
  const int x = tid & 7, y = (tid >> 3) & 7, z0 = tid >> 6, z1 = z0 + 4;

  int w = blockIdx.x;
  if (w < n_work) issue(w, 0);
  cp_async_commit();
  for (int it = 0; w < n_work; w += gridDim.x, ++it) {
    const int s = it & 1;
    const int wn = w + gridDim.x;
    // stage s^1 was last read before the barrier that ended the previous iteration
    if (wn < n_work) issue(wn, s ^ 1);
    cp_async_commit();
    const int b = work[w];
    if (tid < 27) s_nbr[s][tid] = a.nbr[(int64_t)b * 27 + tid];
    if (tid == 32) s_bi[s] = a.binfo[b];
    cp_async_wait1();  // this thread's copies of block w have landed
    __syncthreads();   // ... and every other thread's
    const S* st = s ? stage1 : stage0;
    const int4 bi = s_bi[s];
    const int32_t* nb_row = s_nbr[s];

    // ---- pull from shared memory (the boxes are already shifted by -c_k) ----
    V A[kQ27];
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      const int W = dense_w(k);
      const S* p = st + dense_off(k) + dense_xo(k) + x + y * W;
      A[k] = dec2<S>(p[z0 * 8 * W], p[z1 * 8 * W], k);
    }
    V rho = A[0], jx = splat<V>(T(0)), jy = splat<V>(T(0)), jz = splat<V>(T(0));
#pragma unroll
    for (int k = 1; k < kQ27; ++k) rho = rho + A[k];
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      if (q27_cx(k)) jx = q27_cx(k) > 0 ? jx + A[k] : jx - A[k];
      if (q27_cy(k)) jy = q27_cy(k) > 0 ? jy + A[k] : jy - A[k];
      if (q27_cz(k)) jz = q27_cz(k) > 0 ? jz + A[k] : jz - A[k];
    }
    rho = vmaxc(rho, T(0.01));
    const V inv_rho = vrcp(rho);
    const V ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
    const int64_t v0 = (int64_t)b * kCells + (x | (y << 3) | (z0 << 6)), v1 = v0 + 256;
    {
      float r0, r1, a0, a1;
      f2split(rho, r0, r1); rho_out[v0] = r0; rho_out[v1] = r1;
      f2split(ux, a0, a1); vel_out[v0] = a0; vel_out[v1] = a1;
      f2split(uy, a0, a1); vel_out[v0 + vcs] = a0; vel_out[v1 + vcs] = a1;
      f2split(uz, a0, a1); vel_out[v0 + 2 * vcs] = a0; vel_out[v1 + 2 * vcs] = a1;
    }

    // ---- WALE from the previous step's velocity (kernel_cumulant.jl:496-549) ----
    V nu_eddy = splat<V>(T(0));
    if (cp.flags & CF_GRADIENTS) {
      auto nbv = [&](int dx, int dy, int dz, int c) -> V {
        T v[2];
        const int zl[2] = {z0, z1};
        const int64_t own[2] = {v0, v1};
#pragma unroll
        for (int l = 0; l < 2; ++l) {
          const int nx = x + dx, ny = y + dy, nz = zl[l] + dz;
          const int nb = nb_row[nbr_dir(nx >> 3, ny >> 3, nz >> 3)];
          const int64_t i = nb < n_real ? (int64_t)nb * kCells + ((nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6)) : own[l];
          v[l] = vel_in[i + c * vcs];
        }
        return f2(v[0], v[1]);
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

    // ---- store into the padded grid ----
    const int64_t o0 = dense_idx(a, (bi.x - 1) * kBS + 8 + x, (bi.y - 1) * kBS + 1 + y, (bi.z - 1) * kBS + 1 + z0);
    const int64_t dz4 = (int64_t)4 * a.PX * a.PY;
#pragma unroll
    for (int k = 0; k < kQ27; ++k) enc2_store<S>(fout, o0 + k * kst, o0 + k * kst + dz4, A[k], k);
    __syncthreads();  // stage s is free for the loads issued at the start of iteration it + 1
  }
}

// Resident CTAs per SM the register budget is sized for (two stages of 55 KB fit twice per SM in
// 16-bit storage; 110 KB stages in FP32 fit once).
#ifndef OAL_DENSE_MIN_CTAS
#define OAL_DENSE_MIN_CTAS 1
#endif
template <class S>
constexpr int dense_min_ctas() { return sizeof(S) == 2 ? OAL_DENSE_MIN_CTAS : 1; }

template <class S>
size_t dense_smem_bytes() { return 2 * (size_t)kDenseStageElems * sizeof(S) + 128; }

template <class S>
cudaError_t launch_dense_fast(const StepArgs& a, const int32_t* work, int n_work, int grid, cudaStream_t st) {
  if (n_work <= 0) return cudaSuccess;
  constexpr int MINB = dense_min_ctas<S>();
  static bool attr_set[64] = {};  // the attribute is set once per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !attr_set[dev]) {
    cudaError_t e = cudaFuncSetAttribute(k_dense_fast<S, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)dense_smem_bytes<S>());
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  const int g = grid < n_work ? grid : n_work;
  k_dense_fast<S, MINB><<<g, 256, dense_smem_bytes<S>(), st>>>(a, work, n_work);
  return cudaGetLastError();
}

// CTAs per SM the kernel is built for (grid = SMs x this)
template <class S>
int dense_ctas_per_sm() { return dense_min_ctas<S>(); }

template cudaError_t launch_dense_fast<float>(const StepArgs&, const int32_t*, int, int, cudaStream_t);
template cudaError_t launch_dense_fast<__half>(const StepArgs&, const int32_t*, int, int, cudaStream_t);
template cudaError_t launch_dense_fast<__nv_bfloat16>(const StepArgs&, const int32_t*, int, int, cudaStream_t);
template int dense_ctas_per_sm<float>();
template int dense_ctas_per_sm<__half>();
template int dense_ctas_per_sm<__nv_bfloat16>();

}  // namespace oal
