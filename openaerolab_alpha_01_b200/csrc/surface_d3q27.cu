// surface_d3q27.cu — surface-stress force mapping of a D3Q27 level: the reference's
// compute_aerodynamics! (src/forces/surface.jl:1577-1587) with its default Prandtl force method.
//
// map_stresses_kernel! (surface.jl:636-1031): one thread per triangle walks probe points
// t + n (i + 1/2), i = 1..search_radius, along the triangle's outward normal; each probe is a
// trilinear sample of density and velocity over the fluid corners of its cell stencil
// (trilinear_sample_flow, :502-634; quality = the fluid corners' weight). The closest probe of
// quality >= 1/4 gives the shear sample (else the best lower-quality one); the first
// min(4, radius) good probes give a quality-weighted (Shepard) density for the pressure. A closed
// body whose supplied side finds no fluid tries the opposite side (normal sign -1); a triangle
// still without fluid takes the nearest fluid cell of growing cubic shells on its outward side.
// compute_stress_from_cell (:180-269): gauge pressure (rho - 1) cs^2, wall shear
// rho nu_eff u_t / max(d, 1) with nu_eff = nu + min(max(c_w^2 u_t / max(d, 1), nu_bg), 20 nu).
// integrate_forces_kernel! (:1265-1331): dF = -p n A (pressure) + tau A (viscous), moments about
// the moment centre; the reference adds these with Float32 atomics in arbitrary order, here they
// are written per triangle in FP64 and summed in a fixed order (deterministic).
//
// Every operation is a single IEEE binary32 operation in the reference's order (the library is
// built with -fmad=false; division and square root are correctly rounded), so each triangle's
// values are those of the CPU restatement bit for bit.
#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "surface_d3q27.h"

namespace oal {

__device__ __forceinline__ int64_t cell_at(const SurfArgs& a, int gx, int gy, int gz) {
  if (gx < 1 || gy < 1 || gz < 1) return -1;
  const int bx = (gx - 1) / kBS + 1, by = (gy - 1) / kBS + 1, bz = (gz - 1) / kBS + 1;
  if (bx > a.dim_x || by > a.dim_y || bz > a.dim_z) return -1;
  const int32_t b = a.ptr[(bx - 1) + (int64_t)a.dim_x * ((by - 1) + (int64_t)a.dim_y * (bz - 1))];
  if (b <= 0) return -1;
  return (int64_t)(b - 1) * kCells + (((gx - 1) % kBS) | (((gy - 1) % kBS) << 3) | (((gz - 1) % kBS) << 6));
}

__device__ __forceinline__ bool solid_at(const SurfArgs& a, int64_t c) {
  const int32_t s = a.mslot[c >> 9];
  return s >= 0 && ((a.cmask[(int64_t)s * kCells + (c & 511)] >> 13) & 1u);
}

template <class R>
__device__ __forceinline__ float rho_at(const SurfArgs& a, int64_t c) { return float(static_cast<const R*>(a.rho)[c]); }
template <class R>
__device__ __forceinline__ float vel_at(const SurfArgs& a, int64_t c, int comp) {
  return float(static_cast<const R*>(a.vel)[c + comp * a.vcs]);
}

__device__ __forceinline__ float jclampf(float v, float lo, float hi) { return v > hi ? hi : (v < lo ? lo : v); }

// trilinear_sample_flow (surface.jl:502-634), dx = 1
template <class R>
__device__ bool sample_flow(const SurfArgs& a, float px, float py, float pz, float& r, float& ux, float& uy, float& uz,
                            float& wq) {
  const float fx = px - 0.5f, fy = py - 0.5f, fz = pz - 0.5f;
  const int ix0 = (int)floorf(fx) + 1, iy0 = (int)floorf(fy) + 1, iz0 = (int)floorf(fz) + 1;
  const float wx = jclampf(fx - float(ix0 - 1), 0.0f, 1.0f);
  const float wy = jclampf(fy - float(iy0 - 1), 0.0f, 1.0f);
  const float wz = jclampf(fz - float(iz0 - 1), 0.0f, 1.0f);
  const float w0x = 1.0f - wx, w1x = wx, w0y = 1.0f - wy, w1y = wy, w0z = 1.0f - wz, w1z = wz;
  float ra = 0.0f, xa = 0.0f, ya = 0.0f, za = 0.0f, wa = 0.0f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
    const float wk = (ox ? w1x : w0x) * (oy ? w1y : w0y) * (oz ? w1z : w0z);
    const int64_t e = cell_at(a, ix0 + ox, iy0 + oy, iz0 + oz);
    if (e >= 0 && !solid_at(a, e)) {
      ra += wk * rho_at<R>(a, e);
      xa += wk * vel_at<R>(a, e, 0);
      ya += wk * vel_at<R>(a, e, 1);
      za += wk * vel_at<R>(a, e, 2);
      wa += wk;
    }
  }
  if (wa > 0.01f) {
    const float inv = 1.0f / wa;
    r = ra * inv; ux = xa * inv; uy = ya * inv; uz = za * inv;
    if (!isfinite(r) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz)) { r = 1.0f; ux = uy = uz = 0.0f; wq = 0.0f; return false; }
    wq = wa;
    return true;
  }
  r = 1.0f; ux = uy = uz = 0.0f; wq = 0.0f;
  return false;
}

// compute_stress_from_cell (surface.jl:180-269), athermal (T = 1)
__device__ void stress_from_cell(float rho, float ux, float uy, float uz, float nx, float ny, float nz, float dist,
                                 const SurfArgs& a, float& p, float& tx, float& ty, float& tz) {
  p = tx = ty = tz = 0.0f;
  if (!isfinite(rho) || rho < 0.01f || rho > 10.0f) return;
  if (!isfinite(ux) || !isfinite(uy) || !isfinite(uz)) return;
  const float umag2 = ux * ux + uy * uy + uz * uz;
  if (umag2 > 100.0f) return;
  const float p_phys = ((rho * 1.0f - 1.0f) * a.cs2) * a.pscale;
  const float udn = ux * nx + uy * ny + uz * nz;
  const float utx = ux - udn * nx, uty = uy - udn * ny, utz = uz - udn * nz;
  const float ut = sqrtf(utx * utx + uty * uty + utz * utz);
  const float nu_mol = (a.tau - 0.5f) * a.cs2;
  float nu_sgs = 0.0f;
  const float dw = fmaxf(dist, 1.0f);
  if (a.c_wale > 0.0f && ut > 1e-10f) nu_sgs = (a.c_wale * a.c_wale) * (ut / dw);
  nu_sgs = nu_sgs < a.nu_bg ? a.nu_bg : nu_sgs;
  nu_sgs = nu_sgs > 20.0f * nu_mol ? 20.0f * nu_mol : nu_sgs;
  const float nu_eff = nu_mol + nu_sgs;
  float sx = 0.0f, sy = 0.0f, sz = 0.0f;
  if (ut > 1e-10f && dist > 0.01f) {
    const float tmag = rho * nu_eff * ut / dw * a.sscale;
    sx = (utx / ut) * tmag; sy = (uty / ut) * tmag; sz = (utz / ut) * tmag;
  }
  if (!isfinite(p_phys) || !isfinite(sx) || !isfinite(sy) || !isfinite(sz)) return;
  p = p_phys; tx = sx; ty = sy; tz = sz;
}

template <class R>
__global__ void __launch_bounds__(128) k_surface_map(const SurfArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const float* t = a.tri + (int64_t)i * 7;
  const float tx = t[0], ty = t[1], tz = t[2];
  float nx = t[3], ny = t[4], nz = t[5];
  const float area = t[6];
  float best_rho = 1.0f, bux = 0.0f, buy = 0.0f, buz = 0.0f, best_wd = float(a.radius + 1), best_q = 0.0f;
  bool found = false;
  float prho = 0.0f, pT = 0.0f, pw = 0.0f;
  const float min_q = 0.25f;
  const int ppm = a.radius < 4 ? a.radius : 4;
  for (int pi = 1; pi <= a.radius; ++pi) {
    const float d = float(pi) + 0.5f;
    float r, ux, uy, uz, wq;
    const bool ok = sample_flow<R>(a, tx + nx * d * 1.0f, ty + ny * d * 1.0f, tz + nz * d * 1.0f, r, ux, uy, uz, wq);
    if (ok && wq >= min_q && pi <= ppm) { prho += wq * r; pT += wq * 1.0f; pw += wq; }
    if (ok && wq >= min_q) {
      if (!found) { best_rho = r; bux = ux; buy = uy; buz = uz; best_wd = d; best_q = wq; found = true; }
      if (pi >= ppm) break;
    } else if (ok && wq > best_q && !found) {
      best_rho = r; bux = ux; buy = uy; buz = uz; best_wd = d; best_q = wq; found = true;
    }
  }
  float nsign = 1.0f;
  if (!found && a.recover) {
    for (int pi = 1; pi <= ppm; ++pi) {
      const float d = float(pi) + 0.5f;
      float r, ux, uy, uz, wq;
      const bool ok = sample_flow<R>(a, tx - nx * d * 1.0f, ty - ny * d * 1.0f, tz - nz * d * 1.0f, r, ux, uy, uz, wq);
      if (ok && wq >= min_q) {
        prho += wq * r; pT += wq * 1.0f; pw += wq;
        if (!found) { best_rho = r; bux = ux; buy = uy; buz = uz; best_wd = d; best_q = wq; found = true; nsign = -1.0f; }
      }
    }
    if (nsign < 0.0f) { nx = -nx; ny = -ny; nz = -nz; }
  }
  if (!found) {
    const int gx = (int)floorf(tx / 1.0f) + 1, gy = (int)floorf(ty / 1.0f) + 1, gz = (int)floorf(tz / 1.0f) + 1;
    float best_d2 = 1e10f;
    for (int rad = 1; rad <= a.radius && !found; ++rad)
      for (int dz = -rad; dz <= rad; ++dz)
        for (int dy = -rad; dy <= rad; ++dy)
          for (int dx = -rad; dx <= rad; ++dx) {
            if (!(abs(dx) == rad || abs(dy) == rad || abs(dz) == rad)) continue;
            const int cgx = gx + dx, cgy = gy + dy, cgz = gz + dz;
            const int64_t e = cell_at(a, cgx, cgy, cgz);
            if (e < 0 || solid_at(a, e)) continue;
            const float cr = rho_at<R>(a, e);
            if (!isfinite(cr) || cr < 0.01f || cr > 100.0f) continue;
            const float ccx = (float(cgx) - 0.5f) * 1.0f, ccy = (float(cgy) - 0.5f) * 1.0f, ccz = (float(cgz) - 0.5f) * 1.0f;
            const float ddx = ccx - tx, ddy = ccy - ty, ddz = ccz - tz;
            const float dn = ddx * nx + ddy * ny + ddz * nz;
            if (dn <= 0.0f) continue;
            const float d2 = ddx * ddx + ddy * ddy + ddz * ddz;
            if (d2 < best_d2) {
              best_d2 = d2;
              best_rho = cr; bux = vel_at<R>(a, e, 0); buy = vel_at<R>(a, e, 1); buz = vel_at<R>(a, e, 2);
              best_wd = dn / 1.0f;
              found = true;
            }
          }
  }
  const float p_rho = pw > 0.5f ? prho / pw : best_rho;
  const float p_T = pw > 0.5f ? pT / pw : 1.0f;
  float p = __int_as_float(0x7fc00000), sx = 0.0f, sy = 0.0f, sz = 0.0f;
  if (found) {
    const float wd = fmaxf(best_wd, 0.5f);
    stress_from_cell(best_rho, bux, buy, buz, nx, ny, nz, wd, a, p, sx, sy, sz);
    if (isfinite(p_rho) && p_rho >= 0.01f && p_rho <= 10.0f && isfinite(p_T) && p_T >= 0.1f && p_T <= 10.0f)
      p = (p_rho * p_T - 1.0f) * a.cs2 * a.pscale;
  }
  float* o = a.out + (int64_t)i * 6;
  o[0] = p; o[1] = sx; o[2] = sy; o[3] = sz; o[4] = nsign; o[5] = found ? best_wd * 1.0f : 0.0f;
  // integrate_forces_kernel!: the stored normal (nsign applied) and the triangle's contribution
  double* q = a.part + (int64_t)i * 9;
  if (isfinite(p) && isfinite(sx) && isfinite(sy) && isfinite(sz)) {
    const float mx = t[3] * nsign, my = t[4] * nsign, mz = t[5] * nsign;
    const float fpx = -p * mx * area, fpy = -p * my * area, fpz = -p * mz * area;
    const float fvx = sx * area, fvy = sy * area, fvz = sz * area;
    const float fx = fpx + fvx, fy = fpy + fvy, fz = fpz + fvz;
    const float rx = tx - a.mcx, ry = ty - a.mcy, rz = tz - a.mcz;
    q[0] = fpx; q[1] = fpy; q[2] = fpz; q[3] = fvx; q[4] = fvy; q[5] = fvz;
    q[6] = ry * fz - rz * fy; q[7] = rz * fx - rx * fz; q[8] = rx * fy - ry * fx;
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c) q[c] = 0.0;
  }
}

// fixed-order sum of n rows of 9 doubles (strided per thread, then a fixed tree)
__global__ void k_surface_sum(const double* __restrict__ part, int32_t n, double* __restrict__ out) {
  __shared__ double s[9][256];
  const int t = threadIdx.x;
  double acc[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) acc[c] = 0.0;
  for (int64_t i = t; i < n; i += 256)
#pragma unroll
    for (int c = 0; c < 9; ++c) acc[c] += part[i * 9 + c];
#pragma unroll
  for (int c = 0; c < 9; ++c) s[c][t] = acc[c];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w)
#pragma unroll
      for (int c = 0; c < 9; ++c) s[c][t] += s[c][t + w];
    __syncthreads();
  }
  if (t < 9) out[t] = s[t][0];
}

cudaError_t launch_surface(const SurfArgs& a, bool dbl, double* d_out9, cudaStream_t st) {
  if (a.n <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((a.n + 127) / 128);
  if (dbl) k_surface_map<double><<<grid, 128, 0, st>>>(a);
  else k_surface_map<float><<<grid, 128, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_surface_sum<<<1, 256, 0, st>>>(a.part, a.n, d_out9);
  return cudaGetLastError();
}

}  // namespace oal
