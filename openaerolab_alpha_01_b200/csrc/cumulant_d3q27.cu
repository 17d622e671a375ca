// cumulant_d3q27.cu — fused pull-stream + D3Q27 cumulant collision (+ WALE, sponge, wall model,
// Guo forcing, half-way bounce-back with FP64 momentum exchange) for 8^3-cell blocks on sm_100a.
//
// Behaviour follows the reference's `stream_collide_cumulant!` (src/collision/kernel_cumulant.jl:
// 29-912) for a level without a parent (is_level_1): pull of 27 populations through the 27-entry
// neighbour table (:190-400), full-way bounce-back inside obstacle cells (:402-417), macros,
// sponge and wall model (:420-491), WALE eddy viscosity from the previous step's velocity
// (:496-595), cumulant relaxation with adaptive omega_4 and the factored limiter (:597-844),
// positivity limiter (:849-884) and Guo forcing (:889-908). The half-way link rule with momentum
// exchange is the octree solver's (src/octree_q19/src/stream.jl:229-256) on the 27 links.
//
// Launch shape: one CTA of 128 threads per 8x8x2 slab (four CTAs per block). Blocks whose 26
// neighbours all exist and that touch no solid take a branch-free pull; the others take the
// general path with the domain-face conditions and the per-cell solid masks.
#include "common.cuh"

namespace oal {

// kernel_cumulant.jl:4-14
template <class R>
__device__ __forceinline__ void chimera_fwd(R& a, R& b, R& c, R u) {
  const R m0 = a + b + c, m1 = c - a, m2 = a + c;
  a = m0;
  b = m1 - u * m0;
  c = m2 - R(2) * u * m1 + u * u * m0;
}
// kernel_cumulant.jl:16-26
template <class R>
__device__ __forceinline__ void chimera_bwd(R& a, R& b, R& c, R u) {
  const R m0 = a;
  const R m1 = b + u * a;
  const R m2 = c + R(2) * u * b + u * u * a;
  a = (m2 - m1) * R(0.5);
  b = m0 - m2;
  c = (m2 + m1) * R(0.5);
}

// physics_utils.jl:30-109 (O(u^4) limiter gate off, the reference default build)
template <class R>
__device__ __forceinline__ R feq_auto(R rho, R ux, R uy, R uz, R w, R cx, R cy, R cz, bool comp) {
  const R cu = cx * ux + cy * uy + cz * uz;
  const R usq = ux * ux + uy * uy + uz * uz;
  R val = R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq;
  if (comp) {
    const R cu2 = cu * cu;
    val += (R(4.5) * cu2 * cu - R(4.5) * cu * usq) + (R(3.375) * cu2 * cu2 - R(6.75) * cu2 * usq + R(1.125) * usq * usq);
  }
  return rho * w * val;
}

// physics_utils.jl:5-17
__device__ __forceinline__ float gradient_noise(int32_t gx, int32_t gy, int32_t gz, int32_t seed) {
  uint32_t c = (uint32_t)gx * 374761393u + (uint32_t)gy * 668265263u + (uint32_t)gz * 1274126177u + (uint32_t)seed;
  uint32_t h = c;
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  h = h ^ (h >> 16);
  return ((float)(h & 0xFFFFu) / 32768.0f) - 1.0f;
}

// Population arriving from outside every block of the level (kernel_cumulant.jl:221-391), level 1.
template <class S, class R>
__device__ __noinline__ R face_population(const S* __restrict__ fin, int64_t bbase, int cell, int64_t kst,
                                           const int32_t* s_nbr, int64_t bst, int k, int x, int y, int z, int gx,
                                           int gy, int gz, const CaseParams& cp) {
  const int64_t own = bbase + cell;
  const int cx = q27_cx(k), cy = q27_cy(k), cz = q27_cz(k);
  const R w = R(q27_w(k));
  const int src_gx = gx - cx, src_gy = gy - cy, src_gz = gz - cz;
  const bool is_inlet = src_gx < 1, is_outlet = src_gx > cp.nx;
  const bool is_y_min = src_gy < 1, is_y_max = src_gy > cp.ny;
  const bool is_z_min = src_gz < 1, is_z_max = src_gz > cp.nz;
  const bool comp = (cp.flags & CF_COMPRESSIBLE) != 0;
  auto own_k = [&](int j) -> R { return Codec<S>::dec(fin[own + j * kst], R(q27_w(j)), R(1.0 / q27_w(j))); };
  if (is_inlet) {
    const float noise = (cp.flags & CF_INLET_NOISE)
                            ? gradient_noise(gy, gz, cp.time_step_seed, 1234) * cp.inlet_turbulence * cp.u_inlet
                            : 0.0f;
    const R u_inst = R(cp.u_inlet) + R(noise);
    return feq_auto<R>(R(1), u_inst, R(0), R(0), w, R(cx), R(cy), R(cz), comp);
  }
  if (is_outlet) return own_k(k);
  if ((cp.flags & (CF_ZWALL_SLIP | CF_ZWALL_NOSLIP)) && (is_z_min || is_z_max)) {
    if (cp.flags & CF_ZWALL_NOSLIP) return own_k(q27_opp(k));
    const int zw_k = q27_mir_z(k);
    const int zw_ix = x - cx, zw_iy = y - cy;
    if (zw_ix >= 0 && zw_ix < kBS && zw_iy >= 0 && zw_iy < kBS) {
      const int64_t zc = zw_ix + 8 * zw_iy + 64 * z;
      return Codec<S>::dec(fin[bbase + zc + zw_k * kst], R(q27_w(zw_k)), R(1.0 / q27_w(zw_k)));
    }
    const int zw_ox = zw_ix >> 3, zw_oy = zw_iy >> 3;
    const int zw_nb = s_nbr[nbr_dir(zw_ox, zw_oy, 0)];
    if (zw_nb >= 0) {
      const int64_t zc = (zw_ix & 7) + 8 * (zw_iy & 7) + 64 * z;
      return Codec<S>::dec(fin[zw_nb * bst + zw_k * kst + zc], R(q27_w(zw_k)), R(1.0 / q27_w(zw_k)));
    }
    return own_k(zw_k);
  }
  if ((cp.flags & CF_TRANSVERSE_FS) && (is_y_min || is_y_max || is_z_min || is_z_max)) {
    const R beta = R(cp.transverse_blend);
    const R donor = own_k(k);
    const R fe = feq_auto<R>(R(1), R(cp.u_inlet), R(0), R(0), w, R(cx), R(cy), R(cz), comp);
    return (R(1) - beta) * donor + beta * fe;
  }
  if (is_y_min && (cp.flags & CF_YMIN_WALL)) return own_k(q27_opp(k));
  if (is_y_min || is_y_max) return own_k(q27_mir_y(k));
  if (is_z_min || is_z_max) return own_k(q27_mir_z(k));
  return w;  // level 1: lattice weight (kernel_cumulant.jl:389-391)
}

// Velocity of a face neighbour for the WALE stencil (physics_utils.jl:2001-2035): the own value
// when the neighbour block is missing or the neighbour cell is solid.
template <class R, bool G>
__device__ __forceinline__ void vel_neighbour(const R* __restrict__ vin, int64_t vcs, const int32_t* s_nbr, int b,
                                              int x, int y, int z, int dx, int dy, int dz, uint32_t solid_bit,
                                              R u0, R v0, R w0, R& u, R& v, R& w) {
  const int nx = x + dx, ny = y + dy, nz = z + dz;
  const int nb = (dx | dy | dz) ? s_nbr[nbr_dir(nx >> 3, ny >> 3, nz >> 3)] : b;
  if (G && (nb < 0 || solid_bit)) { u = u0; v = v0; w = w0; return; }
  const int64_t i = (int64_t)nb * kCells + ((nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6));
  u = vin[i]; v = vin[i + vcs]; w = vin[i + 2 * vcs];
}

template <class S, class R, bool G>
__device__ __forceinline__ void cell_step(const StepArgs& a, const CaseParams& cp, const int32_t* s_nbr, int b,
                                          int gx0, int gy0, int gz0, uint32_t bflags, int x, int y, int z,
                                          double& mx, double& my, double& mz) {
  const S* __restrict__ fin = static_cast<const S*>(a.f_in);
  S* __restrict__ fout = static_cast<S*>(a.f_out);
  R* __restrict__ rho_out = static_cast<R*>(a.rho_out);
  R* __restrict__ vel_out = static_cast<R*>(a.vel_out);
  const R* __restrict__ vel_in = static_cast<const R*>(a.vel_in);
  const int64_t bst = a.f_bstride, kst = a.f_kstride, vcs = a.v_cstride;
  const int cell = x | (y << 3) | (z << 6);
  const int64_t own = (int64_t)b * bst + cell;
  const int64_t vown = (int64_t)b * kCells + cell;
  const uint32_t flags = cp.flags;

  uint32_t mask = 0;
  if (G && (bflags & BF_NEAR_SOLID)) mask = a.cmask[(int64_t)a.mslot[b] * kCells + cell];
  const bool is_obs = G && ((mask >> 13) & 1u);
  const bool halfway = (flags & CF_HALFWAY) != 0;

  if (G && is_obs && halfway) {
    // half-way mode: a solid cell holds the rest equilibrium; no fluid cell reads it
#pragma unroll
    for (int k = 0; k < kQ27; ++k) fout[own + k * kst] = Codec<S>::enc(R(q27_w(k)), R(q27_w(k)), R(1.0 / q27_w(k)));
    if ((flags & CF_STORE_POST) && a.f_post) {
      S* fp = static_cast<S*>(a.f_post);
#pragma unroll
      for (int k = 0; k < kQ27; ++k) fp[own + k * kst] = Codec<S>::enc(R(q27_w(k)), R(q27_w(k)), R(1.0 / q27_w(k)));
    }
    rho_out[vown] = R(1);
    vel_out[vown] = R(0); vel_out[vown + vcs] = R(0); vel_out[vown + 2 * vcs] = R(0);
    return;
  }

  // ---- STEP 1: pull (kernel_cumulant.jl:190-400) ----
  R A[kQ27];
  R rho = R(0), jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const int cx = q27_cx(k), cy = q27_cy(k), cz = q27_cz(k);
    const int sx = x - cx, sy = y - cy, sz = z - cz;
    const int nb = s_nbr[nbr_dir(sx >> 3, sy >> 3, sz >> 3)];
    const R w = R(q27_w(k)), iw = R(1.0 / q27_w(k));
    R val;
    if (!G) {
      val = Codec<S>::dec(fin[(int64_t)nb * bst + k * kst + ((sx & 7) | ((sy & 7) << 3) | ((sz & 7) << 6))], w, iw);
    } else if (nb >= 0) {
      if (halfway && ((mask >> k) & 1u)) {
        // the link opp(k) of this cell is cut: its own post-collision population returns
        const int i = q27_opp(k);
        const R fi = Codec<S>::dec(fin[own + i * kst], R(q27_w(i)), R(1.0 / q27_w(i)));
        val = fi;
        if (flags & CF_COLLECT) {
          const double mom = 2.0 * (double)fi;  // (f_i* + f_k(t+1)) c_i, c_i = -c_k
          mx -= mom * cx; my -= mom * cy; mz -= mom * cz;
        }
      } else {
        val = Codec<S>::dec(fin[(int64_t)nb * bst + k * kst + ((sx & 7) | ((sy & 7) << 3) | ((sz & 7) << 6))], w, iw);
      }
    } else {
      val = face_population<S, R>(fin, (int64_t)b * bst, cell, kst, s_nbr, bst, k, x, y, z, gx0 + x, gy0 + y,
                                  gz0 + z, cp);
    }
    A[k] = val;
    rho += val;
    if (cx) jx += cx > 0 ? val : -val;
    if (cy) jy += cy > 0 ? val : -val;
    if (cz) jz += cz > 0 ? val : -val;
  }

  const bool store_post = (flags & CF_STORE_POST) && a.f_post;
  if (G && is_obs) {
    // simple bounce-back inside the obstacle (kernel_cumulant.jl:402-417)
    rho_out[vown] = R(1);
    vel_out[vown] = R(0); vel_out[vown + vcs] = R(0); vel_out[vown + 2 * vcs] = R(0);
#pragma unroll
    for (int k = 0; k < kQ27; ++k) {
      const R w = R(q27_w(k)), iw = R(1.0 / q27_w(k));
      fout[own + k * kst] = Codec<S>::enc(A[q27_opp(k)], w, iw);
      if (store_post) static_cast<S*>(a.f_post)[own + k * kst] = Codec<S>::enc(A[q27_opp(k)], w, iw);
    }
    return;
  }

  // ---- STEP 2: macros, sponge, wall model (kernel_cumulant.jl:420-491) ----
  rho = rho > R(0.01) ? rho : R(0.01);
  const R inv_rho = R(1) / rho;
  R ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  const bool comp = (flags & CF_COMPRESSIBLE) != 0;
  if (G && a.sponge) {
    const R sp = R(a.sponge[vown]);
    if (sp > R(0)) {
      const R ut = R(cp.u_inlet);
      rho = rho * (R(1) - sp) + R(1) * sp;
      ux = ux * (R(1) - sp) + ut * sp;
      uy = uy * (R(1) - sp);
      uz = uz * (R(1) - sp);
      if (flags & CF_SPONGE_BLEND) {
#pragma unroll
        for (int k = 0; k < kQ27; ++k) {
          const R fe = feq_auto<R>(R(1), ut, R(0), R(0), R(q27_w(k)), R(q27_cx(k)), R(q27_cy(k)), R(q27_cz(k)), comp);
          A[k] = A[k] * (R(1) - sp) + fe * sp;
        }
      }
    }
  }
  R Fx = R(0), Fy = R(0), Fz = R(0);
  if (G && (flags & CF_WALL_MODEL) && a.wall_dist) {
    const R dw = R(a.wall_dist[vown]);
    if (dw > R(0) && dw < R(cp.wall_model_max_distance)) {
      const R u_mag = sqrt(ux * ux + uy * uy + uz * uz);
      const R nu_visc = (R(cp.tau) - R(0.5)) / R(3);
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
  const R ux_eq = ux + R(0.5) * Fx * inv_rho;
  const R uy_eq = uy + R(0.5) * Fy * inv_rho;
  const R uz_eq = uz + R(0.5) * Fz * inv_rho;
  rho_out[vown] = rho;
  vel_out[vown] = ux; vel_out[vown + vcs] = uy; vel_out[vown + 2 * vcs] = uz;

  // ---- STEP 3: WALE -> omega_1 (kernel_cumulant.jl:496-595, background SGS path) ----
  R nu_eddy = R(0);
  if (flags & CF_GRADIENTS) {
    const R u0 = vel_in[vown], v0 = vel_in[vown + vcs], w0 = vel_in[vown + 2 * vcs];
    R uE, vE, wE, uW, vW, wW, uN, vN, wN, uS, vS, wS, uT, vT, wT, uB, vB, wB;
    vel_neighbour<R, G>(vel_in, vcs, s_nbr, b, x, y, z, 1, 0, 0, (mask >> 12) & 1u, u0, v0, w0, uE, vE, wE);
    vel_neighbour<R, G>(vel_in, vcs, s_nbr, b, x, y, z, -1, 0, 0, (mask >> 14) & 1u, u0, v0, w0, uW, vW, wW);
    vel_neighbour<R, G>(vel_in, vcs, s_nbr, b, x, y, z, 0, 1, 0, (mask >> 10) & 1u, u0, v0, w0, uN, vN, wN);
    vel_neighbour<R, G>(vel_in, vcs, s_nbr, b, x, y, z, 0, -1, 0, (mask >> 16) & 1u, u0, v0, w0, uS, vS, wS);
    vel_neighbour<R, G>(vel_in, vcs, s_nbr, b, x, y, z, 0, 0, 1, (mask >> 4) & 1u, u0, v0, w0, uT, vT, wT);
    vel_neighbour<R, G>(vel_in, vcs, s_nbr, b, x, y, z, 0, 0, -1, (mask >> 22) & 1u, u0, v0, w0, uB, vB, wB);
    const R h = R(0.5);
    const R g11 = h * (uE - uW), g12 = h * (uN - uS), g13 = h * (uT - uB);
    const R g21 = h * (vE - vW), g22 = h * (vN - vS), g23 = h * (vT - vB);
    const R g31 = h * (wE - wW), g32 = h * (wN - wS), g33 = h * (wT - wB);
    const R gsq11 = g11 * g11 + g12 * g21 + g13 * g31;
    const R gsq12 = g11 * g12 + g12 * g22 + g13 * g32;
    const R gsq13 = g11 * g13 + g12 * g23 + g13 * g33;
    const R gsq21 = g21 * g11 + g22 * g21 + g23 * g31;
    const R gsq22 = g21 * g12 + g22 * g22 + g23 * g32;
    const R gsq23 = g21 * g13 + g22 * g23 + g23 * g33;
    const R gsq31 = g31 * g11 + g32 * g21 + g33 * g31;
    const R gsq32 = g31 * g12 + g32 * g22 + g33 * g32;
    const R gsq33 = g31 * g13 + g32 * g23 + g33 * g33;
    const R tr = (gsq11 + gsq22 + gsq33) / R(3);
    const R Sd11 = gsq11 - tr, Sd22 = gsq22 - tr, Sd33 = gsq33 - tr;
    const R Sd12 = R(0.5) * (gsq12 + gsq21), Sd13 = R(0.5) * (gsq13 + gsq31), Sd23 = R(0.5) * (gsq23 + gsq32);
    const R S12 = R(0.5) * (g12 + g21), S13 = R(0.5) * (g13 + g31), S23 = R(0.5) * (g23 + g32);
    const R OP1 = Sd11 * Sd11 + Sd22 * Sd22 + Sd33 * Sd33 + R(2) * (Sd12 * Sd12 + Sd13 * Sd13 + Sd23 * Sd23);
    const R OP2 = g11 * g11 + g22 * g22 + g33 * g33 + R(2) * (S12 * S12 + S13 * S13 + S23 * S23);
    if (OP1 > R(1e-12)) {
      const R OP1_32 = OP1 * sqrt(OP1);
      const R OP2_52 = OP2 * OP2 * sqrt(OP2 > R(1e-12) ? OP2 : R(1e-12));
      const R den = OP2_52 + OP1 * sqrt(sqrt(OP1 > R(1e-12) ? OP1 : R(1e-12)));
      if (den > R(1e-12)) nu_eddy = (R(cp.c_wale) * R(cp.c_wale)) * OP1_32 / den;
    }
    nu_eddy = nu_eddy * R(cp.amr_sgs_scale);
  }
  {
    const R bg = R(cp.nu_sgs_bg) * R(cp.amr_sgs_scale);
    nu_eddy = nu_eddy > bg ? nu_eddy : bg;
  }
  const R nu_mol = (R(cp.tau) - R(0.5)) / R(3);
  const R tau_eff = R(0.5) + R(3) * (nu_mol + nu_eddy);
  const R omega1 = R(1) / (tau_eff > R(0.500001) ? tau_eff : R(0.500001));
  const R omega_bulk = R(cp.omega_bulk), omega3 = R(cp.omega3), omega4 = R(cp.omega4);
  R omega4_diag = omega4;
  if (flags & CF_ADAPTIVE_OMEGA4) {
    const R om = omega1 - R(2);
    const R Av = -(om * om) / (R(cp.lambda_param) * omega1 + R(1e-10));
    omega4_diag = Av < R(0.01) ? R(0.01) : (Av > R(2) ? R(2) : Av);
  }

  // ---- STEP 4: chimera forward (kernel_cumulant.jl:612-656) ----
#pragma unroll
  for (int n = 0; n < 9; ++n) chimera_fwd(A[3 * n], A[3 * n + 1], A[3 * n + 2], ux_eq);
#pragma unroll
  for (int iz = 0; iz < 3; ++iz)
#pragma unroll
    for (int ma = 0; ma < 3; ++ma) chimera_fwd(A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz], uy_eq);
#pragma unroll
  for (int n = 0; n < 9; ++n) chimera_fwd(A[n], A[n + 9], A[n + 18], uz_eq);

  // ---- STEP 5-7: cumulants, relaxation, reconstruction (kernel_cumulant.jl:661-781) ----
  const R k000 = A[0];
  const R inv_r = R(1) / (k000 > R(0.01) ? k000 : R(0.01));
  const R c200 = A[2] * inv_r, c020 = A[6] * inv_r, c002 = A[18] * inv_r;
  const R c110 = A[4] * inv_r, c101 = A[10] * inv_r, c011 = A[12] * inv_r;
  const R c210 = A[5] * inv_r, c120 = A[7] * inv_r, c201 = A[11] * inv_r;
  const R c021 = A[15] * inv_r, c102 = A[19] * inv_r, c012 = A[21] * inv_r;
  const R c111 = A[13] * inv_r;
  const R C220 = A[8] * inv_r - c200 * c020 - R(2) * c110 * c110;
  const R C202 = A[20] * inv_r - c200 * c002 - R(2) * c101 * c101;
  const R C022 = A[24] * inv_r - c020 * c002 - R(2) * c011 * c011;
  const R C211 = A[14] * inv_r - c200 * c011 - R(2) * c110 * c101;
  const R C121 = A[16] * inv_r - c020 * c101 - R(2) * c110 * c011;
  const R C112 = A[22] * inv_r - c002 * c110 - R(2) * c101 * c011;

  const R cs2 = R(1) / R(3);  // == float(0.333333333) in float (kernel_cumulant.jl:710)
  const R Dtr = c200 + c020 + c002;
  const R Dtr_s = (R(1) - omega_bulk) * Dtr + omega_bulk * (R(3) * cs2);
  const R D1_s = (R(1) - omega1) * (c200 - c020);
  const R D2_s = (R(1) - omega1) * (c200 - c002);
  const R c200s = (Dtr_s + D1_s + D2_s) / R(3);
  const R c020s = (Dtr_s - R(2) * D1_s + D2_s) / R(3);
  const R c002s = (Dtr_s + D1_s - R(2) * D2_s) / R(3);
  R c110s = (R(1) - omega1) * c110;
  R c101s = (R(1) - omega1) * c101;
  R c011s = (R(1) - omega1) * c011;
  if (flags & CF_LIMITER_FACTORED) {
    const R p1 = c200s * c020s, p2 = c200s * c002s, p3 = c020s * c002s;
    const R b110 = sqrt(p1 > R(0) ? p1 : R(0));
    const R b101 = sqrt(p2 > R(0) ? p2 : R(0));
    const R b011 = sqrt(p3 > R(0) ? p3 : R(0));
    c110s = c110s < -b110 ? -b110 : (c110s > b110 ? b110 : c110s);
    c101s = c101s < -b101 ? -b101 : (c101s > b101 ? b101 : c101s);
    c011s = c011s < -b011 ? -b011 : (c011s > b011 ? b011 : c011s);
  }
  const R o3 = R(1) - omega3;
  const R c210s = o3 * c210, c120s = o3 * c120, c201s = o3 * c201;
  const R c021s = o3 * c021, c102s = o3 * c102, c012s = o3 * c012, c111s = o3 * c111;
  const R C220s = (R(1) - omega4_diag) * C220;
  const R C202s = (R(1) - omega4_diag) * C202;
  const R C022s = (R(1) - omega4_diag) * C022;
  const R C211s = (R(1) - omega4) * C211;
  const R C121s = (R(1) - omega4) * C121;
  const R C112s = (R(1) - omega4) * C112;

  const R c220s = C220s + c200s * c020s + R(2) * c110s * c110s;
  const R c202s = C202s + c200s * c002s + R(2) * c101s * c101s;
  const R c022s = C022s + c020s * c002s + R(2) * c011s * c011s;
  const R c211s = C211s + c200s * c011s + R(2) * c110s * c101s;
  const R c121s = C121s + c020s * c101s + R(2) * c110s * c011s;
  const R c112s = C112s + c002s * c110s + R(2) * c101s * c011s;
  const R c221s = c200s * c021s + c020s * c201s + R(4) * c110s * c111s + R(2) * c101s * c120s + R(2) * c011s * c210s;
  const R c212s = c200s * c012s + c002s * c210s + R(2) * c110s * c102s + R(4) * c101s * c111s + R(2) * c011s * c201s;
  const R c122s = c020s * c102s + c002s * c120s + R(2) * c110s * c012s + R(4) * c011s * c111s + R(2) * c101s * c021s;
  R c222s = c200s * C022s + c020s * C202s + c002s * C220s + R(4) * (c110s * C112s + c101s * C121s + c011s * C211s);
  c222s += R(2) * (c210s * c012s + c201s * c021s + c120s * c102s) + R(4) * c111s * c111s;
  c222s += c200s * c020s * c002s + R(2) * (c200s * c011s * c011s + c020s * c101s * c101s + c002s * c110s * c110s) +
           R(8) * c110s * c101s * c011s;

  // ---- STEP 8: post-collision central moments (kernel_cumulant.jl:786-804) ----
  const R r = k000;
  A[0] = r; A[1] = R(0); A[3] = R(0); A[9] = R(0);
  A[2] = r * c200s; A[6] = r * c020s; A[18] = r * c002s;
  A[4] = r * c110s; A[10] = r * c101s; A[12] = r * c011s;
  A[5] = r * c210s; A[7] = r * c120s; A[11] = r * c201s;
  A[15] = r * c021s; A[19] = r * c102s; A[21] = r * c012s;
  A[13] = r * c111s;
  A[8] = r * c220s; A[20] = r * c202s; A[24] = r * c022s;
  A[14] = r * c211s; A[16] = r * c121s; A[22] = r * c112s;
  A[17] = r * c221s; A[23] = r * c212s; A[25] = r * c122s;
  A[26] = r * c222s;

  // ---- STEP 9: chimera backward z, y, x (kernel_cumulant.jl:810-844) ----
#pragma unroll
  for (int n = 0; n < 9; ++n) chimera_bwd(A[n], A[n + 9], A[n + 18], uz_eq);
#pragma unroll
  for (int iz = 0; iz < 3; ++iz)
#pragma unroll
    for (int ma = 0; ma < 3; ++ma) chimera_bwd(A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz], uy_eq);
#pragma unroll
  for (int n = 0; n < 9; ++n) chimera_bwd(A[3 * n], A[3 * n + 1], A[3 * n + 2], ux_eq);

  // ---- positivity limiter (kernel_cumulant.jl:849-884) ----
  if (flags & CF_LIMITER_POSITIVITY) {
    R fmin = A[0];
#pragma unroll
    for (int k = 1; k < kQ27; ++k) fmin = A[k] < fmin ? A[k] : fmin;
    if (fmin < R(0)) {
      R alpha = R(1);
#pragma unroll
      for (int k = 0; k < kQ27; ++k) {
        const R fe = feq_auto<R>(rho, ux_eq, uy_eq, uz_eq, R(q27_w(k)), R(q27_cx(k)), R(q27_cy(k)), R(q27_cz(k)), comp);
        const R fneq = A[k] - fe;
        if (fneq < R(0) && fe > R(1e-15)) {
          const R ak = fe / (fe - fneq + R(1e-15));
          alpha = ak < alpha ? ak : alpha;
        }
      }
      alpha = alpha > R(0) ? alpha : R(0);
#pragma unroll
      for (int k = 0; k < kQ27; ++k) {
        const R fe = feq_auto<R>(rho, ux_eq, uy_eq, uz_eq, R(q27_w(k)), R(q27_cx(k)), R(q27_cy(k)), R(q27_cz(k)), comp);
        A[k] = fe + alpha * (A[k] - fe);
      }
    }
  }

  // ---- STEP 10: Guo forcing + store (kernel_cumulant.jl:889-908) ----
  const bool forced = G && (Fx != R(0) || Fy != R(0) || Fz != R(0));
  const R gpre = R(1) - R(0.5) * omega1;
#pragma unroll
  for (int k = 0; k < kQ27; ++k) {
    const R w = R(q27_w(k)), iw = R(1.0 / q27_w(k));
    R fc = A[k];
    if (forced) {
      const R cxf = R(q27_cx(k)), cyf = R(q27_cy(k)), czf = R(q27_cz(k));
      const R cu = cxf * ux_eq + cyf * uy_eq + czf * uz_eq;
      const R ft = w * R(3) * ((cxf - ux + R(3) * cu * cxf) * Fx + (cyf - uy + R(3) * cu * cyf) * Fy +
                               (czf - uz + R(3) * cu * czf) * Fz);
      fc = A[k] + gpre * ft;
    }
    if (store_post) static_cast<S*>(a.f_post)[own + k * kst] = Codec<S>::enc(fc, w, iw);
    fout[own + k * kst] = Codec<S>::enc(fc, w, iw);
  }
}

template <class S, class R>
__global__ void __launch_bounds__(128) k_cumulant_d3q27(const StepArgs a) {
  __shared__ int32_t s_nbr[32];
  __shared__ CaseParams s_cp;
  __shared__ int4 s_info;
  __shared__ uint32_t s_bflags;
  __shared__ double s_mom[4][3];

  const int tid = threadIdx.x;
  const int b = a.block_base + (int)(blockIdx.x >> 2);
  const int slab = blockIdx.x & 3;
  if (tid < 27) s_nbr[tid] = a.nbr[(int64_t)b * 27 + tid];
  if (tid == 32) {
    s_info = a.binfo[b];
    s_bflags = a.bflags[b];
  }
  __syncthreads();
  if (tid < (int)(sizeof(CaseParams) / 4)) {
    const uint32_t* src = a.cases ? reinterpret_cast<const uint32_t*>(a.cases + s_info.w)
                                  : reinterpret_cast<const uint32_t*>(&a.p0);
    reinterpret_cast<uint32_t*>(&s_cp)[tid] = src[tid];
  }
  __syncthreads();

  const int x = tid & 7, y = (tid >> 3) & 7, z = 2 * slab + (tid >> 6);
  const uint32_t bflags = s_bflags;
  // 1-based global coordinates of local cell (0,0,0) + 1 (kernel_cumulant.jl:181-183)
  const int gx0 = (s_info.x - 1) * kBS + 1, gy0 = (s_info.y - 1) * kBS + 1, gz0 = (s_info.z - 1) * kBS + 1;
  double mx = 0.0, my = 0.0, mz = 0.0;
  if ((bflags & BF_INTERIOR) && !(bflags & BF_NEAR_SOLID)) {
    cell_step<S, R, false>(a, s_cp, s_nbr, b, gx0, gy0, gz0, bflags, x, y, z, mx, my, mz);
  } else {
    cell_step<S, R, true>(a, s_cp, s_nbr, b, gx0, gy0, gz0, bflags, x, y, z, mx, my, mz);
  }

  if ((s_cp.flags & CF_COLLECT) && a.force_part) {
    // deterministic FP64 reduction: warp tree, then the four warps in order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mx += __shfl_down_sync(0xffffffffu, mx, o);
      my += __shfl_down_sync(0xffffffffu, my, o);
      mz += __shfl_down_sync(0xffffffffu, mz, o);
    }
    if ((tid & 31) == 0) { s_mom[tid >> 5][0] = mx; s_mom[tid >> 5][1] = my; s_mom[tid >> 5][2] = mz; }
    __syncthreads();
    if (tid < 3) {
      const double s = ((s_mom[0][tid] + s_mom[1][tid]) + s_mom[2][tid]) + s_mom[3][tid];
      a.force_part[(int64_t)blockIdx.x * 3 + tid] = s;
    }
  }
}

// Launch over `n_blocks` blocks starting at a.block_base.
template <class S, class R>
cudaError_t launch_cumulant(const StepArgs& a, int n_blocks, cudaStream_t st) {
  if (n_blocks <= 0) return cudaSuccess;
  k_cumulant_d3q27<S, R><<<dim3((unsigned)n_blocks * 4u), dim3(128), 0, st>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_cumulant<float, float>(const StepArgs&, int, cudaStream_t);
template cudaError_t launch_cumulant<__half, float>(const StepArgs&, int, cudaStream_t);
template cudaError_t launch_cumulant<__nv_bfloat16, float>(const StepArgs&, int, cudaStream_t);
template cudaError_t launch_cumulant<double, double>(const StepArgs&, int, cudaStream_t);

}  // namespace oal
