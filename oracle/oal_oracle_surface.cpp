// oal_oracle_surface.cpp — CPU ORACLE (test infrastructure only; never linked into the product).
//
// A plain C++ restatement of the reference's surface-stress force mapping with its default
// Prandtl force method (OpenAeroLab, Julia, src/forces/surface.jl):
//   get_cell_at_position ......... :271-307
//   trilinear_sample_flow ........ :502-634
//   compute_stress_from_cell ..... :180-269 (athermal: T = 1)
//   map_stresses_kernel! ......... :636-1031 (probe walk, Shepard pressure, normal recovery of
//                                  closed bodies, shell-search fallback)
//   integrate_forces_kernel! ..... :1265-1331 (per-triangle pressure / viscous force and moment)
// Float32 arithmetic in the reference's operation order (built with -ffp-contract=off), dx = 1
// (cell units), mesh offset 0. Parity: the reference's GPU path cannot run here (Julia); the
// restatement is checked against closed forms in tests/test_surface.py.
#include <cmath>
#include <cstdint>

namespace {

struct Field {
  const float* rho;
  const float* vel;
  int64_t vcs;
  const uint8_t* obstacle;
  const int32_t* ptr;
  int dim_x, dim_y, dim_z;
};

int64_t cell_at(const Field& F, int gx, int gy, int gz) {
  if (gx < 1 || gy < 1 || gz < 1) return -1;
  const int bx = (gx - 1) / 8 + 1, by = (gy - 1) / 8 + 1, bz = (gz - 1) / 8 + 1;
  if (bx < 1 || bx > F.dim_x || by < 1 || by > F.dim_y || bz < 1 || bz > F.dim_z) return -1;
  const int32_t b = F.ptr[(bx - 1) + (int64_t)F.dim_x * ((by - 1) + (int64_t)F.dim_y * (bz - 1))];
  if (b <= 0) return -1;
  const int lx = (gx - 1) % 8, ly = (gy - 1) % 8, lz = (gz - 1) % 8;
  return (int64_t)(b - 1) * 512 + lx + 8 * ly + 64 * lz;
}

float clampf(float v, float lo, float hi) { return v > hi ? hi : (v < lo ? lo : v); }

bool trilinear(const Field& F, float px, float py, float pz, float& r, float& u, float& v, float& w, float& wq) {
  const float inv_dx = 1.0f / 1.0f;
  const float fx = px * inv_dx - 0.5f, fy = py * inv_dx - 0.5f, fz = pz * inv_dx - 0.5f;
  const int ix0 = (int)std::floor(fx) + 1, iy0 = (int)std::floor(fy) + 1, iz0 = (int)std::floor(fz) + 1;
  const float wx = clampf(fx - (float)(ix0 - 1), 0.0f, 1.0f);
  const float wy = clampf(fy - (float)(iy0 - 1), 0.0f, 1.0f);
  const float wz = clampf(fz - (float)(iz0 - 1), 0.0f, 1.0f);
  const float w0x = 1.0f - wx, w1x = wx, w0y = 1.0f - wy, w1y = wy, w0z = 1.0f - wz, w1z = wz;
  float ra = 0.0f, ua = 0.0f, va = 0.0f, wa_ = 0.0f, wsum = 0.0f;
  // the eight corners in the reference's order: x fastest, then y, then z
  const int offs[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  for (int c = 0; c < 8; ++c) {
    const float wk = (offs[c][0] ? w1x : w0x) * (offs[c][1] ? w1y : w0y) * (offs[c][2] ? w1z : w0z);
    const int64_t e = cell_at(F, ix0 + offs[c][0], iy0 + offs[c][1], iz0 + offs[c][2]);
    if (e >= 0 && !F.obstacle[e]) {
      ra += wk * F.rho[e];
      ua += wk * F.vel[e];
      va += wk * F.vel[e + F.vcs];
      wa_ += wk * F.vel[e + 2 * F.vcs];
      wsum += wk;
    }
  }
  r = 1.0f; u = v = w = 0.0f; wq = 0.0f;
  if (wsum > 0.01f) {
    const float inv = 1.0f / wsum;
    const float ro = ra * inv, uo = ua * inv, vo = va * inv, wo = wa_ * inv;
    if (!std::isfinite(ro) || !std::isfinite(uo) || !std::isfinite(vo) || !std::isfinite(wo)) return false;
    r = ro; u = uo; v = vo; w = wo; wq = wsum;
    return true;
  }
  return false;
}

struct Stress { float p, tx, ty, tz; };

Stress stress_from_cell(float rho, float ux, float uy, float uz, float nx, float ny, float nz, float dist, float tau,
                        float pscale, float sscale, float c_wale, float nu_bg, float cs2) {
  Stress z{0.0f, 0.0f, 0.0f, 0.0f};
  if (!std::isfinite(rho) || rho < 0.01f || rho > 10.0f) return z;
  if (!std::isfinite(ux) || !std::isfinite(uy) || !std::isfinite(uz)) return z;
  const float usq = ux * ux + uy * uy + uz * uz;
  if (usq > 100.0f) return z;
  const float p_gauge = (rho * 1.0f - 1.0f) * cs2;
  const float p_phys = p_gauge * pscale;
  const float udn = ux * nx + uy * ny + uz * nz;
  const float utx = ux - udn * nx, uty = uy - udn * ny, utz = uz - udn * nz;
  const float ut = std::sqrt(utx * utx + uty * uty + utz * utz);
  const float nu_mol = (tau - 0.5f) * cs2;
  float nu_sgs = 0.0f;
  const float dwe = dist > 1.0f ? dist : 1.0f;
  if (c_wale > 0.0f && ut > 1.0e-10f) {
    const float S = ut / dwe;
    nu_sgs = (c_wale * c_wale) * S;
  }
  if (nu_sgs < nu_bg) nu_sgs = nu_bg;
  if (nu_sgs > 20.0f * nu_mol) nu_sgs = 20.0f * nu_mol;
  const float nu_eff = nu_mol + nu_sgs;
  float sx = 0.0f, sy = 0.0f, sz = 0.0f;
  if (ut > 1.0e-10f && dist > 0.01f) {
    const float tlat = rho * nu_eff * ut / dwe;
    const float tphys = tlat * sscale;
    sx = (utx / ut) * tphys; sy = (uty / ut) * tphys; sz = (utz / ut) * tphys;
  }
  if (!std::isfinite(p_phys) || !std::isfinite(sx) || !std::isfinite(sy) || !std::isfinite(sz)) return z;
  return Stress{p_phys, sx, sy, sz};
}

}  // namespace

extern "C" {

// Per triangle: out[6] = pressure, shear x, y, z, normal sign, probe wall distance; part[9] =
// pressure force, viscous force and moment about mc (zeros where the pressure is not finite).
void ora_surface_map(int32_t n, const float* tri, const float* rho, const float* vel, int64_t vcs,
                     const uint8_t* obstacle, const int32_t* ptr, int32_t dim_x, int32_t dim_y, int32_t dim_z,
                     int32_t radius, int32_t recover, float tau, float c_wale, float nu_bg, float pscale, float sscale,
                     float cs2, const float* mc, float* out, double* part) {
  const Field F{rho, vel, vcs, obstacle, ptr, dim_x, dim_y, dim_z};
  const float dx = 1.0f;
  for (int32_t i = 0; i < n; ++i) {
    const float* t = tri + (int64_t)i * 7;
    const float tx = t[0] + 0.0f, ty = t[1] + 0.0f, tz = t[2] + 0.0f;
    float nx = t[3], ny = t[4], nz = t[5];
    float best_rho = 1.0f, best_u = 0.0f, best_v = 0.0f, best_w = 0.0f;
    float best_wd = (float)(radius + 1), best_q = 0.0f;
    bool found = false;
    float p_rho = 0.0f, p_T = 0.0f, p_w = 0.0f;
    const float min_quality = 0.25f;
    const int pmax = radius < 4 ? radius : 4;
    for (int k = 1; k <= radius; ++k) {
      const float d = (float)k + 0.5f;
      float r, u, v, w, q;
      const bool ok = trilinear(F, tx + nx * d * dx, ty + ny * d * dx, tz + nz * d * dx, r, u, v, w, q);
      if (ok && q >= min_quality && k <= pmax) {
        p_rho += q * r;
        p_T += q * 1.0f;
        p_w += q;
      }
      if (ok && q >= min_quality) {
        if (!found) {
          best_rho = r; best_u = u; best_v = v; best_w = w; best_wd = d; best_q = q;
          found = true;
        }
        if (k >= pmax) break;
      } else if (ok && q > best_q && !found) {
        best_rho = r; best_u = u; best_v = v; best_w = w; best_wd = d; best_q = q;
        found = true;
      }
    }
    float sign = 1.0f;
    if (!found && recover) {
      for (int k = 1; k <= pmax; ++k) {
        const float d = (float)k + 0.5f;
        float r, u, v, w, q;
        const bool ok = trilinear(F, tx - nx * d * dx, ty - ny * d * dx, tz - nz * d * dx, r, u, v, w, q);
        if (ok && q >= min_quality) {
          p_rho += q * r;
          p_T += q * 1.0f;
          p_w += q;
          if (!found) {
            best_rho = r; best_u = u; best_v = v; best_w = w; best_wd = d; best_q = q;
            found = true;
            sign = -1.0f;
          }
        }
      }
      if (sign < 0.0f) { nx = -nx; ny = -ny; nz = -nz; }
    }
    if (!found) {
      const int gx = (int)std::floor(tx / dx) + 1, gy = (int)std::floor(ty / dx) + 1, gz = (int)std::floor(tz / dx) + 1;
      float best_d2 = 1e10f;
      for (int rad = 1; rad <= radius; ++rad) {
        if (found) break;
        for (int dz = -rad; dz <= rad; ++dz)
          for (int dy = -rad; dy <= rad; ++dy)
            for (int ddx = -rad; ddx <= rad; ++ddx) {
              const bool shell = std::abs(ddx) == rad || std::abs(dy) == rad || std::abs(dz) == rad;
              if (!shell) continue;
              const int cx = gx + ddx, cy = gy + dy, cz = gz + dz;
              const int64_t e = cell_at(F, cx, cy, cz);
              if (e < 0 || obstacle[e]) continue;
              const float cr = rho[e];
              if (!std::isfinite(cr) || cr < 0.01f || cr > 100.0f) continue;
              const float ccx = ((float)cx - 0.5f) * dx, ccy = ((float)cy - 0.5f) * dx, ccz = ((float)cz - 0.5f) * dx;
              const float dxp = ccx - tx, dyp = ccy - ty, dzp = ccz - tz;
              const float dn = dxp * nx + dyp * ny + dzp * nz;
              if (dn <= 0.0f) continue;
              const float d2 = dxp * dxp + dyp * dyp + dzp * dzp;
              if (d2 < best_d2) {
                best_d2 = d2;
                best_rho = cr; best_u = vel[e]; best_v = vel[e + vcs]; best_w = vel[e + 2 * vcs];
                best_wd = dn / dx;
                found = true;
              }
            }
      }
    }
    const float prho = p_w > 0.5f ? p_rho / p_w : best_rho;
    const float pT = p_w > 0.5f ? p_T / p_w : 1.0f;
    float p = NAN, sx = 0.0f, sy = 0.0f, sz = 0.0f;
    if (found) {
      const float wd = best_wd > 0.5f ? best_wd : 0.5f;
      const Stress s = stress_from_cell(best_rho, best_u, best_v, best_w, nx, ny, nz, wd, tau, pscale, sscale, c_wale,
                                        nu_bg, cs2);
      p = s.p; sx = s.tx; sy = s.ty; sz = s.tz;
      if (std::isfinite(prho) && prho >= 0.01f && prho <= 10.0f && std::isfinite(pT) && pT >= 0.1f && pT <= 10.0f)
        p = (prho * pT - 1.0f) * cs2 * pscale;
    }
    float* o = out + (int64_t)i * 6;
    o[0] = p; o[1] = sx; o[2] = sy; o[3] = sz; o[4] = sign; o[5] = found ? best_wd * dx : 0.0f;
    double* q = part + (int64_t)i * 9;
    for (int c = 0; c < 9; ++c) q[c] = 0.0;
    if (std::isfinite(p) && std::isfinite(sx) && std::isfinite(sy) && std::isfinite(sz)) {
      const float mx = t[3] * sign, my = t[4] * sign, mz = t[5] * sign, A = t[6];
      const float fpx = -p * mx * A, fpy = -p * my * A, fpz = -p * mz * A;
      const float fvx = sx * A, fvy = sy * A, fvz = sz * A;
      const float fx = fpx + fvx, fy = fpy + fvy, fz = fpz + fvz;
      const float rx = tx - mc[0], ry = ty - mc[1], rz = tz - mc[2];
      q[0] = fpx; q[1] = fpy; q[2] = fpz; q[3] = fvx; q[4] = fvy; q[5] = fvz;
      q[6] = ry * fz - rz * fy; q[7] = rz * fx - rx * fz; q[8] = rx * fy - ry * fx;
    }
  }
}

}  // extern "C"
