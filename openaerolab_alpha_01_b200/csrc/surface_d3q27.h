// surface_d3q27.h — internal interface of the surface-stress mapping (surface_d3q27.cu) for the
// level API (level.cu). Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace oal {

struct SurfArgs {
  const float* tri;     // [n * 7]: centroid x, y, z, unit normal x, y, z, area (cell units)
  int32_t n;
  const void* rho;      // compute type (double when dbl), [nb * 512]
  const void* vel;      // compute type, component stride vcs
  int64_t vcs;
  const int32_t* ptr;   // [dim_x * dim_y * dim_z], x fastest: 1-based block, 0 = none
  int32_t dim_x, dim_y, dim_z;
  const int32_t* mslot; // solid masks: bit 13 of cmask[mslot[b] * 512 + cell]
  const uint32_t* cmask;
  int32_t radius, recover;
  float tau, c_wale, nu_bg, pscale, sscale, cs2;
  float mcx, mcy, mcz;  // moment centre
  float* out;           // [n * 6]: p, tau_x, tau_y, tau_z, normal sign, wall distance
  double* part;         // [n * 9]: pressure force, viscous force, moment (per triangle)
};

// Maps the stresses of every triangle and sums their forces and moments into d_out9.
cudaError_t launch_surface(const SurfArgs& a, bool dbl, double* d_out9, cudaStream_t st);

}  // namespace oal
