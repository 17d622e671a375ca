// kbc_d3q39.h — internal interface between the level API (level.cu) and the D3Q39 entropic KBC
// level state (kbc_d3q39.cu). Not part of the C ABI.
#pragma once
#include <stdint.h>
#include "../../include/oal.h"

struct KbcLevel;

// What a D3Q39 level reads of its geometry. The neighbour table is ghost-indexed: a missing
// neighbour block is one of n_ghost ghost blocks (ids nb .. nb + n_ghost - 1), whose populations
// the level's face fill writes before each step; solid cells come from the per-block masks of the
// D3Q27 geometry (bit 13: the cell itself; bits 4, 10, 12, 14, 16, 22: its face neighbours).
struct KbcGeometry {
  int32_t nb = 0, n_ghost = 0, nx = 0, ny = 0, nz = 0;
  const int32_t* d_nbr = nullptr;       // [nb*27] 0-based, the block itself at entry 13
  const int32_t* h_nbr = nullptr;       // host copy
  const void* d_binfo = nullptr;        // [nb] int4 (bx, by, bz, case), 1-based
  const uint32_t* h_bflags = nullptr;   // [nb] host
  const uint32_t* d_bflags = nullptr;   // [nb]
  const int32_t* d_mslot = nullptr;     // [nb] mask slot or -1
  const uint32_t* d_cmask = nullptr;    // [slots*512]
  bool has_solid = false;
  const float* d_sponge = nullptr;      // [nb*512] sponge strength or null
  const float* d_wdist = nullptr;       // [nb*512] wall distance (NaN = none) or null
};
oal_status kbc_create(int device, const KbcGeometry& G, KbcLevel** out);
// exp and log of the step: exact = the software routines shared with the CPU restatement
// (bit-identical to it), otherwise CUDA's expf / logf
void kbc_set_exact_math(KbcLevel* L, bool exact);
void kbc_destroy(KbcLevel* L);
oal_status kbc_init_equilibrium(KbcLevel* L, const double* rho_host, const double* vel_host);
oal_status kbc_set_state(KbcLevel* L, const double* f_host, const double* rho_host, const double* vel_host);
oal_status kbc_get_state(KbcLevel* L, double* f_host, double* rho_host, double* vel_host);
oal_status kbc_lambda(KbcLevel* L, float* get_host, const float* set_host);
oal_status kbc_step(KbcLevel* L, const oal_step_params* p, void* stream);
oal_status kbc_advance(KbcLevel* L, const oal_step_params* p, int32_t n, void* stream);
oal_status kbc_mass_momentum(KbcLevel* L, double out[4]);
oal_status kbc_device_state(KbcLevel* L, void** f, void** rho, void** vel);
int64_t kbc_device_bytes(const KbcLevel* L);
oal_status kbc_layout(const KbcLevel* L, int64_t out[6]);
