// kbc_d3q39.h — internal interface between the level API (level.cu) and the D3Q39 entropic KBC
// level state (kbc_d3q39.cu). Not part of the C ABI.
#pragma once
#include <stdint.h>
#include "../../include/oal.h"

struct KbcLevel;

// A D3Q39 level on a geometry whose blocks all have their 26 neighbours (d_nbr: device [nb*27],
// 0-based, the block itself at entry 13).
oal_status kbc_create(int device, int32_t nb, const int32_t* d_nbr, KbcLevel** out);
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
